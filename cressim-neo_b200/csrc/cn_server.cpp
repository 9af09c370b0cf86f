// cn_server.cpp -- the serving loop over a cn_batch (no reference counterpart).
//
// Scenes are registered once (the server keeps a host copy of each) and become resident in the
// batch's device pool when a request needs them and the memory budget allows; when the budget is
// full, resident scenes with no pending work are written back to their host copies and evicted,
// least recently used first.  Requests ask for k frames of one scene, each frame with its own
// kinematic tool target.  Every tick steps one frame of every resident scene that has pending
// work (continuous batching: a request submitted while ticks are running joins the next tick),
// and the host prepares and launches tick k+1 before it waits for tick k, so the device is never
// idle between ticks.  Completion times are taken when a request's last tick is seen finished.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_internal.h"

using cn::setError;

namespace {

// A deep host copy of one scene's SoA (the arrays the batch reads), with a view into it.
struct SceneStore {
    std::vector<float> x, v, radii, contactMaterials, bodyPos, bodyRot, bodyLin, bodyAng, bodyScale, bodyInvI,
        bodyKinPos, bodyKinRot, colMat;
    std::vector<uint32_t> kinds, meta, matIdx, fluidMatIdx, ownerTypes, ownerIdx, adjOff, adjCnt, bodyTypes,
        bodyKinFlags, bodyColRanges, bodyColIdx;
    std::vector<cn_soft_edge> edges;
    std::vector<cn_soft_tet> tets;
    std::vector<cn_collider_geometry> colGeo;
    std::vector<cn_collider_broadphase> colBp;
    cn_world_soa soa{};

    template <class T> static void copy(std::vector<T> &dst, const T *src, size_t n)
    {
        dst.assign(src ? src : nullptr, src ? src + n : nullptr);
    }
    void assign(const cn_world_soa &w)
    {
        const size_t N = w.particle_count, B = w.rigid_body_count, C = w.collider_count;
        copy(x, w.positions_inv_mass, 4 * N);
        copy(v, w.velocities, 4 * N);
        copy(radii, w.radii, N);
        copy(kinds, w.kinds, N);
        copy(meta, w.metadata, 4 * N);
        copy(matIdx, w.material_indices, N);
        copy(fluidMatIdx, w.fluid_material_indices, N);
        copy(ownerTypes, w.owner_types, N);
        copy(ownerIdx, w.owner_indices, N);
        copy(adjOff, w.adjacency_offsets, N);
        copy(adjCnt, w.adjacency_counts, N);
        copy(contactMaterials, w.contact_materials, 4 * size_t(w.contact_material_count));
        copy(edges, w.edges, w.edge_count);
        copy(tets, w.tets, w.tet_count);
        copy(bodyPos, w.body_positions_inv_mass, 4 * B);
        copy(bodyRot, w.body_orientations, 4 * B);
        copy(bodyLin, w.body_linear_velocities, 4 * B);
        copy(bodyAng, w.body_angular_velocities, 4 * B);
        copy(bodyScale, w.body_scales, 4 * B);
        copy(bodyInvI, w.body_inverse_inertia, 4 * B);
        copy(bodyTypes, w.body_types, B);
        copy(bodyKinPos, w.body_kinematic_target_positions, 4 * B);
        copy(bodyKinRot, w.body_kinematic_target_orientations, 4 * B);
        copy(bodyKinFlags, w.body_kinematic_target_flags, B);
        copy(bodyColRanges, w.body_collider_ranges, 2 * B);
        copy(bodyColIdx, w.body_collider_indices, w.body_collider_index_count);
        copy(colGeo, w.collider_geometry, C);
        copy(colBp, w.collider_broadphase, C);
        copy(colMat, w.collider_materials, 4 * C);
        soa = cn_world_soa{};
        soa.particle_count = w.particle_count;
        soa.positions_inv_mass = x.data();
        soa.velocities = v.data();
        soa.radii = radii.data();
        soa.kinds = kinds.data();
        soa.metadata = meta.data();
        soa.material_indices = matIdx.data();
        soa.fluid_material_indices = fluidMatIdx.data();
        soa.owner_types = ownerTypes.data();
        soa.owner_indices = ownerIdx.data();
        soa.adjacency_offsets = adjOff.data();
        soa.adjacency_counts = adjCnt.data();
        soa.particle_grid_cell_size = w.particle_grid_cell_size;
        soa.contact_material_count = w.contact_material_count;
        soa.contact_materials = contactMaterials.data();
        soa.edge_count = w.edge_count;
        soa.edges = edges.data();
        soa.tet_count = w.tet_count;
        soa.tets = tets.data();
        soa.rigid_body_count = w.rigid_body_count;
        soa.body_positions_inv_mass = bodyPos.data();
        soa.body_orientations = bodyRot.data();
        soa.body_linear_velocities = bodyLin.data();
        soa.body_angular_velocities = bodyAng.data();
        soa.body_scales = bodyScale.data();
        soa.body_inverse_inertia = bodyInvI.data();
        soa.body_types = bodyTypes.data();
        soa.body_kinematic_target_positions = bodyKinPos.data();
        soa.body_kinematic_target_orientations = bodyKinRot.data();
        soa.body_kinematic_target_flags = bodyKinFlags.data();
        soa.body_collider_ranges = bodyColRanges.data();
        soa.body_collider_indices = bodyColIdx.data();
        soa.body_collider_index_count = w.body_collider_index_count;
        soa.collider_count = w.collider_count;
        soa.collider_geometry = colGeo.data();
        soa.collider_broadphase = colBp.data();
        soa.collider_materials = colMat.data();
    }
};

struct Request {
    uint64_t id = 0;
    uint32_t scene = 0, steps = 0, issued = 0, toolBody = 0;
    std::vector<float> targets; // steps x 7 (position xyz, orientation xyzw), may be empty
    double submit = 0.0, firstTick = -1.0;
};

struct SceneSlot {
    SceneSlot() = default;
    SceneSlot(const SceneSlot &) = delete;
    SceneSlot &operator=(const SceneSlot &) = delete;
    SceneStore store;
    // the scene's upload image, built at registration; admission refreshes its state sections
    cn::SceneImage image;
    cn_status imageStatus = CN_OK;
    std::string imageError;
    bool resident = false;
    uint32_t batchId = 0;
    std::deque<Request> queue;
    uint64_t lastTick = 0;
};

struct Tick {
    cudaEvent_t begin = nullptr, end = nullptr;
    std::vector<cn_request_done> finishing; // requests whose last frame is in this tick
    bool inFlight = false;
};

} // namespace

struct cn_server {
    cn_batch *batch = nullptr;
    cn_server_desc desc{};
    // Slots are heap-allocated: each store's SoA view points into the store's own vectors, so
    // a slot must never be copied or moved.
    std::vector<std::unique_ptr<SceneSlot>> scenes;
    std::vector<cn_request_done> done;
    Tick ticks[2];
    int cur = 0;
    uint64_t nextRequest = 1, tickCount = 0, sceneSteps = 0, particleSubsteps = 0, admissions = 0, evictions = 0;
    uint64_t completed = 0;
    double gpuMs = 0.0;
    std::vector<float> tickMs;
    uint32_t substeps = 1;
    cudaStream_t ownStream = nullptr; // ticks run here when the caller passes no stream
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// Makes `id` resident, evicting idle resident scenes (least recently stepped first) when the
// budget or the pool is full.  Returns false if it has to wait for room.  A scene already taken
// into the tick being assembled (lastTick = the coming tick) is not idle even when that tick
// issues its request's last frame: evicting it would drop it from the tick and hand its batch id
// to the scene being admitted, which the tick would then step twice.
bool admit(cn_server *srv, uint32_t id)
{
    SceneSlot &sc = *srv->scenes[id];
    for (;;) {
        uint32_t bid = 0;
        if (sc.imageStatus != CN_OK) {
            cn::setError(sc.imageStatus, sc.imageError);
            return false;
        }
        cn::refreshSceneImage(sc.store.soa, sc.image);
        const cn_status st = cn::batchAdmitImage(srv->batch, sc.image, &bid);
        if (st == CN_OK) {
            sc.resident = true;
            sc.batchId = bid;
            ++srv->admissions;
            return true;
        }
        if (st != CN_ERR_CAPACITY) return false;
        int victim = -1;
        for (uint32_t k = 0; k < srv->scenes.size(); ++k) {
            const SceneSlot &o = *srv->scenes[k];
            if (!o.resident || !o.queue.empty() || k == id || o.lastTick > srv->tickCount) continue;
            if (victim < 0 || o.lastTick < srv->scenes[victim]->lastTick) victim = int(k);
        }
        if (victim < 0) return false;
        SceneSlot &v = *srv->scenes[victim];
        if (cn_batch_export_scene(srv->batch, v.batchId, &v.store.soa) != CN_OK) return false;
        if (cn_batch_remove_scene(srv->batch, v.batchId) != CN_OK) return false;
        v.resident = false;
        ++srv->evictions;
    }
}

void retire(cn_server *srv, Tick &t)
{
    if (!t.inFlight) return;
    cudaEventSynchronize(t.end);
    const double when = srv->now();
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, t.begin, t.end) == cudaSuccess) {
        srv->gpuMs += ms;
        srv->tickMs.push_back(ms);
    }
    for (auto &r : t.finishing) {
        r.done_s = when;
        srv->done.push_back(r);
        ++srv->completed;
    }
    t.finishing.clear();
    t.inFlight = false;
}

} // namespace

extern "C" {

CN_API void cn_server_desc_defaults(cn_server_desc *d)
{
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->frame_dt = 1.0f / 60.0f;
}

CN_API cn_status cn_server_create(cn_batch *batch, const cn_server_desc *d, uint32_t substeps, cn_server **out)
{
    if (!batch || !d || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_create: null argument");
    if (!(d->frame_dt > 0.0f)) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_create: frame_dt must be > 0");
    auto *srv = new cn_server();
    srv->batch = batch;
    srv->desc = *d;
    srv->substeps = std::max<uint32_t>(substeps, 1u);
    for (auto &t : srv->ticks) {
        cudaEventCreate(&t.begin);
        cudaEventCreate(&t.end);
    }
    cudaStreamCreateWithFlags(&srv->ownStream, cudaStreamNonBlocking);
    *out = srv;
    return CN_OK;
}

CN_API void cn_server_destroy(cn_server *srv)
{
    if (!srv) return;
    for (auto &t : srv->ticks) {
        if (t.inFlight) cudaEventSynchronize(t.end);
        cudaEventDestroy(t.begin);
        cudaEventDestroy(t.end);
    }
    for (auto &sc : srv->scenes)
        if (sc->resident) cn_batch_remove_scene(srv->batch, sc->batchId);
    if (srv->ownStream) cudaStreamDestroy(srv->ownStream);
    delete srv;
}

CN_API cn_status cn_server_register_scene(cn_server *srv, const cn_world_soa *w, uint32_t *scene)
{
    if (!srv || !w || !scene) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_register_scene: null argument");
    srv->scenes.push_back(std::make_unique<SceneSlot>());
    SceneSlot &sc = *srv->scenes.back();
    sc.store.assign(*w);
    sc.imageStatus = cn::buildSceneImage(sc.store.soa, cn::batchRigidPairsPerParticle(srv->batch),
                                          cn::batchColoured(srv->batch), sc.image);
    if (sc.imageStatus != CN_OK) sc.imageError = cn_last_error();
    cn::clearError();
    *scene = uint32_t(srv->scenes.size() - 1);
    return CN_OK;
}

CN_API cn_status cn_server_admit(cn_server *srv, uint32_t scene)
{
    if (!srv || scene >= srv->scenes.size()) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_admit: bad scene");
    if (srv->scenes[scene]->resident) return CN_OK;
    if (!admit(srv, scene)) return setError(CN_ERR_CAPACITY, "cn_server_admit: no room within the budget");
    return CN_OK;
}

CN_API cn_status cn_server_submit(cn_server *srv, uint32_t scene, uint32_t steps, uint32_t tool_body,
                                  const float *tool_targets, uint64_t *request_id)
{
    if (!srv || scene >= srv->scenes.size() || steps == 0)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_submit: bad scene or zero steps");
    SceneSlot &sc = *srv->scenes[scene];
    if (tool_targets && tool_body >= sc.store.soa.rigid_body_count)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_submit: tool body out of range");
    Request r;
    r.id = srv->nextRequest++;
    r.scene = scene;
    r.steps = steps;
    r.toolBody = tool_body;
    if (tool_targets) r.targets.assign(tool_targets, tool_targets + size_t(steps) * 7u);
    r.submit = srv->now();
    sc.queue.push_back(std::move(r));
    if (request_id) *request_id = sc.queue.back().id;
    return CN_OK;
}

CN_API cn_status cn_server_tick(cn_server *srv, void *stream, uint32_t *stepped)
{
    if (!srv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_tick: null server");
    if (stepped) *stepped = 0;
    // events and the batch step on one stream, so the tick's events bracket its work
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : srv->ownStream;
    Tick &t = srv->ticks[srv->cur];
    retire(srv, t); // the tick before the previous one: long finished in steady state
    std::vector<uint32_t> ids;
    const uint32_t cap = srv->desc.max_scenes_per_tick ? srv->desc.max_scenes_per_tick : 0xffffffffu;
    for (uint32_t k = 0; k < srv->scenes.size() && ids.size() < cap; ++k) {
        SceneSlot &sc = *srv->scenes[k];
        if (sc.queue.empty()) continue;
        if (!sc.resident && !admit(srv, k)) continue;
        Request &r = sc.queue.front();
        if (!r.targets.empty()) {
            const float *tg = r.targets.data() + size_t(r.issued) * 7u;
            const cn_status s2 = cn_batch_set_kinematic_target(srv->batch, sc.batchId, r.toolBody, tg, tg + 3);
            if (s2 != CN_OK) return s2;
        }
        ids.push_back(sc.batchId);
        const double when = srv->now();
        if (r.firstTick < 0.0) r.firstTick = when;
        ++r.issued;
        sc.lastTick = srv->tickCount + 1;
        srv->particleSubsteps += uint64_t(sc.store.soa.particle_count) * srv->substeps;
        if (r.issued == r.steps) {
            cn_request_done d{};
            d.request_id = r.id;
            d.scene = k;
            d.steps = r.steps;
            d.submit_s = r.submit;
            d.first_tick_s = r.firstTick;
            t.finishing.push_back(d);
            sc.queue.pop_front();
        }
    }
    if (ids.empty()) {
        retire(srv, srv->ticks[srv->cur ^ 1]);
        return CN_OK;
    }
    cudaEventRecord(t.begin, st);
    const cn_status s3 = cn_batch_step(srv->batch, ids.data(), uint32_t(ids.size()), srv->desc.frame_dt, st);
    if (s3 != CN_OK) return s3;
    cudaEventRecord(t.end, st);
    t.inFlight = true;
    ++srv->tickCount;
    srv->sceneSteps += ids.size();
    if (stepped) *stepped = uint32_t(ids.size());
    // launch first, then wait for the previous tick: the device always has the next tick queued
    srv->cur ^= 1;
    retire(srv, srv->ticks[srv->cur]);
    return CN_OK;
}

CN_API cn_status cn_server_drain(cn_server *srv, void *stream)
{
    if (!srv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_drain: null server");
    for (;;) {
        bool pending = false;
        for (const auto &sc : srv->scenes) pending = pending || !sc->queue.empty();
        if (!pending) break;
        uint32_t n = 0;
        const cn_status st = cn_server_tick(srv, stream, &n);
        if (st != CN_OK) return st;
        if (n == 0) return setError(CN_ERR_CAPACITY, "cn_server_drain: pending scenes cannot be admitted");
    }
    for (auto &t : srv->ticks) retire(srv, t);
    return CN_OK;
}

CN_API cn_status cn_server_poll(cn_server *srv, cn_request_done *out, uint32_t capacity, uint32_t *count)
{
    if (!srv || !count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_poll: null argument");
    const uint32_t n = uint32_t(std::min<size_t>(srv->done.size(), capacity));
    if (out)
        for (uint32_t k = 0; k < n; ++k) out[k] = srv->done[k];
    srv->done.erase(srv->done.begin(), srv->done.begin() + n);
    *count = n;
    return CN_OK;
}

CN_API cn_status cn_server_get_stats(cn_server *srv, cn_server_stats *out)
{
    if (!srv || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_get_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    out->ticks = srv->tickCount;
    out->scene_steps = srv->sceneSteps;
    out->particle_substeps = srv->particleSubsteps;
    out->admissions = srv->admissions;
    out->evictions = srv->evictions;
    out->completed = srv->completed;
    for (const auto &sc : srv->scenes) {
        out->pending += sc->queue.size();
        if (sc->resident) ++out->resident_scenes;
    }
    out->registered_scenes = uint32_t(srv->scenes.size());
    out->gpu_ms = srv->gpuMs;
    std::vector<float> ms = srv->tickMs;
    if (!ms.empty()) {
        std::sort(ms.begin(), ms.end());
        out->tick_ms_p50 = ms[ms.size() / 2];
        out->tick_ms_p99 = ms[std::min(ms.size() - 1, size_t(double(ms.size()) * 0.99))];
    }
    return CN_OK;
}

CN_API cn_status cn_server_read_particles(cn_server *srv, uint32_t scene, float *x, float *v, uint32_t count)
{
    if (!srv || scene >= srv->scenes.size()) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_read_particles: bad scene");
    SceneSlot &sc = *srv->scenes[scene];
    if (count > sc.store.soa.particle_count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_server_read_particles: count");
    if (sc.resident) return cn_batch_read_particles(srv->batch, sc.batchId, x, v, count);
    if (x) std::memcpy(x, sc.store.x.data(), sizeof(float) * 4 * count);
    if (v) std::memcpy(v, sc.store.v.data(), sizeof(float) * 4 * count);
    return CN_OK;
}

} // extern "C"
