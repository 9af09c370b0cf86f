// cn_batch.cpp -- many independent soft-tissue scenes resident in one device pool and stepped
// together (no reference counterpart: the reference steps one PhysicsWorld per PhysicsSolver).
//
// Each admitted scene owns contiguous ranges of the pool's particle, edge, tet, incidence,
// body, collider and material arrays; its indices are rebased into those ranges on upload, so
// every per-element computation of the substep reads exactly the values it reads in a solver of
// its own and produces the same bits.  A tick steps any subset of the resident scenes: the host
// writes the tick's work lists (element ranges of the chosen scenes, cut into tiles) and staged
// kinematic targets, and replays one CUDA graph whose kernels stride over those lists with a
// fixed grid.  The graph is captured once per frame dt; the tile size and grid are tuned by
// cn_batch_autotune on the resident scenes.  A batch created with a coloured XPBD schedule also
// holds each scene's edge and tet colourings (made as a solver of its own makes them), and its
// colour passes run one kernel per colour over all stepped scenes.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_device.h"
#include "cn_internal.h"

using cn::setError;

namespace {

#define CN_CUDA(call)                                                                                  \
    do {                                                                                               \
        const cudaError_t e__ = (call);                                                                \
        if (e__ != cudaSuccess)                                                                        \
            return setError(e__ == cudaErrorMemoryAllocation ? CN_ERR_OUT_OF_MEMORY : CN_ERR_CUDA,     \
                            std::string(#call) + ": " + cudaGetErrorString(e__));                      \
    } while (0)

// First-fit allocator of index ranges in [0, capacity), merging neighbours on release.
class RangeAlloc {
public:
    void reset(uint32_t capacity)
    {
        free_.clear();
        if (capacity) free_[0] = capacity;
        capacity_ = capacity;
        used_ = 0;
    }
    bool alloc(uint32_t n, uint32_t &start)
    {
        start = 0;
        if (n == 0) return true;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            start = it->first;
            const uint32_t rest = it->second - n;
            free_.erase(it);
            if (rest) free_[start + n] = rest;
            used_ += n;
            return true;
        }
        return false;
    }
    void release(uint32_t start, uint32_t n)
    {
        if (n == 0) return;
        used_ -= n;
        auto it = free_.emplace(start, n).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint32_t used() const { return used_; }
    uint32_t capacity() const { return capacity_; }

private:
    std::map<uint32_t, uint32_t> free_;
    uint32_t capacity_ = 0, used_ = 0;
};

// Ranges of one resident scene (start, count) per pool family.
struct Range {
    uint32_t start = 0, count = 0;
};
struct BatchScene {
    bool live = false;
    uint64_t stepStamp = 0; // the cn_batch_step call that last listed it (duplicate check)
    Range p, e, t, ei, ti, b, c, ci, m, k;
    uint32_t edgeColours = 0;
    uint32_t queryCount = 0; // colliders in its query order (a prefix-free range starting at c.start)
    uint64_t bytes = 0;
};

inline uint32_t asBits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    return u;
}
inline float fromBits(uint32_t u)
{
    float f;
    std::memcpy(&f, &u, sizeof(f));
    return f;
}

// Device bytes one element of each family takes in the pool (used for the budget accounting).
constexpr uint64_t kBytesPerParticle = 3 * 16 + 6 * 4 + 16 + 2 * 8 + 2 * 4 + 8;
constexpr uint64_t kBytesPerEdge = 16 + 4 + 2 * 16 + 2 * 4;
constexpr uint64_t kBytesPerTet = 32 + 4 + 4 * 16 + 4 * 4;
constexpr uint64_t kBytesPerBody = 16 * 16 + 8 + 8;
constexpr uint64_t kBytesPerCollider = 48 + 32 + 16 + 3 * 16 + 4 * 16 + 4 + 4;

} // namespace

struct cn_batch {
    cn_batch_desc desc{};
    int device = 0;
    cudaStream_t ownStream = nullptr;
    cn::Scene s{};
    cn::Config cfg{};
    void *arena = nullptr;
    size_t arenaBytes = 0;
    uint32_t *scanScratch = nullptr;
    size_t scanScratchBytes = 0;
    uint32_t P = 0, E = 0, T = 0, B = 0, C = 0, M = 0, pairCap = 0, K = 0;
    RangeAlloc aP, aE, aT, aEI, aTI, aB, aC, aCI, aM, aK;
    // XPBD schedule: the running one, and whether the pool holds colour tables (a batch created
    // with a coloured schedule); colours = the most any resident scene's edges / tets need
    uint32_t schedule = CN_XPBD_GATHER;
    bool coloured = false;
    uint32_t colours[2] = {0, 0};
    std::vector<BatchScene> scenes;
    uint64_t bytesAdmitted = 0;
    // work lists: 5 tile regions + 6 counters (5 lists + targets) on the device and in two pinned
    // staging areas; staged kinematic targets
    uint32_t capTiles[5] = {0, 0, 0, 0, 0};
    uint32_t tileOffset[5] = {0, 0, 0, 0, 0};
    uint32_t tileTotal = 0, targetCap = 0;
    uint2 *dTiles = nullptr;
    uint32_t *dCounts = nullptr;
    cn::BodyTarget *dTargets = nullptr;
    uint8_t *hStage[2] = {nullptr, nullptr};
    cudaEvent_t stageDone[2] = {nullptr, nullptr};
    int stageIdx = 0;
    std::vector<cn::BodyTarget> pendingTargets;
    // graph of one tick
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    float graphDt = -1.0f;
    uint32_t substeps = 1, softIt = 1, contactIt = 1, maxIt = 1;
    uint32_t tileElems = 256, blocksPerSm = 8, smCount = 148, grid = 0;
    uint64_t ticks = 0, stepCalls = 0;
    // persistent fused iterations: CTAs per scene cluster (0: per-phase kernels), clusters of the
    // grid; the tick's scene list (cn::kSceneListStride uint2 per stepped scene; counter 6 =
    // scenes, counter 7 = the next scene to take, both staged with the work lists)
    uint32_t clusterCtas = 0, clusters = 0;
    uint2 *dScenes = nullptr;
    uint2 *hScenes[2] = {nullptr, nullptr};
    // admission: scene images are copied and scattered on the upload stream; the next tick waits
    // for the last one
    cudaStream_t upStream = nullptr;
    cudaEvent_t upDone = nullptr;
    uint8_t *dStage = nullptr;
    size_t stageBytes = 0;
    bool uploadPending = false;
};

namespace {

void releaseGraph(cn_batch *b)
{
    if (b->graphExec) cudaGraphExecDestroy(b->graphExec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graphExec = nullptr;
    b->graph = nullptr;
    b->graphDt = -1.0f;
}

// Pinned staging layout: tiles, then 8 counters, then the targets (16-byte aligned: float4s).
size_t stageTileBytes(const cn_batch *b) { return (size_t(b->tileTotal) * sizeof(uint2) + 15) & ~size_t(15); }
size_t stageBytes(const cn_batch *b)
{
    return stageTileBytes(b) + 8 * sizeof(uint32_t) + size_t(std::max<uint32_t>(b->targetCap, 1u)) * sizeof(cn::BodyTarget);
}

// Number of tiles the largest possible tick needs per family for the current tile size.
void sizeWorkLists(cn_batch *b)
{
    const uint32_t te = b->tileElems;
    const uint32_t maxScenes = std::max<uint32_t>(b->desc.max_scenes, 1u);
    const uint32_t cnt[5] = {b->P, b->E, b->T, b->B, b->C};
    b->tileTotal = 0;
    for (int k = 0; k < 5; ++k) {
        // every scene adds at most one partial tile per family
        b->capTiles[k] = (k >= 3 ? cnt[k] : (cnt[k] + te - 1) / te) + maxScenes;
        b->tileOffset[k] = b->tileTotal;
        b->tileTotal += b->capTiles[k];
    }
    b->targetCap = std::max<uint32_t>(b->B, 1u);
}

cn_status allocWorkLists(cn_batch *b)
{
    sizeWorkLists(b);
    if (b->dTiles) cudaFree(b->dTiles);
    if (b->dCounts) cudaFree(b->dCounts);
    if (b->dTargets) cudaFree(b->dTargets);
    for (int k = 0; k < 2; ++k)
        if (b->hStage[k]) cudaFreeHost(b->hStage[k]);
    b->dTiles = nullptr; b->dCounts = nullptr; b->dTargets = nullptr;
    b->hStage[0] = b->hStage[1] = nullptr;
    if (b->dScenes) cudaFree(b->dScenes);
    for (int k = 0; k < 2; ++k)
        if (b->hScenes[k]) cudaFreeHost(b->hScenes[k]);
    b->dScenes = nullptr;
    b->hScenes[0] = b->hScenes[1] = nullptr;
    const size_t sceneListBytes = size_t(cn::kSceneListStride) * std::max<uint32_t>(b->desc.max_scenes, 1u) * sizeof(uint2);
    CN_CUDA(cudaMalloc(&b->dScenes, sceneListBytes));
    for (int k = 0; k < 2; ++k) CN_CUDA(cudaMallocHost(&b->hScenes[k], sceneListBytes));
    CN_CUDA(cudaMalloc(&b->dTiles, size_t(b->tileTotal) * sizeof(uint2)));
    CN_CUDA(cudaMalloc(&b->dCounts, 8 * sizeof(uint32_t)));
    CN_CUDA(cudaMalloc(&b->dTargets, size_t(b->targetCap) * sizeof(cn::BodyTarget)));
    CN_CUDA(cudaMemset(b->dCounts, 0, 8 * sizeof(uint32_t)));
    for (int k = 0; k < 2; ++k) CN_CUDA(cudaMallocHost(&b->hStage[k], stageBytes(b)));
    cn::Scene &s = b->s;
    cn::WorkList *lists[5] = {&s.wP, &s.wE, &s.wT, &s.wB, &s.wC};
    for (int k = 0; k < 5; ++k) {
        lists[k]->tiles = b->dTiles + b->tileOffset[k];
        lists[k]->count = b->dCounts + k;
        lists[k]->grid = b->grid;
    }
    return CN_OK;
}

void layoutPool(cn_batch *b, cn::Arena &a)
{
    cn::Scene &s = b->s;
    const uint32_t P = b->P, E = b->E, T = b->T, B = std::max<uint32_t>(b->B, 1u), C = std::max<uint32_t>(b->C, 1u);
    s.N = P;
    s.x = a.take<float4>(P); s.xprev = a.take<float4>(P); s.v = a.take<float4>(P);
    s.radii = a.take<float>(P);
    s.kinds = a.take<uint32_t>(P);
    s.meta = a.take<uint4>(P);
    s.matIdx = a.take<uint32_t>(P);
    s.fluidMatIdx = a.take<uint32_t>(P);
    s.ownerTypes = a.take<uint32_t>(P);
    s.ownerIdx = a.take<uint32_t>(P);
    s.contactMaterials = a.take<float4>(std::max<uint32_t>(b->M, 1u));
    s.fluidMaterials = a.take<cn_fluid_material>(1);
    s.E = E; s.T = T;
    s.edgesP = a.take<cn::PackedEdge>(E);
    s.tets = a.take<cn_soft_tet>(T);
    s.edgeRanges = a.take<uint2>(P);
    s.tetRanges = a.take<uint2>(P);
    s.edgeDst = a.take<uint32_t>(size_t(E) * 2);
    s.tetDst = a.take<uint32_t>(size_t(T) * 4);
    s.edgeLambda = a.take<float>(E);
    s.tetLambda = a.take<float>(T);
    s.edgeCorr = a.take<float4>(size_t(E) * 2);
    s.tetCorr = a.take<float4>(size_t(T) * 4);
    s.pColRange = a.take<uint2>(P);
    s.B = b->B;
    s.C = b->C;
    s.bodyPos = a.take<float4>(B); s.bodyRot = a.take<float4>(B); s.bodyLin = a.take<float4>(B);
    s.bodyAng = a.take<float4>(B); s.bodyScale = a.take<float4>(B); s.bodyInvInertia = a.take<float4>(B);
    s.bodyType = a.take<uint32_t>(B);
    s.bodyKinPos = a.take<float4>(B); s.bodyKinRot = a.take<float4>(B); s.bodyKinFlags = a.take<uint32_t>(B);
    s.bodyColRanges = a.take<uint2>(B);
    s.bodyColIdx = a.take<uint32_t>(C);
    s.colGeo = a.take<cn_collider_geometry>(C);
    s.colBp = a.take<cn_collider_broadphase>(C);
    s.colMat = a.take<float4>(C);
    s.prevBodyPos = a.take<float4>(B); s.prevBodyRot = a.take<float4>(B);
    s.predBodyPos = a.take<float4>(B); s.predBodyRot = a.take<float4>(B);
    s.predBodyLin = a.take<float4>(B); s.predBodyAng = a.take<float4>(B);
    s.colAabbMin = a.take<float4>(C); s.colAabbMax = a.take<float4>(C);
    s.colFrame = a.take<float4>(size_t(C) * 4);
    s.colQueryOrder = a.take<uint32_t>(C);
    s.candCount = a.take<uint32_t>(P);
    s.candOffset = a.take<uint32_t>(P);
    s.rigidPairCapacity = b->pairCap;
    s.rigidPairs = a.take<uint2>(b->pairCap);
    s.rigidContacts = a.take<cn::RigidContact>(b->pairCap);
    s.meta_ = a.take<cn::DeviceMeta>(1);
    if (b->coloured) {
        s.edgesC = a.take<cn::PackedEdge>(E);
        s.tetsC = a.take<cn_soft_tet>(T);
        s.tetRecC = a.take<float4>(size_t(T) * 4);
        s.softAcc = a.take<float4>(P);
        s.batchColStarts = a.take<uint32_t>(b->K);
    }
    b->scanScratchBytes = (size_t(2) * P + 4) * sizeof(uint32_t) + cn::scanScratchBytes(std::max<uint32_t>(P, 1u));
    b->scanScratch = a.take<uint32_t>(b->scanScratchBytes / sizeof(uint32_t));
}

// One tick: staged targets, then `substeps` substeps of the XPBD soft families and the
// particle-rigid contacts in the order of PhysicsSolver::step (the subset of the single-world
// schedule that soft-tissue scenes exercise).
void enqueueTick(cn_batch *b, float frameDt, cudaStream_t st)
{
    const cn::Scene &s = b->s;
    const cn::Config &c = b->cfg;
    const float dt = frameDt / float(b->substeps);
    cn::launchApplyBodyTargets(s, b->dTargets, b->dCounts + 5, b->targetCap, st);
    for (uint32_t sub = 0; sub < b->substeps; ++sub) {
        cn::launchRigidPredict(s, dt, c.gravity[0], c.gravity[1], c.gravity[2], st);
        cn::launchPredictAndKeys(s, dt, c, st);
        if (b->contactIt) cn::launchRigidCandidates(s, b->scanScratch, b->scanScratchBytes, st);
        if (s.E) cudaMemsetAsync(s.edgeLambda, 0, sizeof(float) * s.E, st);
        if (s.T) cudaMemsetAsync(s.tetLambda, 0, sizeof(float) * s.T, st);
        if (b->clusterCtas) {
            // every iteration of the substep in one persistent kernel, one scene per cluster
            cn::BatchFusedPlan plan{};
            plan.iterations = b->maxIt;
            plan.softIterations = b->softIt;
            plan.contactIterations = b->contactIt;
            plan.scenes = b->dScenes;
            plan.sceneCount = b->dCounts + 6;
            plan.next = b->dCounts + 7;
            if (sub > 0) cudaMemsetAsync(b->dCounts + 7, 0, sizeof(uint32_t), st);
            cn::launchBatchFusedIterations(s, c, dt, plan, b->clusterCtas, b->clusters, st);
        }
        for (uint32_t it = 0; it < (b->clusterCtas ? 0u : b->maxIt); ++it) {
            const bool runSoft = (s.E || s.T) && it < b->softIt;
            const bool runRigid = it < b->contactIt;
            if (!runSoft && !runRigid) break;
            // the contact records are read after the iterations: written by the last contact pass only
            cn::Scene si = s;
            si.storeRigidContacts = it + 1 == b->contactIt ? 1u : 0u;
            if (b->schedule != CN_XPBD_GATHER) {
                // one kernel per colour over every stepped scene, then the contacts
                if (runSoft)
                    cn::launchBatchColourIteration(s, dt, c, b->schedule, b->colours, b->dScenes, b->dCounts + 6,
                                                   b->grid, st);
                if (runRigid) cn::launchContacts(si, c, false, true, st);
                continue;
            }
            // the rigid contacts run in the tet gather's pass when there is a tet family
            const bool contactsDone = runSoft && cn::launchSoftIteration(si, dt, c, st, runRigid);
            if (runRigid && !contactsDone) cn::launchContacts(si, c, false, true, st);
        }
        cn::launchUpdateVelocities(s, dt, nullptr, st);
        if (b->contactIt) cn::launchRigidContactVelocities(s, b->contactIt, c, st);
        cn::launchCopyPredictedRigid(s, st);
    }
}

cn_status ensureGraph(cn_batch *b, float frameDt)
{
    if (b->graphExec && b->graphDt == frameDt) return CN_OK;
    releaseGraph(b);
    CN_CUDA(cudaStreamBeginCapture(b->ownStream, cudaStreamCaptureModeThreadLocal));
    enqueueTick(b, frameDt, b->ownStream);
    const cudaError_t e = cudaStreamEndCapture(b->ownStream, &b->graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return setError(CN_ERR_CUDA, std::string("batch graph capture failed: ") + cudaGetErrorString(e));
    }
    CN_CUDA(cudaGraphInstantiate(&b->graphExec, b->graph, 0));
    b->graphDt = frameDt;
    return CN_OK;
}

template <class T> cudaError_t upTo(T *dst, const T *src, size_t count, cudaStream_t st)
{
    if (!count || !src) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
}

void releaseScene(cn_batch *b, BatchScene &sc)
{
    b->aP.release(sc.p.start, sc.p.count);
    b->aE.release(sc.e.start, sc.e.count);
    b->aT.release(sc.t.start, sc.t.count);
    b->aEI.release(sc.ei.start, sc.ei.count);
    b->aTI.release(sc.ti.start, sc.ti.count);
    b->aB.release(sc.b.start, sc.b.count);
    b->aC.release(sc.c.start, sc.c.count);
    b->aCI.release(sc.ci.start, sc.ci.count);
    b->aM.release(sc.m.start, sc.m.count);
    b->aK.release(sc.k.start, sc.k.count);
    b->bytesAdmitted -= sc.bytes;
    sc = BatchScene{};
}

} // namespace

namespace cn {

cn_status buildSceneImage(const cn_world_soa &w, uint32_t rigidPairsPerParticle, bool coloured, SceneImage &img)
{
    const uint32_t N = w.particle_count;
    if (N == 0) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_add_scene: empty scene");
    if (!w.positions_inv_mass || !w.velocities || !w.radii || !w.kinds || !w.metadata || !w.material_indices ||
        !w.owner_types || !w.owner_indices)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_add_scene: missing particle array");
    // The batch runs the soft-tissue families: edges, tets, static / kinematic colliders.
    if (w.bend_count || w.dihedral_count || w.strand_segment_count || w.strand_joint_count || w.strand_distance_count)
        return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: cloth and strand constraints are not batched");
    std::vector<uint32_t> groups;
    for (uint32_t i = 0; i < N; ++i) {
        if (w.kinds[i] == CN_PARTICLE_FLUID)
            return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: fluid particles are not batched");
        if (w.owner_types[i] == CN_OWNER_RIGID_BODY)
            return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: rigid proxy particles are not batched");
        const uint32_t ph = w.metadata[4 * i + 1];
        if (ph & CN_PHASE_SELF_COLLIDE)
            return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: self-colliding bodies are not batched");
        const uint32_t g = ph & CN_PHASE_GROUP_MASK;
        if (std::find(groups.begin(), groups.end(), g) == groups.end()) groups.push_back(g);
    }
    if (groups.size() > 1)
        return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: scenes with particle-particle contacts are not batched");
    for (uint32_t k = 0; k < w.rigid_body_count; ++k)
        if (w.body_types[k] == CN_BODY_DYNAMIC) return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: dynamic rigid bodies");
    std::vector<uint32_t> order;
    colliderQueryOrder(w, order);
    const Incidence edgeI = buildIncidence(N, w.edge_count, 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? w.edges[c].particle_a : w.edges[c].particle_b;
    });
    const Incidence tetI = buildIncidence(N, w.tet_count, 4, [&](uint32_t c, uint32_t k) {
        return w.tets[c].particle_indices[k];
    });
    // coloured schedules: the colourings a solver of this scene makes, and per family the words
    // colours, particle window, colour starts
    Colouring edgeCol, tetCol;
    std::vector<uint32_t> colWords;
    if (coloured) {
        edgeCol = colourGreedy(N, w.edge_count, 2, [&](uint32_t c, uint32_t k) {
            return k == 0 ? w.edges[c].particle_a : w.edges[c].particle_b;
        });
        tetCol = colourGreedy(N, w.tet_count, 4, [&](uint32_t c, uint32_t k) { return w.tets[c].particle_indices[k]; });
        if (edgeCol.colours() > kBatchMaxColours || tetCol.colours() > kBatchMaxColours)
            return setError(CN_ERR_UNSUPPORTED, "cn_batch_add_scene: more than " + std::to_string(kBatchMaxColours) +
                                                    " colours in one constraint family");
        const Colouring *fam[2] = {&edgeCol, &tetCol};
        const uint2 win[2] = {incidenceWindow(edgeI), incidenceWindow(tetI)};
        for (int f = 0; f < 2; ++f) {
            colWords.push_back(fam[f]->colours());
            colWords.push_back(win[f].x);
            colWords.push_back(win[f].y);
            if (fam[f]->colours()) colWords.insert(colWords.end(), fam[f]->starts.begin(), fam[f]->starts.end());
            else colWords.push_back(0u);
        }
    }

    AdmitImage &L = img.layout;
    L = AdmitImage{};
    img.colours[0] = edgeCol.colours();
    img.colours[1] = tetCol.colours();
    L.N = N;
    L.E = w.edge_count;
    L.T = w.tet_count;
    L.B = w.rigid_body_count;
    L.C = w.collider_count;
    L.CI = w.body_collider_index_count;
    L.M = std::max<uint32_t>(w.contact_material_count, 1u);
    L.queryCount = uint32_t(order.size());
    L.colWords = uint32_t(colWords.size());
    const size_t sizes[kAdmSegments] = {
        16ull * N, 16ull * N, 4ull * N, 4ull * N, 16ull * N, 4ull * N, 4ull * N, 4ull * N, 8ull * N, 8ull * N,
        sizeof(cn_soft_edge) * L.E, 8ull * L.E, sizeof(cn_soft_tet) * L.T, 16ull * L.T, 16ull * L.M,
        16ull * L.B, 16ull * L.B, 16ull * L.B, 16ull * L.B, 16ull * L.B, 16ull * L.B, 4ull * L.B, 16ull * L.B,
        16ull * L.B, 4ull * L.B, 8ull * L.B, 4ull * L.CI, sizeof(cn_collider_geometry) * L.C,
        sizeof(cn_collider_broadphase) * L.C, 16ull * L.C, 4ull * L.queryCount, 4ull * edgeCol.order.size(),
        4ull * tetCol.order.size(), 4ull * L.colWords};
    size_t at = 0;
    for (uint32_t k = 0; k < kAdmSegments; ++k) {
        L.off[k] = at;
        at += (sizes[k] + 15) & ~size_t(15);
    }
    img.bytes.assign(at, 0);
    auto put = [&](uint32_t seg, const void *src, size_t bytes) {
        if (bytes && src) std::memcpy(img.bytes.data() + L.off[seg], src, bytes);
    };
    put(kAdmRadii, w.radii, 4ull * N);
    put(kAdmKinds, w.kinds, 4ull * N);
    put(kAdmMeta, w.metadata, 16ull * N);
    put(kAdmMatIdx, w.material_indices, 4ull * N);
    put(kAdmOwnerTypes, w.owner_types, 4ull * N);
    put(kAdmOwnerIdx, w.owner_indices, 4ull * N);
    put(kAdmEdgeRanges, edgeI.ranges.data(), 8ull * N);
    put(kAdmTetRanges, tetI.ranges.data(), 8ull * N);
    put(kAdmEdges, w.edges, sizeof(cn_soft_edge) * L.E);
    put(kAdmEdgeDst, edgeI.dst.data(), 8ull * L.E);
    put(kAdmTets, w.tets, sizeof(cn_soft_tet) * L.T);
    put(kAdmTetDst, tetI.dst.data(), 16ull * L.T);
    put(kAdmMaterials, w.contact_materials, 16ull * w.contact_material_count);
    put(kAdmBodyScale, w.body_scales, 16ull * L.B);
    put(kAdmBodyInvI, w.body_inverse_inertia, 16ull * L.B);
    put(kAdmBodyType, w.body_types, 4ull * L.B);
    put(kAdmBodyColRanges, w.body_collider_ranges, 8ull * L.B);
    put(kAdmBodyColIdx, w.body_collider_indices, 4ull * L.CI);
    put(kAdmColGeo, w.collider_geometry, sizeof(cn_collider_geometry) * L.C);
    put(kAdmColBp, w.collider_broadphase, sizeof(cn_collider_broadphase) * L.C);
    put(kAdmColMat, w.collider_materials, 16ull * L.C);
    put(kAdmQueryOrder, order.data(), 4ull * L.queryCount);
    put(kAdmEdgeColOrder, edgeCol.order.data(), 4ull * edgeCol.order.size());
    put(kAdmTetColOrder, tetCol.order.data(), 4ull * tetCol.order.size());
    put(kAdmColStarts, colWords.data(), 4ull * L.colWords);
    refreshSceneImage(w, img);
    img.budgetBytes = N * kBytesPerParticle + uint64_t(L.E) * kBytesPerEdge + uint64_t(L.T) * kBytesPerTet +
                      uint64_t(L.B) * kBytesPerBody + uint64_t(L.C) * kBytesPerCollider +
                      uint64_t(N) * rigidPairsPerParticle * 72u;
    if (coloured) // colour-ordered edges and tets with the tets' records, the colour-Jacobi sums, the tables
        img.budgetBytes += sizeof(cn::PackedEdge) * uint64_t(L.E) + (sizeof(cn_soft_tet) + 64ull) * L.T + 16ull * N +
                           4ull * L.colWords;
    return CN_OK;
}

void refreshSceneImage(const cn_world_soa &w, SceneImage &img)
{
    const AdmitImage &L = img.layout;
    auto put = [&](uint32_t seg, const void *src, size_t bytes) {
        if (bytes && src) std::memcpy(img.bytes.data() + L.off[seg], src, bytes);
    };
    put(kAdmX, w.positions_inv_mass, 16ull * L.N);
    put(kAdmV, w.velocities, 16ull * L.N);
    put(kAdmBodyPos, w.body_positions_inv_mass, 16ull * L.B);
    put(kAdmBodyRot, w.body_orientations, 16ull * L.B);
    put(kAdmBodyLin, w.body_linear_velocities, 16ull * L.B);
    put(kAdmBodyAng, w.body_angular_velocities, 16ull * L.B);
    put(kAdmKinPos, w.body_kinematic_target_positions, 16ull * L.B);
    put(kAdmKinRot, w.body_kinematic_target_orientations, 16ull * L.B);
    put(kAdmKinFlags, w.body_kinematic_target_flags, 4ull * L.B);
}

// The device side of an admission: a recapture when the scene brings more colours than the tick's
// graph passes over, one transfer into the staging buffer (grown when a larger scene arrives),
// then the scatter into the scene's ranges; all on the upload stream, which the next tick waits for.
static cudaError_t uploadScene(cn_batch *b, const SceneImage &img, const BatchScene &sc)
{
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return e;
    if (b->coloured && (img.colours[0] > b->colours[0] || img.colours[1] > b->colours[1])) {
        b->colours[0] = std::max(b->colours[0], img.colours[0]);
        b->colours[1] = std::max(b->colours[1], img.colours[1]);
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e; // no tick of the old graph in flight
        releaseGraph(b);
    }
    const size_t bytes = img.bytes.size();
    if (bytes > b->stageBytes) {
        const size_t cap = std::max(bytes, 2 * b->stageBytes);
        if ((e = cudaStreamSynchronize(b->upStream)) != cudaSuccess) return e;
        if (b->dStage) cudaFree(b->dStage);
        b->dStage = nullptr;
        b->stageBytes = 0;
        if ((e = cudaMalloc(&b->dStage, cap)) != cudaSuccess) return e;
        b->stageBytes = cap;
    }
    if ((e = cudaMemcpyAsync(b->dStage, img.bytes.data(), bytes, cudaMemcpyHostToDevice, b->upStream)) != cudaSuccess)
        return e;
    AdmitImage a = img.layout;
    a.img = b->dStage;
    a.p0 = sc.p.start; a.e0 = sc.e.start; a.t0 = sc.t.start; a.ei0 = sc.ei.start; a.ti0 = sc.ti.start;
    a.b0 = sc.b.start; a.c0 = sc.c.start; a.ci0 = sc.ci.start; a.m0 = sc.m.start; a.k0 = sc.k.start;
    launchAdmitScene(b->s, a, b->upStream);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaEventRecord(b->upDone, b->upStream);
}

cn_status batchAdmitImage(cn_batch *b, const SceneImage &img, uint32_t *scene_id)
{
    const AdmitImage &L = img.layout;
    if ((L.colWords != 0u) != b->coloured)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_add_scene: the scene image does not match the batch's schedule");
    if (b->bytesAdmitted + img.budgetBytes > b->desc.memory_budget_bytes)
        return setError(CN_ERR_CAPACITY, "cn_batch_add_scene: the device-memory budget is full");
    BatchScene sc;
    bool ok = b->aP.alloc(L.N, sc.p.start);
    sc.p.count = ok ? L.N : 0;
    auto take = [&](RangeAlloc &ra, uint32_t n, Range &r) {
        if (!ok) return;
        ok = ra.alloc(n, r.start);
        r.count = ok ? n : 0;
    };
    take(b->aE, L.E, sc.e);
    take(b->aT, L.T, sc.t);
    take(b->aEI, L.E * 2u, sc.ei);
    take(b->aTI, L.T * 4u, sc.ti);
    take(b->aB, L.B, sc.b);
    take(b->aC, L.C, sc.c);
    take(b->aCI, L.CI, sc.ci);
    take(b->aM, L.M, sc.m);
    take(b->aK, L.colWords, sc.k);
    if (!ok) {
        releaseScene(b, sc);
        return setError(CN_ERR_CAPACITY, "cn_batch_add_scene: the pool has no room for this scene");
    }
    sc.live = true;
    sc.queryCount = L.queryCount;
    sc.edgeColours = img.colours[0];
    sc.bytes = img.budgetBytes;
    b->bytesAdmitted += img.budgetBytes;
    const cudaError_t e = uploadScene(b, img, sc);
    if (e != cudaSuccess) { // the ranges and the budget go back; the pool keeps no part of the scene
        releaseScene(b, sc);
        return setError(e == cudaErrorMemoryAllocation ? CN_ERR_OUT_OF_MEMORY : CN_ERR_CUDA,
                        std::string("cn_batch_add_scene: ") + cudaGetErrorString(e));
    }
    b->uploadPending = true;
    uint32_t id = 0;
    while (id < b->scenes.size() && b->scenes[id].live) ++id;
    if (id == b->scenes.size()) b->scenes.emplace_back();
    b->scenes[id] = sc;
    *scene_id = id;
    clearError();
    return CN_OK;
}

uint32_t batchRigidPairsPerParticle(const cn_batch *b) { return b->desc.rigid_pairs_per_particle; }
bool batchColoured(const cn_batch *b) { return b->coloured; }

} // namespace cn

extern "C" {

CN_API void cn_batch_desc_defaults(cn_batch_desc *d)
{
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    cn_solver_desc_defaults(&d->solver);
    d->solver.enable_blocking_readback = 0;
    d->memory_budget_bytes = uint64_t(1) << 30;
    d->max_scenes = 1024;
    d->tile_elements = 256;
    d->blocks_per_sm = 8;
    d->rigid_pairs_per_particle = 4;
}

CN_API cn_status cn_batch_create(const cn_batch_desc *d, int device, cn_batch **out)
{
    if (!d || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_create: null argument");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return setError(CN_ERR_NO_DEVICE, "cn_batch_create: no CUDA device");
    }
    if (device < 0 || device >= count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_create: bad device");
    const uint32_t schedule = d->solver.soft.xpbd_schedule;
    if (schedule > CN_XPBD_COLOUR_GAUSS_SEIDEL)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_create: unknown soft.xpbd_schedule");
    if (schedule != CN_XPBD_GATHER && d->fused_cluster_ctas)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_create: the fused iterations run the gather schedule");
    auto *b = new cn_batch();
    b->schedule = schedule;
    b->coloured = schedule != CN_XPBD_GATHER;
    b->desc = *d;
    b->device = device;
    CN_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    b->smCount = uint32_t(std::max(prop.multiProcessorCount, 1));
    b->tileElems = std::max<uint32_t>(d->tile_elements, 32u);
    b->blocksPerSm = std::max<uint32_t>(d->blocks_per_sm, 1u);
    b->grid = b->smCount * b->blocksPerSm;
    // Capacities: given explicitly, or split from the budget by the soft-tissue lattice mix
    // (about 6.5 edges and 5 tets per particle, one body and one collider per 256 particles).
    uint32_t P = d->particle_capacity, E = d->edge_capacity, T = d->tet_capacity;
    uint32_t B = d->body_capacity, C = d->collider_capacity;
    if (P == 0) {
        const uint64_t perParticle = kBytesPerParticle + 4 * 72 + 7 * kBytesPerEdge + 5 * kBytesPerTet + 64;
        P = uint32_t(std::min<uint64_t>(d->memory_budget_bytes / perParticle, (1u << 29)));
    }
    if (E == 0) E = P * 7u;
    if (T == 0) T = P * 5u;
    if (B == 0) B = std::max<uint32_t>(P / 256u, 2u * std::max<uint32_t>(d->max_scenes, 1u));
    if (C == 0) C = B;
    b->P = P; b->E = E; b->T = T; b->B = B; b->C = C;
    b->M = std::max<uint32_t>(B, 1u);
    b->pairCap = std::max<uint32_t>(P * std::max<uint32_t>(d->rigid_pairs_per_particle, 1u), 64u);
    b->aP.reset(P); b->aE.reset(E); b->aT.reset(T); b->aEI.reset(E * 2u); b->aTI.reset(T * 4u);
    b->aB.reset(B); b->aC.reset(C); b->aCI.reset(C); b->aM.reset(b->M);
    // colour-table words: a scene takes edge colours + tet colours + 8 <= its edges + tets + 8
    // particles' worth
    b->K = b->coloured ? uint32_t(std::min<uint64_t>(8ull * P + uint64_t(E) + T, 0xffffffffull)) : 0u;
    b->aK.reset(b->K);
    cn::Arena a;
    a.reset(nullptr);
    layoutPool(b, a);
    b->arenaBytes = a.size();
    const cudaError_t e = cudaMalloc(&b->arena, b->arenaBytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return setError(CN_ERR_OUT_OF_MEMORY, "cn_batch_create: cannot allocate the pool (" +
                                                  std::to_string(a.size()) + " bytes)");
    }
    a.reset(static_cast<uint8_t *>(b->arena));
    layoutPool(b, a);
    cudaStreamCreateWithFlags(&b->ownStream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&b->upStream, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&b->upDone, cudaEventDisableTiming);
    cudaMemsetAsync(b->arena, 0, b->arenaBytes, b->ownStream);
    for (int k = 0; k < 2; ++k) cudaEventCreateWithFlags(&b->stageDone[k], cudaEventDisableTiming);
    const cn_status st = allocWorkLists(b);
    if (st != CN_OK) {
        cn_batch_destroy(b);
        return st;
    }
    if (d->fused_cluster_ctas) {
        const cn_status fs = cn_batch_set_fused(b, d->fused_cluster_ctas);
        if (fs != CN_OK) {
            cn_batch_destroy(b);
            return fs;
        }
    }
    b->cfg = cn::configFromDesc(d->solver);
    const cn_solver_desc &sd = d->solver;
    b->substeps = std::max<uint32_t>(sd.substeps, 1u);
    const uint32_t defIt = std::max<uint32_t>(sd.default_iterations, 1u);
    b->softIt = cn::resolveIter(sd.soft_internal_iterations, defIt);
    b->contactIt = cn::resolveIter(sd.soft_contact_iterations, defIt);
    const uint32_t fluidIt = cn::resolveIter(sd.fluid_iterations, defIt);
    const uint32_t jointIt = cn::resolveIter(sd.rigid_joint_iterations, defIt);
    const uint32_t rrIt = cn::resolveIter(sd.rigid_rigid_contact_iterations, defIt);
    b->maxIt = std::max(std::max(std::max(fluidIt, b->softIt), b->contactIt), std::max(jointIt, rrIt));
    if (cudaStreamSynchronize(b->ownStream) != cudaSuccess) {
        cudaGetLastError();
        cn_batch_destroy(b);
        return setError(CN_ERR_CUDA, "cn_batch_create: pool initialisation failed");
    }
    *out = b;
    cn::clearError();
    return CN_OK;
}

CN_API void cn_batch_destroy(cn_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->ownStream) cudaStreamSynchronize(b->ownStream);
    cudaDeviceSynchronize();
    releaseGraph(b);
    if (b->arena) cudaFree(b->arena);
    if (b->dTiles) cudaFree(b->dTiles);
    if (b->dCounts) cudaFree(b->dCounts);
    if (b->dTargets) cudaFree(b->dTargets);
    if (b->dScenes) cudaFree(b->dScenes);
    for (int k = 0; k < 2; ++k) {
        if (b->hStage[k]) cudaFreeHost(b->hStage[k]);
        if (b->hScenes[k]) cudaFreeHost(b->hScenes[k]);
        if (b->stageDone[k]) cudaEventDestroy(b->stageDone[k]);
    }
    if (b->ownStream) cudaStreamDestroy(b->ownStream);
    if (b->upStream) cudaStreamDestroy(b->upStream);
    if (b->upDone) cudaEventDestroy(b->upDone);
    if (b->dStage) cudaFree(b->dStage);
    delete b;
}

CN_API cn_status cn_batch_add_scene(cn_batch *b, const cn_world_soa *w, uint32_t *scene_id)
{
    if (!b || !w || !scene_id) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_add_scene: null argument");
    cn::SceneImage img;
    const cn_status st = cn::buildSceneImage(*w, b->desc.rigid_pairs_per_particle, b->coloured, img);
    if (st != CN_OK) return st;
    return cn::batchAdmitImage(b, img, scene_id);
}

CN_API cn_status cn_batch_remove_scene(cn_batch *b, uint32_t scene_id)
{
    if (!b || scene_id >= b->scenes.size() || !b->scenes[scene_id].live)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_remove_scene: no such scene");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize()); // a tick in flight may still read the scene's ranges
    const BatchScene &sc = b->scenes[scene_id];
    b->pendingTargets.erase(std::remove_if(b->pendingTargets.begin(), b->pendingTargets.end(),
                                           [&](const cn::BodyTarget &t) {
                                               const uint32_t body = asBits(t.pos.w);
                                               return body >= sc.b.start && body < sc.b.start + sc.b.count;
                                           }),
                            b->pendingTargets.end());
    releaseScene(b, b->scenes[scene_id]);
    return CN_OK;
}

CN_API cn_status cn_batch_set_kinematic_target(cn_batch *b, uint32_t scene_id, uint32_t body,
                                               const float position[3], const float orientation[4])
{
    if (!b || !position || !orientation) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_kinematic_target: null argument");
    if (scene_id >= b->scenes.size() || !b->scenes[scene_id].live || body >= b->scenes[scene_id].b.count)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_kinematic_target: bad scene or body");
    cn::BodyTarget t;
    const uint32_t global = b->scenes[scene_id].b.start + body;
    t.pos = make_float4(position[0], position[1], position[2], fromBits(global));
    t.rot = make_float4(orientation[0], orientation[1], orientation[2], orientation[3]);
    // a later target of the same body replaces an earlier one staged for the same tick
    for (auto &p : b->pendingTargets)
        if (asBits(p.pos.w) == global) {
            p = t;
            return CN_OK;
        }
    b->pendingTargets.push_back(t);
    return CN_OK;
}

CN_API cn_status cn_batch_step(cn_batch *b, const uint32_t *scene_ids, uint32_t count, float frame_dt, void *stream)
{
    if (!b || (count && !scene_ids)) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_step: null argument");
    if (!(frame_dt > 0.0f)) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_step: frame_dt must be > 0");
    CN_CUDA(cudaSetDevice(b->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->ownStream;
    // Work lists of this tick in a pinned staging area (the one not used by the previous tick).
    const int k = b->stageIdx;
    b->stageIdx ^= 1;
    CN_CUDA(cudaEventSynchronize(b->stageDone[k]));
    uint8_t *stage = b->hStage[k];
    uint2 *tiles = reinterpret_cast<uint2 *>(stage);
    uint32_t *counts = reinterpret_cast<uint32_t *>(stage + stageTileBytes(b));
    cn::BodyTarget *targets = reinterpret_cast<cn::BodyTarget *>(counts + 8);
    std::memset(counts, 0, 8 * sizeof(uint32_t));
    const uint32_t te = b->tileElems;
    if (count > std::max<uint32_t>(b->desc.max_scenes, 1u))
        return setError(CN_ERR_CAPACITY, "cn_batch_step: more scenes than max_scenes");
    uint2 *sceneList = b->hScenes[k];
    const uint64_t stamp = ++b->stepCalls;
    for (uint32_t n = 0; n < count; ++n) {
        const uint32_t id = scene_ids[n];
        if (id >= b->scenes.size() || !b->scenes[id].live)
            return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_step: scene " + std::to_string(id) + " is not resident");
        BatchScene &sc = b->scenes[id];
        if (sc.stepStamp == stamp)
            return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_step: scene " + std::to_string(id) + " is listed twice");
        sc.stepStamp = stamp;
        uint2 *row = sceneList + size_t(cn::kSceneListStride) * n;
        row[0] = make_uint2(sc.p.start, sc.p.start + sc.p.count);
        row[1] = make_uint2(sc.e.start, sc.e.start + sc.e.count);
        row[2] = make_uint2(sc.t.start, sc.t.start + sc.t.count);
        row[3] = make_uint2(sc.k.start, sc.k.start + sc.edgeColours + 4u); // edge, tet colour tables
        const Range fam[5] = {sc.p, sc.e, sc.t, sc.b, sc.c};
        for (int f = 0; f < 5; ++f) {
            const uint32_t step = f >= 3 ? std::max<uint32_t>(fam[f].count, 1u) : te;
            for (uint32_t a = 0; a < fam[f].count; a += step) {
                if (counts[f] >= b->capTiles[f]) return setError(CN_ERR_CAPACITY, "cn_batch_step: work list overflow");
                tiles[b->tileOffset[f] + counts[f]++] =
                    make_uint2(fam[f].start + a, fam[f].start + std::min(fam[f].count, a + step));
            }
        }
    }
    const uint32_t nt = uint32_t(std::min<size_t>(b->pendingTargets.size(), b->targetCap));
    std::copy(b->pendingTargets.begin(), b->pendingTargets.begin() + nt, targets);
    counts[5] = nt;
    counts[6] = count; // scenes of the fused iterations; counts[7] (the next one to take) stays 0
    b->pendingTargets.erase(b->pendingTargets.begin(), b->pendingTargets.begin() + nt);
    const cn_status gs = ensureGraph(b, frame_dt);
    if (gs != CN_OK) return gs;
    if (b->uploadPending) { // admitted scenes' uploads land before this tick reads the pool
        CN_CUDA(cudaStreamWaitEvent(st, b->upDone, 0));
        b->uploadPending = false;
    }
    for (int f = 0; f < 5; ++f)
        if (counts[f])
            CN_CUDA(cudaMemcpyAsync(b->dTiles + b->tileOffset[f], tiles + b->tileOffset[f], size_t(counts[f]) * sizeof(uint2),
                                    cudaMemcpyHostToDevice, st));
    CN_CUDA(cudaMemcpyAsync(b->dCounts, counts, 8 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    if (nt) CN_CUDA(cudaMemcpyAsync(b->dTargets, targets, size_t(nt) * sizeof(cn::BodyTarget), cudaMemcpyHostToDevice, st));
    if (count && (b->clusterCtas || b->schedule != CN_XPBD_GATHER))
        CN_CUDA(cudaMemcpyAsync(b->dScenes, sceneList, size_t(cn::kSceneListStride) * count * sizeof(uint2),
                                cudaMemcpyHostToDevice, st));
    CN_CUDA(cudaEventRecord(b->stageDone[k], st));
    CN_CUDA(cudaGraphLaunch(b->graphExec, st));
    CN_CUDA(cudaGetLastError());
    ++b->ticks;
    return CN_OK;
}

CN_API cn_status cn_batch_read_particles(cn_batch *b, uint32_t scene_id, float *x, float *v, uint32_t count)
{
    if (!b || scene_id >= b->scenes.size() || !b->scenes[scene_id].live)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_read_particles: no such scene");
    const BatchScene &sc = b->scenes[scene_id];
    if (count > sc.p.count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_read_particles: count > particles");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    if (x) CN_CUDA(cudaMemcpy(x, b->s.x + sc.p.start, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    if (v) CN_CUDA(cudaMemcpy(v, b->s.v + sc.p.start, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    return CN_OK;
}

CN_API cn_status cn_batch_export_scene(cn_batch *b, uint32_t scene_id, cn_world_soa *w)
{
    if (!b || !w || scene_id >= b->scenes.size() || !b->scenes[scene_id].live)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_export_scene: no such scene");
    const BatchScene &sc = b->scenes[scene_id];
    if (w->particle_count != sc.p.count || w->rigid_body_count != sc.b.count)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_export_scene: the SoA does not match the scene");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    const cn::Scene &s = b->s;
    CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->positions_inv_mass)), s.x + sc.p.start, sizeof(float4) * sc.p.count, cudaMemcpyDeviceToHost));
    CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->velocities)), s.v + sc.p.start, sizeof(float4) * sc.p.count, cudaMemcpyDeviceToHost));
    if (sc.b.count) {
        const size_t nb = sizeof(float4) * sc.b.count;
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_positions_inv_mass)), s.bodyPos + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_orientations)), s.bodyRot + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_linear_velocities)), s.bodyLin + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_angular_velocities)), s.bodyAng + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_kinematic_target_positions)), s.bodyKinPos + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_kinematic_target_orientations)), s.bodyKinRot + sc.b.start, nb, cudaMemcpyDeviceToHost));
        CN_CUDA(cudaMemcpy(const_cast<void *>(static_cast<const void *>(w->body_kinematic_target_flags)), s.bodyKinFlags + sc.b.start, sizeof(uint32_t) * sc.b.count,
                           cudaMemcpyDeviceToHost));
    }
    return CN_OK;
}

CN_API cn_status cn_batch_get_stats(cn_batch *b, cn_batch_stats *out)
{
    if (!b || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_get_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    for (const auto &sc : b->scenes)
        if (sc.live) ++out->resident_scenes;
    out->particles_used = b->aP.used(); out->particle_capacity = b->aP.capacity();
    out->edges_used = b->aE.used(); out->edge_capacity = b->aE.capacity();
    out->tets_used = b->aT.used(); out->tet_capacity = b->aT.capacity();
    out->budget_bytes = b->desc.memory_budget_bytes;
    out->budget_used_bytes = b->bytesAdmitted;
    out->pool_bytes = b->arenaBytes;
    out->ticks = b->ticks;
    out->tile_elements = b->tileElems;
    out->grid_blocks = b->grid;
    out->fused_cluster_ctas = b->clusterCtas;
    out->xpbd_schedule = b->schedule;
    return CN_OK;
}

CN_API cn_status cn_batch_set_xpbd_schedule(cn_batch *b, uint32_t schedule)
{
    if (!b) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_xpbd_schedule: null batch");
    if (schedule > CN_XPBD_COLOUR_GAUSS_SEIDEL)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_xpbd_schedule: unknown schedule");
    if (schedule != CN_XPBD_GATHER && !b->coloured)
        return setError(CN_ERR_UNSUPPORTED, "cn_batch_set_xpbd_schedule: the batch was created without colour tables");
    if (schedule != CN_XPBD_GATHER && b->clusterCtas)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_xpbd_schedule: the fused iterations run the gather schedule");
    if (schedule == b->schedule) return CN_OK;
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    b->schedule = schedule;
    releaseGraph(b);
    return CN_OK;
}

CN_API cn_status cn_batch_set_fused(cn_batch *b, uint32_t cluster_ctas)
{
    if (!b) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_fused: null batch");
    if (cluster_ctas != 0u && cluster_ctas != 1u && cluster_ctas != 2u && cluster_ctas != 4u && cluster_ctas != 8u)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_fused: cluster_ctas is 0, 1, 2, 4 or 8");
    if (cluster_ctas && b->schedule != CN_XPBD_GATHER)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_fused: the fused iterations run the gather schedule");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    uint32_t clusters = 0;
    if (cluster_ctas) {
        clusters = cn::batchFusedClusters(cluster_ctas);
        if (clusters == 0u) return setError(CN_ERR_UNSUPPORTED, "cn_batch_set_fused: clusters of this size cannot be formed");
        clusters = std::min<uint32_t>(clusters, std::max<uint32_t>(b->desc.max_scenes, 1u));
    }
    b->clusterCtas = cluster_ctas;
    b->clusters = clusters;
    releaseGraph(b);
    return CN_OK;
}

CN_API cn_status cn_batch_set_schedule(cn_batch *b, uint32_t tile_elements, uint32_t blocks_per_sm)
{
    if (!b || tile_elements < 32u || blocks_per_sm == 0u)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_set_schedule: tile_elements >= 32, blocks_per_sm >= 1");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    b->tileElems = tile_elements;
    b->blocksPerSm = blocks_per_sm;
    b->grid = b->smCount * blocks_per_sm;
    releaseGraph(b);
    return allocWorkLists(b);
}

// Times one tick of the given scenes under each (tile size, blocks per SM) candidate, the fused
// iterations and, in a colour-Jacobi batch, colour Jacobi, and keeps the fastest.  The trial
// ticks' effects are discarded: the scenes' particles, velocities and bodies are restored from
// host copies, and the correction records (which a tet that keeps its previous corrections
// re-applies) from a device copy.
CN_API cn_status cn_batch_autotune(cn_batch *b, const uint32_t *scene_ids, uint32_t count, float frame_dt,
                                   cn_batch_tuning *out)
{
    if (!b || !out || (count && !scene_ids)) return setError(CN_ERR_INVALID_ARGUMENT, "cn_batch_autotune: null argument");
    CN_CUDA(cudaSetDevice(b->device));
    CN_CUDA(cudaDeviceSynchronize());
    cn::Scene &s = b->s;
    // snapshot of the mutable state
    std::vector<float4> x(b->P), v(b->P), xp(b->P), bp(b->B), br(b->B), bl(b->B), ba(b->B), kp(b->B), kr(b->B);
    std::vector<uint32_t> kf(b->B);
    auto save = [&](bool toHost) -> cudaError_t {
        struct Item { void *dev; void *host; size_t bytes; };
        const Item items[] = {{s.x, x.data(), x.size() * 16}, {s.v, v.data(), v.size() * 16},
                              {s.xprev, xp.data(), xp.size() * 16}, {s.bodyPos, bp.data(), bp.size() * 16},
                              {s.bodyRot, br.data(), br.size() * 16}, {s.bodyLin, bl.data(), bl.size() * 16},
                              {s.bodyAng, ba.data(), ba.size() * 16}, {s.bodyKinPos, kp.data(), kp.size() * 16},
                              {s.bodyKinRot, kr.data(), kr.size() * 16}, {s.bodyKinFlags, kf.data(), kf.size() * 4}};
        for (const Item &it : items) {
            const cudaError_t e = toHost ? cudaMemcpy(it.host, it.dev, it.bytes, cudaMemcpyDeviceToHost)
                                         : cudaMemcpy(it.dev, it.host, it.bytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    CN_CUDA(save(true));
    // the correction records, kept on the device (edge and tet gather slots, colour-ordered tet records)
    struct DevItem { void *dev; size_t bytes; };
    const DevItem records[] = {{s.edgeCorr, sizeof(float4) * 2 * size_t(b->E)},
                               {s.tetCorr, sizeof(float4) * 4 * size_t(b->T)},
                               {s.tetRecC, s.tetRecC ? sizeof(float4) * 4 * size_t(b->T) : 0}};
    size_t recordBytes = 0;
    for (const DevItem &it : records) recordBytes += it.bytes;
    uint8_t *recordCopy = nullptr;
    CN_CUDA(cudaMalloc(&recordCopy, std::max<size_t>(recordBytes, 16)));
    auto copyRecords = [&](bool toCopy) -> cudaError_t {
        size_t at = 0;
        for (const DevItem &it : records) {
            if (!it.bytes) continue;
            const cudaError_t e = toCopy ? cudaMemcpy(recordCopy + at, it.dev, it.bytes, cudaMemcpyDeviceToDevice)
                                         : cudaMemcpy(it.dev, recordCopy + at, it.bytes, cudaMemcpyDeviceToDevice);
            if (e != cudaSuccess) return e;
            at += it.bytes;
        }
        return cudaSuccess;
    };
    if (copyRecords(true) != cudaSuccess) {
        cudaFree(recordCopy);
        return setError(CN_ERR_CUDA, "cn_batch_autotune: cannot copy the correction records");
    }
    const std::vector<cn::BodyTarget> staged = b->pendingTargets;
    b->pendingTargets.clear();
    const uint32_t tiles[] = {128, 256, 512, 1024};
    const uint32_t blocks[] = {4, 8, 16, 32};
    const uint32_t clusterSizes[] = {1, 2, 4, 8};
    float best = 1e30f;
    uint32_t bestTile = b->tileElems, bestBlocks = b->blocksPerSm, bestCtas = 0, bestSchedule = b->schedule;
    const uint32_t created = b->desc.solver.soft.xpbd_schedule;
    const uint32_t tileSchedule = created == CN_XPBD_COLOUR_GAUSS_SEIDEL ? created : uint32_t(CN_XPBD_GATHER);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::memset(out, 0, sizeof(*out));
    uint32_t n = 0;
    const uint32_t capacity = uint32_t(sizeof(out->candidates) / sizeof(out->candidates[0]));
    // warm-up (capture + first replay), then three timed ticks; the state is restored after
    auto trial = [&](uint32_t te, uint32_t bps, uint32_t ctas, uint32_t schedule) -> cn_status {
        cn_status st = cn_batch_step(b, scene_ids, count, frame_dt, b->ownStream);
        if (st != CN_OK) return st;
        cudaEventRecord(e0, b->ownStream);
        for (int r = 0; r < 3; ++r) cn_batch_step(b, scene_ids, count, frame_dt, b->ownStream);
        cudaEventRecord(e1, b->ownStream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 3.0f;
        if (n < capacity) out->candidates[n++] = cn_batch_candidate{te, bps, ms, ctas, schedule};
        if (ms < best) {
            best = ms;
            bestTile = te;
            bestBlocks = bps;
            bestCtas = ctas;
            bestSchedule = schedule;
        }
        cudaError_t e = save(false);
        if (e == cudaSuccess) e = copyRecords(false);
        return e == cudaSuccess ? CN_OK : setError(CN_ERR_CUDA, std::string("cn_batch_autotune: ") + cudaGetErrorString(e));
    };
    cn_status st = cn_batch_set_fused(b, 0);
    if (st == CN_OK) st = cn_batch_set_xpbd_schedule(b, tileSchedule);
    for (uint32_t te : tiles)
        for (uint32_t bps : blocks) {
            if (st == CN_OK) st = cn_batch_set_schedule(b, te, bps);
            if (st == CN_OK) st = trial(te, bps, 0, tileSchedule);
        }
    // the persistent fused iterations (gather), with the other phases at the best tile schedule
    const uint32_t tileForFused = bestTile, blocksForFused = bestBlocks;
    if (st == CN_OK) st = cn_batch_set_schedule(b, tileForFused, blocksForFused);
    for (uint32_t ctas : clusterSizes) {
        if (st != CN_OK || tileSchedule != CN_XPBD_GATHER) break;
        if (cn_batch_set_fused(b, ctas) != CN_OK) {
            cn::clearError(); // clusters of this size cannot be formed: not a candidate
            continue;
        }
        st = trial(tileForFused, blocksForFused, ctas, CN_XPBD_GATHER);
    }
    // colour Jacobi at the best tile size, its colour passes over grids of 4 .. 32 blocks per SM
    if (st == CN_OK && created == CN_XPBD_COLOUR_JACOBI) {
        st = cn_batch_set_fused(b, 0);
        if (st == CN_OK) st = cn_batch_set_xpbd_schedule(b, CN_XPBD_COLOUR_JACOBI);
        for (uint32_t bps : blocks) {
            if (st == CN_OK) st = cn_batch_set_schedule(b, tileForFused, bps);
            if (st == CN_OK) st = trial(tileForFused, bps, 0, CN_XPBD_COLOUR_JACOBI);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out->candidate_count = n;
    out->tile_elements = bestTile;
    out->blocks_per_sm = bestBlocks;
    out->cluster_ctas = bestCtas;
    out->xpbd_schedule = bestSchedule;
    out->tick_ms = best;
    if (st == CN_OK) st = cn_batch_set_fused(b, 0);
    if (st == CN_OK) st = cn_batch_set_xpbd_schedule(b, bestSchedule);
    if (st == CN_OK) st = cn_batch_set_schedule(b, bestTile, bestBlocks);
    if (st == CN_OK) st = cn_batch_set_fused(b, bestCtas);
    const cudaError_t restored = save(false) == cudaSuccess ? copyRecords(false) : cudaErrorUnknown;
    cudaFree(recordCopy);
    if (restored != cudaSuccess) return setError(CN_ERR_CUDA, "cn_batch_autotune: cannot restore the scenes' state");
    b->pendingTargets = staged;
    b->ticks = 0;
    return st;
}

} // extern "C"
