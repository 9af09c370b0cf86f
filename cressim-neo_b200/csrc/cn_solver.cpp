// cn_solver.cpp -- PhysicsSolver mirror behind the C ABI: device buffers, upload, the substep
// schedule and its CUDA-graph replay.
//
// Reference: include/physics/physics_solver.h:150-205 (API), src/physics/physics_solver.cpp:173-1401
// (syncWorldState + step), src/physics/physics_scene_gpu_state.cpp (buffers, incidence tables,
// readback).  The pass order and gating flags of step() are reproduced; passes the reference
// dispatches with provably empty inputs (for example particle-particle contacts in a scene
// whose particles are all fluid) are not launched.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_device.h"
#include "cn_internal.h"

namespace cn {

thread_local std::string g_lastError;

cn_status setError(cn_status status, const std::string &message)
{
    g_lastError = message;
    return status;
}
void clearError() { g_lastError.clear(); }

} // namespace cn

using cn::setError;

struct cn_solver {
    cn_solver_desc desc{};
    int device = 0;
    // what cn_solver_update_world may not change: the constraints' particle (segment) indices,
    // which the incidence tables and colourings are built from, and the body types
    uint64_t topologyHash = 0;
    std::vector<uint32_t> bodyTypes;
    uint32_t attributeStructure = 0; // attributeStructure() of the synced world
    std::vector<uint32_t> queryOrder; // the colliders queried (enabled, of a present body), in order
    std::vector<cn::PackedEdge> edgesC; // host staging of the colour-ordered copies (coloured schedules)
    std::vector<cn_soft_tet> tetsC;
    cudaStream_t ownStream = nullptr;
    cn::Scene s{};
    cn::Config cfg{};
    void *arena = nullptr;
    size_t arenaBytes = 0;
    void *sortScratch = nullptr;
    uint32_t *scanScratch = nullptr;
    size_t scanScratchBytes = 0;
    float *hostX = nullptr, *hostV = nullptr;
    bool synced = false;
    bool hasFluid = false, ppPossible = false, rigidPossible = false, hasBroadphase = false, hasDynamic = false;
    bool fluidBoundaryLists = false, vorticity = false, fluidXMoves = false;
    uint32_t nProxy = 0;          // rigid proxy particles (the leading particles)
    bool proxyContacts = false;   // proxy particle -> collider contacts in the rigid contact solve
    uint32_t substeps = 1, fluidIt = 1, softIt = 1, contactIt = 1, maxIt = 1, jointIt = 1, rrIt = 1;
    bool rigidRigid = false;       // dynamic bodies among >= 2 colliders: rigid-rigid contacts
    void *rigidScratch = nullptr;
    bool postUpdateNeighbors = false, writeFluidDebug = false, forceBroadphase = false, walkCells = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    float graphDt = -1.0f;
    uint64_t bindingGeneration = 0;
    // host-side sizes needed by debug reads
    uint32_t cellRangeCapacity = 0;
    // timing probes: event pairs recorded around kernel groups of the captured frame
    bool timing = false;
    struct Probe { const char *name; cudaEvent_t begin, end; };
    std::vector<Probe> probes;
    uint32_t graphKernelNodes = 0, graphNodes = 0;
    uint32_t contactMaterialCapacity = 0, fluidMaterialCapacity = 0, surfIdxCapacity = 0;
    // XPBD schedule: per-family colourings (coloured schedules), the plan the launches read, and
    // whether each substep's iterations run in one cluster kernel
    cn::Colouring colouring[cn::kFamilies];
    cn::XpbdPlan plan{};
    bool fused = false;
    cn::FusedShape fusedShape{};
    bool fusedShapeQueried = false;
    // Concurrent branches of an iteration (gather schedule): families and the fluid chain whose
    // particles are disjoint run on side streams forked from and joined to the frame's stream,
    // each particle seeing the same updates in the same order.
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, joinFluid = nullptr, joinStrands = nullptr, afterEdges = nullptr, joinBends = nullptr;
    bool branchFluid = false, branchStrands = false, branchBends = false;
};

namespace {

#define CN_CUDA(call)                                                                                  \
    do {                                                                                               \
        const cudaError_t e__ = (call);                                                                \
        if (e__ != cudaSuccess)                                                                        \
            return setError(e__ == cudaErrorMemoryAllocation ? CN_ERR_OUT_OF_MEMORY : CN_ERR_CUDA,     \
                            std::string(#call) + ": " + cudaGetErrorString(e__));                      \
    } while (0)

void releaseGraph(cn_solver *sv)
{
    if (sv->graphExec) cudaGraphExecDestroy(sv->graphExec);
    if (sv->graph) cudaGraphDestroy(sv->graph);
    sv->graphExec = nullptr;
    sv->graph = nullptr;
    sv->graphDt = -1.0f;
    for (auto &p : sv->probes) {
        cudaEventDestroy(p.begin);
        cudaEventDestroy(p.end);
    }
    sv->probes.clear();
}

// Runs `fn` between two recorded events when timing is on (the events become graph nodes).
template <class F> void probe(cn_solver *sv, const char *name, cudaStream_t st, F &&fn)
{
    if (!sv->timing) {
        fn();
        return;
    }
    cn_solver::Probe p{name, nullptr, nullptr};
    cudaEventCreate(&p.begin);
    cudaEventCreate(&p.end);
    // External records become event-record nodes of the captured graph (plain records inside a
    // capture only express ordering).
    cudaEventRecordWithFlags(p.begin, st, cudaEventRecordExternal);
    fn();
    cudaEventRecordWithFlags(p.end, st, cudaEventRecordExternal);
    sv->probes.push_back(p);
}

void releaseBuffers(cn_solver *sv)
{
    releaseGraph(sv);
    if (sv->arena) cudaFree(sv->arena);
    sv->arena = nullptr;
    sv->arenaBytes = 0;
    sv->s = cn::Scene{};
    sv->synced = false;
}

// Lays out every device buffer; `upload` false only sizes the arena.
void layout(cn_solver *sv, cn::Arena &a, const cn_world_soa &w, const cn::Incidence &edgeI, const cn::Incidence &bendI,
            const cn::Incidence &tetI, const cn::Incidence &segI, const cn::Incidence &jointI)
{
    cn::Scene &s = sv->s;
    const uint32_t N = w.particle_count;
    s.N = N;
    s.x = a.take<float4>(N); s.xprev = a.take<float4>(N); s.v = a.take<float4>(N);
    s.radii = a.take<float>(N);
    s.kinds = a.take<uint32_t>(N);
    s.meta = a.take<uint4>(N);
    s.matIdx = a.take<uint32_t>(N);
    s.fluidMatIdx = a.take<uint32_t>(N);
    s.ownerTypes = a.take<uint32_t>(N);
    s.ownerIdx = a.take<uint32_t>(N);
    s.fluidGroup = a.take<uint32_t>(N);
    s.adjOff = a.take<uint32_t>(N);
    s.adjCnt = a.take<uint32_t>(N);
    s.adjIdx = a.take<uint32_t>(std::max<uint32_t>(w.adjacency_index_count, 1u));
    s.contactMaterials = a.take<float4>(std::max<uint32_t>(w.contact_material_count, 1u));
    s.fluidMaterials = a.take<cn_fluid_material>(std::max<uint32_t>(w.fluid_material_count, 1u));
    s.E = w.edge_count; s.Bn = w.bend_count; s.D = w.dihedral_count; s.T = w.tet_count;
    s.S = w.strand_segment_count; s.J = w.strand_joint_count; s.SD = w.strand_distance_count;
    s.edges = a.take<cn_soft_edge>(s.E);
    s.bends = a.take<cn_soft_bend>(s.Bn);
    s.dihedrals = a.take<cn_cloth_dihedral>(s.D);
    s.tets = a.take<cn_soft_tet>(s.T);
    s.segs = a.take<cn_strand_segment>(s.S);
    s.joints = a.take<cn_strand_joint>(s.J);
    s.dists = a.take<cn_strand_distance>(s.SD);
    s.segOrient = a.take<float4>(s.S);
    s.edgeRanges = a.take<uint2>(N);
    s.bendRanges = a.take<uint2>(N);
    s.tetRanges = a.take<uint2>(N);
    s.segRanges = a.take<uint2>(N); s.segInc = a.take<uint2>(segI.inc.size());
    s.segJointRanges = a.take<uint2>(s.S); s.segJointInc = a.take<uint2>(jointI.inc.size());
    s.edgeDst = a.take<uint32_t>(size_t(s.E) * 2);
    s.bendDst = a.take<uint32_t>(size_t(s.Bn + s.D) * 4);
    s.tetDst = a.take<uint32_t>(size_t(s.T) * 4);
    s.distDst = a.take<uint32_t>(size_t(s.SD) * 2);
    s.edgeLambda = a.take<float>(s.E);
    s.bendLambda = a.take<float>(s.Bn + s.D);
    s.tetLambda = a.take<float>(s.T);
    s.distLambda = a.take<float>(s.SD);
    s.segLambda = a.take<float4>(s.S);
    s.jointLambda = a.take<float4>(s.J);
    s.edgeCorr = a.take<float4>(size_t(s.E) * 2);
    s.bendCorr = a.take<float4>(size_t(s.Bn + s.D) * 4);
    s.tetCorr = a.take<float4>(size_t(s.T) * 4);
    s.segCorr = a.take<float4>(size_t(s.S) * 3);
    s.jointCorr = a.take<float4>(size_t(s.J) * 2);
    // the distance gather walks every strand-segment incidence entry: slots of segments without a
    // distance constraint stay zero
    s.distCorr = a.take<float4>(s.SD ? std::max<size_t>(size_t(s.SD) * 2, segI.inc.size()) : 0);
    s.posCorr = a.take<float4>(N);
    s.velCorr = a.take<float4>(N);
    for (uint32_t f = 0; f < cn::kFamilies; ++f) {
        const cn::Colouring &col = sv->colouring[f];
        s.colOrder[f] = col.colours() ? a.take<uint32_t>(col.order.size()) : nullptr;
        sv->plan.devStarts[f] = col.colours() ? a.take<uint32_t>(col.starts.size()) : nullptr;
    }
    const bool coloured = sv->plan.schedule != CN_XPBD_GATHER;
    // the coloured schedules read the edges and tets in colour order (a colour is a contiguous
    // range); their lambdas are indexed by colour position and the tets' last corrections sit in
    // the tet records, by colour position, which the gather schedule would use otherwise
    s.edgesC = coloured && s.E ? a.take<cn::PackedEdge>(s.E) : nullptr;
    s.tetsC = coloured && s.T ? a.take<cn_soft_tet>(s.T) : nullptr;
    s.tetRecC = s.tetsC ? s.tetCorr : nullptr;
    s.softAcc = coloured ? a.take<float4>(N) : nullptr;
    s.orientAcc = coloured ? a.take<float4>(w.strand_segment_count) : nullptr;
    s.B = w.rigid_body_count;
    s.C = w.collider_count;
    const uint32_t B = std::max<uint32_t>(s.B, 1u), C = std::max<uint32_t>(s.C, 1u);
    s.bodyPos = a.take<float4>(B); s.bodyRot = a.take<float4>(B); s.bodyLin = a.take<float4>(B);
    s.bodyAng = a.take<float4>(B); s.bodyScale = a.take<float4>(B); s.bodyInvInertia = a.take<float4>(B);
    s.bodyType = a.take<uint32_t>(B);
    s.bodyKinPos = a.take<float4>(B); s.bodyKinRot = a.take<float4>(B); s.bodyKinFlags = a.take<uint32_t>(B);
    s.bodyColRanges = a.take<uint2>(B);
    s.bodyColIdx = a.take<uint32_t>(std::max<uint32_t>(w.body_collider_index_count, 1u));
    s.colGeo = a.take<cn_collider_geometry>(C);
    s.colBp = a.take<cn_collider_broadphase>(C);
    s.colMat = a.take<float4>(C);
    s.prevBodyPos = a.take<float4>(B); s.prevBodyRot = a.take<float4>(B);
    s.predBodyPos = a.take<float4>(B); s.predBodyRot = a.take<float4>(B);
    s.predBodyLin = a.take<float4>(B); s.predBodyAng = a.take<float4>(B);
    s.colAabbMin = a.take<float4>(C); s.colAabbMax = a.take<float4>(C);
    s.nProxy = sv->nProxy;
    s.proxyLocal = a.take<float4>(sv->nProxy);
    s.bodyProxyMat = a.take<float4>(sv->nProxy ? B : 0u);
    s.hasDynamic = sv->hasDynamic ? 1u : 0u;
    if (sv->hasDynamic) {
        s.bodyTransCorr = a.take<float4>(B); s.bodyRotCorr = a.take<float4>(B);
        s.bodyLinVelCorr = a.take<float4>(B); s.bodyAngVelCorr = a.take<float4>(B);
    }
    s.rrCapacity = 0;
    s.proxyCapacity = 0;
    s.rrSlotCapacity = 0;
    if (sv->rigidRigid) {
        // estimateRigidCandidatePairCapacityFromColliderCount (rigid_body_common.cpp:35-47): 32
        // pairs per collider; proxy contact slots: 8 per proxy, the particle-rigid candidate rate
        const uint32_t P = std::max<uint32_t>(64u, 32u * C);
        s.rrCapacity = P;
        s.proxyCapacity = sv->proxyContacts ? std::max<uint32_t>(64u, cn::rigidPairsPerParticle(sv->desc) * sv->nProxy) : 0u;
        s.rrCount = a.take<uint32_t>(C); s.rrOffset = a.take<uint32_t>(C);
        s.rrStage = a.take<uint2>(size_t(C) * 64u); // kPairStage per collider
        const uint32_t K = P * cn::kRigidPairContacts + s.proxyCapacity;
        s.rrSlotCapacity = K;
        s.rrPairs = a.take<uint2>(P);
        s.rrContacts = a.take<cn::RigidPairContact>(K);
        s.rrSlots = a.take<cn::RigidSlot>(K);
        s.rrKeyA = a.take<uint32_t>(K); s.rrValA = a.take<uint32_t>(K);
        s.rrKeyB = a.take<uint32_t>(K); s.rrValB = a.take<uint32_t>(K);
        s.rrHead = a.take<uint32_t>(K); s.rrGroupOf = a.take<uint32_t>(K);
        s.rrGroups = a.take<uint2>(K);
        sv->rigidScratch = a.take<uint8_t>(cn::rigidScratchBytes(C, K));
    } else if (sv->fluidBoundaryLists) {
        sv->rigidScratch = a.take<uint8_t>(cn::rigidScratchBytes(C, 1u));
    }
    if (sv->rigidRigid || sv->fluidBoundaryLists) { // the LBVH over the colliders
        s.bvhKeyA = a.take<uint32_t>(C); s.bvhValA = a.take<uint32_t>(C);
        s.bvhKeyB = a.take<uint32_t>(C); s.bvhValB = a.take<uint32_t>(C);
        s.bvhChildren = a.take<uint2>(C);
        s.bvhParent = a.take<uint32_t>(2 * C); s.bvhVisits = a.take<uint32_t>(C);
        s.bvhMin = a.take<float4>(2 * C); s.bvhMax = a.take<float4>(2 * C);
        s.bvhWide = a.take<float4>(4 * C);
        s.bvhBounds = a.take<float4>(2);
    }
    s.colBvh = sv->fluidBoundaryLists ? 1u : 0u;
    s.colFrame = a.take<float4>(size_t(C) * 4);
    s.colQueryOrder = a.take<uint32_t>(C);
    {
        const cn_surface_render_data *sr = w.surface_render;
        s.surfV = sr ? sr->vertex_count : 0u;
        s.surfT = sr ? sr->triangle_count : 0u;
        s.surfS = sr ? sr->surface_count : 0u;
        s.surfChunks = 0;
        for (uint32_t k = 0; k < s.surfS; ++k) s.surfChunks += (sr->surface_particle_ranges[2 * k + 1] + 63u) / 64u;
        const uint32_t idxCount = sr ? sr->vertex_triangle_index_count : 0u;
        s.surfBind = a.take<uint4>(size_t(s.surfV) * 2);
        s.surfFallback = a.take<float4>(s.surfV);
        s.surfRanges = a.take<uint4>(s.surfV);
        s.surfIdx = a.take<uint32_t>(idxCount);
        s.surfTri = a.take<uint4>(s.surfT);
        s.surfChunk = a.take<uint4>(s.surfChunks);
        s.surfChunkRange = a.take<uint2>(s.surfS);
        s.surfPos = a.take<float4>(s.surfV);
        s.surfNrm = a.take<float4>(s.surfV);
        s.surfTriN = a.take<float4>(s.surfT);
        s.surfChunkAabb = a.take<float4>(size_t(s.surfChunks) * 2);
        s.surfWorldAabb = a.take<float4>(size_t(s.surfS) * 2);
    }
    if (sv->hasBroadphase) {
        s.entries = a.take<int4>(N);
        s.keysA = a.take<uint32_t>(N); s.keysB = a.take<uint32_t>(N);
        s.valsA = a.take<uint32_t>(N); s.valsB = a.take<uint32_t>(N);
        s.rank = a.take<uint32_t>(N);
        const uint32_t cap = cn::nextPow2(std::max<uint32_t>(2u * N, 64u));
        s.tableMask = cap - 1u;
        s.tableKeys = a.take<uint32_t>(cap);
        s.tableStart = a.take<uint32_t>(cap);
        s.cellEnd = a.take<uint32_t>(N);
        s.sCell = a.take<int4>(N);
    }
    s.hasFluid = sv->hasFluid ? 1u : 0u;
    if (sv->hasFluid) {
        s.Xs = a.take<float4>(N); s.P = a.take<float4>(N);
        s.Da = a.take<float4>(N); s.Db = a.take<float4>(N);
        s.Cs = a.take<float4>(N); s.Dx = a.take<float4>(N);
        s.sMeta = a.take<uint4>(N);
        s.sInfo = a.take<uint32_t>(N);
        s.sBoundary = a.take<unsigned long long>(N);
        if (sv->fluidBoundaryLists) {
            // physics_scene_gpu_state.cpp:728-729: 32 boundary candidates per particle
            s.bListCap = std::max<uint32_t>(N * 32u, 64u);
            s.bCount = a.take<uint32_t>(N); s.bOffset = a.take<uint32_t>(N);
            s.bList = a.take<uint32_t>(s.bListCap);
        }
        s.runFlag = a.take<uint32_t>(N);
        s.runIdx = a.take<uint32_t>(N);
        s.runStartOf = a.take<uint32_t>(N);
        s.runNbr = a.take<uint2>(size_t(N) * 27u);
        s.runKey = a.take<uint32_t>(N); s.runVal = a.take<uint32_t>(N);
        s.runKeyB = a.take<uint32_t>(N); s.runValB = a.take<uint32_t>(N);
        s.runHashStart = a.take<uint32_t>(N); s.runLen = a.take<uint32_t>(N);
        s.runTotal = a.take<uint32_t>(1);
        s.runLenSorted = a.take<uint32_t>(N); s.runCompStart = a.take<uint32_t>(N);
        s.runComp = a.take<uint32_t>(N); s.runPos = a.take<uint32_t>(N);
        s.cvals = a.take<uint32_t>(N); s.cCell = a.take<int4>(N); s.cRun = a.take<uint32_t>(N);
        s.fluidMaxDelta = a.take<uint32_t>(64);
        // Superset lists (k_fluidNeighborsDensity modes 1 and 2).  Without particle-particle
        // contacts fluid x is fixed over the iterations and the positions are double-buffered;
        // with them the gather records each iteration's largest move from the build positions P0.
        s.supCap = 160u;
        s.sup = a.take<uint32_t>(size_t(N) * s.supCap);
        s.supCount = a.take<uint32_t>(N);
        if (!sv->fluidXMoves) s.Pb = a.take<float4>(N);
        else s.P0 = a.take<float4>(N);
        s.maxNbr = sv->desc.max_fluid_neighborhood;
        s.nbr = a.take<uint32_t>(std::max<size_t>(size_t(N) * s.maxNbr, 1));
        s.nbrCount = a.take<uint32_t>(N);
        if (sv->vorticity) s.fluidVort = a.take<float4>(N);
    }
    if (sv->rigidPossible || sv->proxyContacts) {
        s.candCount = a.take<uint32_t>(N);
        s.candOffset = a.take<uint32_t>(N);
        s.rigidPairCapacity = std::max<uint32_t>(N * cn::rigidPairsPerParticle(sv->desc), 64u);
        s.rigidPairs = a.take<uint2>(s.rigidPairCapacity);
        s.rigidContacts = a.take<cn::RigidContact>(s.rigidPairCapacity);
    }
    if (sv->ppPossible) {
        s.ppCount = a.take<uint32_t>(N);
        s.ppStage = a.take<uint2>(size_t(N) * 8u); // kPairStageP per particle
        s.ppOffset = a.take<uint32_t>(N);
        s.particlePairCapacity = std::max<uint32_t>(N * 8u, 64u);
        s.particlePairs = a.take<uint2>(s.particlePairCapacity);
        s.particleContacts = a.take<cn::ParticleContact>(s.particlePairCapacity);
    }
    s.meta_ = a.take<cn::DeviceMeta>(1);
    sv->sortScratch = a.take<uint8_t>(sv->hasBroadphase ? cn::radixSortScratchBytes(N) : 0);
    sv->scanScratchBytes = (size_t(2) * N + 4) * sizeof(uint32_t) + cn::scanScratchBytes(std::max<uint32_t>(N, 1u));
    sv->scanScratch = a.take<uint32_t>(sv->scanScratchBytes / sizeof(uint32_t));
}

template <class T> cudaError_t up(const T *dst, const void *src, size_t count, cudaStream_t st)
{
    if (!count || !src) return cudaSuccess;
    return cudaMemcpyAsync(const_cast<T *>(dst), src, count * sizeof(T), cudaMemcpyHostToDevice, st);
}

// Index checks of the surface render arrays (the kernels trust them), and the 64-particle bounds
// chunks of each surface (physics_scene_gpu_state.cpp:3482-3500).
std::string checkSurfaceRender(const cn_world_soa &w)
{
    const cn_surface_render_data *sr = w.surface_render;
    if (!sr) return {};
    const uint32_t N = w.particle_count;
    auto need = [](uint32_t n, const void *p) { return n == 0u || p != nullptr; };
    if (!need(sr->vertex_count, sr->vertex_bindings) || !need(sr->vertex_count, sr->fallback_normals) ||
        !need(sr->vertex_count, sr->vertex_triangle_ranges) ||
        !need(sr->vertex_triangle_index_count, sr->vertex_triangle_indices) ||
        !need(sr->triangle_count, sr->triangle_particle_indices) || !need(sr->surface_count, sr->surface_particle_ranges))
        return "surface render: missing array";
    for (uint32_t v = 0; v < sr->vertex_count; ++v) {
        for (uint32_t p : sr->vertex_bindings[v].particle_indices)
            if (p >= N) return "surface render: vertex binding particle index out of range";
        const cn_surface_triangle_range &r = sr->vertex_triangle_ranges[v];
        if (uint64_t(r.start) + r.count > sr->vertex_triangle_index_count)
            return "surface render: vertex triangle range out of range";
    }
    for (uint32_t k = 0; k < sr->vertex_triangle_index_count; ++k)
        if (sr->vertex_triangle_indices[k] >= sr->triangle_count) return "surface render: triangle index out of range";
    for (uint32_t t = 0; t < sr->triangle_count; ++t)
        for (uint32_t k = 0; k < 3; ++k)
            if (sr->triangle_particle_indices[4 * size_t(t) + k] >= N)
                return "surface render: triangle particle index out of range";
    for (uint32_t k = 0; k < sr->surface_count; ++k)
        if (uint64_t(sr->surface_particle_ranges[2 * k]) + sr->surface_particle_ranges[2 * k + 1] > N)
            return "surface render: surface particle range out of range";
    return {};
}

cn_status uploadSurfaceRender(cn_solver *sv, const cn_world_soa &w, cudaStream_t st)
{
    const cn_surface_render_data *sr = w.surface_render;
    const cn::Scene &s = sv->s;
    if (!sr) return CN_OK;
    CN_CUDA(up(s.surfBind, reinterpret_cast<const uint4 *>(sr->vertex_bindings), size_t(s.surfV) * 2, st));
    CN_CUDA(up(s.surfFallback, reinterpret_cast<const float4 *>(sr->fallback_normals), s.surfV, st));
    CN_CUDA(up(s.surfRanges, reinterpret_cast<const uint4 *>(sr->vertex_triangle_ranges), s.surfV, st));
    CN_CUDA(up(s.surfIdx, sr->vertex_triangle_indices, sr->vertex_triangle_index_count, st));
    CN_CUDA(up(s.surfTri, reinterpret_cast<const uint4 *>(sr->triangle_particle_indices), s.surfT, st));
    std::vector<uint4> chunks;
    std::vector<uint2> ranges(s.surfS);
    for (uint32_t k = 0; k < s.surfS; ++k) {
        const uint32_t off = sr->surface_particle_ranges[2 * k], cnt = sr->surface_particle_ranges[2 * k + 1];
        ranges[k] = make_uint2(uint32_t(chunks.size()), 0u);
        for (uint32_t o = 0; o < cnt; o += 64u) {
            chunks.push_back(make_uint4(k, off + o, std::min(64u, cnt - o), 0u));
            ++ranges[k].y;
        }
    }
    CN_CUDA(up(s.surfChunk, chunks.data(), chunks.size(), st));
    CN_CUDA(up(s.surfChunkRange, ranges.data(), ranges.size(), st));
    CN_CUDA(cudaStreamSynchronize(st)); // the host tables above go out of scope
    return CN_OK;
}

// One iteration's soft families with the strand families on a side stream and, once the edges
// are applied, the cloth bends on another, joined back before the stream goes on (each particle's
// families still in the order of physics_solver.cpp:915-1019).
void launchSoftBranches(cn_solver *sv, float dt, cudaStream_t st)
{
    const cn::Scene &s = sv->s;
    const cn::Config &c = sv->cfg;
    const uint32_t strandFams = (1u << cn::kFamSegments) | (1u << cn::kFamJoints) | (1u << cn::kFamDistances);
    uint32_t mainFams = cn::kAllFamilies;
    if (sv->branchStrands) {
        cudaStreamWaitEvent(sv->side[1], sv->fork, 0);
        cn::launchSoftFamilies(s, dt, c, sv->side[1], strandFams);
        cudaEventRecord(sv->joinStrands, sv->side[1]);
        mainFams &= ~strandFams;
    }
    if (sv->branchBends) {
        cn::launchSoftFamilies(s, dt, c, st, mainFams & (1u << cn::kFamEdges));
        cudaEventRecord(sv->afterEdges, st);
        cudaStreamWaitEvent(sv->side[2], sv->afterEdges, 0);
        cn::launchSoftFamilies(s, dt, c, sv->side[2], 1u << cn::kFamBends);
        cudaEventRecord(sv->joinBends, sv->side[2]);
        cn::launchSoftFamilies(s, dt, c, st, mainFams & ~((1u << cn::kFamEdges) | (1u << cn::kFamBends)));
        cudaStreamWaitEvent(st, sv->joinBends, 0);
    } else {
        cn::launchSoftFamilies(s, dt, c, st, mainFams);
    }
    if (sv->branchStrands) cudaStreamWaitEvent(st, sv->joinStrands, 0);
}

void enqueueFrame(cn_solver *sv, float frameDt, cudaStream_t st)
{
    const cn::Scene &s = sv->s;
    const float dt = frameDt / float(sv->substeps);
    const cn::Config &c = sv->cfg;
    const uint32_t N = s.N;
    for (uint32_t sub = 0; sub < sv->substeps; ++sub) {
        probe(sv, "rigid_predict", st, [&] { cn::launchRigidPredict(s, dt, c.gravity[0], c.gravity[1], c.gravity[2], st); });
        if (s.colBvh) probe(sv, "collider_bvh", st, [&] { cn::launchColliderBvh(s, sv->rigidScratch, st); });
        if (sv->rigidRigid)
            probe(sv, "rigid_broadphase_contacts", st, [&] { cn::launchRigidBroadphaseAndContacts(s, c, sv->rigidScratch, st); });
        probe(sv, "predict_keys", st, [&] { cn::launchPredictAndKeys(s, dt, c, st); });
        if (sv->hasBroadphase && (sv->hasFluid || sv->ppPossible || sv->forceBroadphase)) {
            probe(sv, "radix_sort", st, [&] {
                cn::radixSortPairs(s.keysA, s.valsA, s.keysB, s.valsB, N, sv->sortScratch, &s.meta_->waitTimeouts, st);
            });
            probe(sv, "cell_setup", st, [&] { cn::launchCellSetup(s, sv->scanScratch, sv->sortScratch, st); });
        }
        if (sv->ppPossible)
            probe(sv, "particle_candidates", st, [&] { cn::launchParticleCandidates(s, sv->scanScratch, sv->scanScratchBytes, st); });
        if (sv->rigidPossible || sv->proxyContacts)
            probe(sv, "rigid_candidates", st, [&] { cn::launchRigidCandidates(s, sv->scanScratch, sv->scanScratchBytes, st); });
        // generateProxyRigidContacts (physics_solver.cpp:722-727)
        if (sv->proxyContacts) cn::launchProxyRigidContacts(s, st);
        // initRigidContactVelocities (physics_solver.cpp:736-743)
        if (sv->rigidRigid) cn::launchRigidVelocityInit(s, c, sv->rigidScratch, st);
        // clearSoftConstraintState (physics_clear_soft_constraint_state.cs.hlsl:14-54)
        if (s.E) cudaMemsetAsync(s.edgeLambda, 0, sizeof(float) * s.E, st);
        if (s.Bn + s.D) cudaMemsetAsync(s.bendLambda, 0, sizeof(float) * (s.Bn + s.D), st);
        if (s.T) cudaMemsetAsync(s.tetLambda, 0, sizeof(float) * s.T, st);
        if (s.SD) cudaMemsetAsync(s.distLambda, 0, sizeof(float) * s.SD, st);
        if (s.S) cudaMemsetAsync(s.segLambda, 0, sizeof(float4) * s.S, st);
        if (s.J) cudaMemsetAsync(s.jointLambda, 0, sizeof(float4) * s.J, st);
        if (s.fluidMaxDelta) cudaMemsetAsync(s.fluidMaxDelta, 0, sizeof(uint32_t) * 64, st);
        if (s.hasDynamic) { // clearRigidCorrections (physics_rigid_clear_corrections.cs.hlsl)
            cudaMemsetAsync(s.bodyTransCorr, 0, sizeof(float4) * s.B, st);
            cudaMemsetAsync(s.bodyRotCorr, 0, sizeof(float4) * s.B, st);
            cudaMemsetAsync(s.bodyLinVelCorr, 0, sizeof(float4) * s.B, st);
            cudaMemsetAsync(s.bodyAngVelCorr, 0, sizeof(float4) * s.B, st);
        }
        if (sv->ppPossible) {
            cudaMemsetAsync(s.posCorr, 0, sizeof(float4) * N, st);
            cudaMemsetAsync(s.velCorr, 0, sizeof(float4) * N, st);
        }
        const bool hasSoftInternal = N > 0 && (s.E || s.Bn || s.D || s.T || s.S || s.J || s.SD);
        if (sv->fused) {
            // every iteration of the substep in one cluster kernel (soft families, then the
            // particle-rigid contacts of the iteration)
            const uint32_t softIt = hasSoftInternal ? sv->softIt : 0u;
            const uint32_t contactIt = sv->rigidPossible ? sv->contactIt : 0u;
            probe(sv, "fused_iterations", st, [&] {
                cn::launchFusedIterations(s, c, dt, sv->plan, std::max(softIt, contactIt), softIt, contactIt,
                                          sv->rigidPossible, sv->fusedShape, st);
            });
        }
        for (uint32_t it = 0; it < (sv->fused ? 0u : sv->maxIt); ++it) {
            const bool runFluid = sv->hasFluid && it < sv->fluidIt;
            const bool runSoft = hasSoftInternal && it < sv->softIt;
            const bool runPP = sv->ppPossible && it < sv->contactIt;
            const bool runRigid = sv->rigidPossible && it < sv->contactIt;
            const bool runRigidRigid = sv->rigidRigid && it < sv->rrIt;
            if (!runFluid && !runSoft && !runPP && !runRigid && !runRigidRigid) break; // remaining iterations are empty
            // fork: the fluid chain and the branched soft families leave the frame's stream here
            const bool fluidBranch = sv->branchFluid && runFluid && runSoft;
            const bool softBranches = runSoft && (sv->branchStrands || sv->branchBends);
            if (fluidBranch || softBranches) cudaEventRecord(sv->fork, st);
            const cudaStream_t fst = fluidBranch ? sv->side[0] : st;
            if (fluidBranch) cudaStreamWaitEvent(fst, sv->fork, 0);
            if (runFluid) {
                if (it == 0 || cn::fluidGatherEachIteration(s))
                    probe(sv, "fluid_gather", fst, [&] { cn::launchFluidGather(s, it, fst); });
                // the first iteration of a substep also records the superset lists when they are on
                probe(sv, (it == 0 && s.sup && !sv->walkCells) ? "fluid_neighbors_superset" : "fluid_neighbors_density", fst,
                      [&] { cn::launchFluidNeighborsDensity(s, c, it, sv->walkCells, fst); });
                probe(sv, "fluid_delta_apply_clamp", fst,
                      [&] { cn::launchFluidDeltaApplyClamp(s, it, dt, c, sv->writeFluidDebug, fst); });
            }
            if (fluidBranch) cudaEventRecord(sv->joinFluid, fst);
            // without particle-particle contacts (and without soft branches) the rigid contacts run
            // in the tet gather's pass; their records are read after the iterations, so only the last
            // contact pass writes them
            cn::Scene si = s;
            si.storeRigidContacts = it + 1 == sv->contactIt ? 1u : 0u;
            bool contactsDone = false;
            if (runSoft && softBranches)
                probe(sv, "soft_constraints", st, [&] { launchSoftBranches(sv, dt, st); });
            else if (runSoft)
                probe(sv, "soft_constraints", st, [&] {
                    contactsDone = cn::launchSoftIteration(si, dt, c, sv->plan, st, runRigid && !runPP);
                });
            if (fluidBranch) cudaStreamWaitEvent(st, sv->joinFluid, 0);
            if ((runPP || runRigid) && !contactsDone)
                probe(sv, "contacts", st, [&] { cn::launchContacts(si, c, runPP, runRigid, st); });
            // finalRigidContactDepenetration (physics_solver.cpp:1111-1117)
            if (runRigidRigid) probe(sv, "rigid_depenetration", st, [&] { cn::launchRigidDepenetration(s, c, st); });
            // applyRigidCorrections (physics_solver.cpp:1170-1177); with only static and kinematic
            // bodies the summed corrections are zero and the pass is left out
            if ((runRigid || runRigidRigid) && s.hasDynamic) {
                cn::launchApplyRigidCorrections(s, c, st);
                cn::launchSyncRigidProxies(s, st); // syncRigidProxyParticles (physics_solver.cpp:1178-1186)
            }
        }
        // updateRigidVelocities (physics_solver.cpp:1241-1246): for static and kinematic bodies it
        // restates what the rigid predict wrote, so it runs for scenes with dynamic bodies
        if (s.hasDynamic) cn::launchUpdateRigidVelocities(s, dt, st);
        const float4 *fluidDelta = sv->hasFluid ? ((sv->fluidIt & 1u) ? s.Db : s.Da) : nullptr;
        probe(sv, "update_velocities", st, [&] { cn::launchUpdateVelocities(s, dt, fluidDelta, st); });
        if (sv->hasFluid) probe(sv, "fluid_boundary_velocities", st, [&] { cn::launchFluidBoundaryVelocities(s, dt, c, st); });
        // post-update neighbour rebuild and vorticity confinement (physics_solver.cpp:1262-1285)
        if (sv->hasFluid && (sv->postUpdateNeighbors || sv->vorticity)) cn::launchFluidNeighborsOnly(s, st);
        if (sv->vorticity) probe(sv, "fluid_vorticity", st, [&] { cn::launchFluidVorticity(s, dt, st); });
        if (sv->ppPossible && sv->contactIt)
            probe(sv, "contact_velocities", st, [&] { cn::launchParticleContactVelocities(s, sv->contactIt, c, st); });
        if (sv->rigidPossible && sv->contactIt) {
            if (s.hasDynamic)
                probe(sv, "contact_velocities", st,
                      [&] { cn::launchRigidContactVelocitiesDynamic(s, sv->contactIt, c, st); });
            else
                probe(sv, "contact_velocities", st, [&] { cn::launchRigidContactVelocities(s, sv->contactIt, c, st); });
        }
        // solveRigidContactVelocities (physics_solver.cpp:1345-1354)
        if (sv->rigidRigid)
            probe(sv, "rigid_contact_velocities", st, [&] {
                cn::launchRigidContactVelocitySolve(s, c, std::max(sv->rrIt, sv->jointIt), sv->rrIt, st);
            });
        cn::launchCopyPredictedRigid(s, st);
    }
    // physics_solver.cpp:1310-1337 (after the last substep: see launchSurfaceRender)
    if (s.surfV || s.surfT || s.surfS) probe(sv, "surface_render", st, [&] { cn::launchSurfaceRender(s, st); });
}

cn_status runFrames(cn_solver *sv, float frameDt, uint32_t frames, cudaStream_t st)
{
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_step: no world synced");
    if (sv->s.N == 0 && sv->s.B == 0) return CN_OK;
    CN_CUDA(cudaSetDevice(sv->device));
    if (sv->graphExec == nullptr || sv->graphDt != frameDt) {
        releaseGraph(sv);
        cudaStream_t cap = sv->ownStream;
        CN_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        enqueueFrame(sv, frameDt, cap);
        const cudaError_t endErr = cudaStreamEndCapture(cap, &sv->graph);
        if (endErr != cudaSuccess) {
            cudaGetLastError();
            return setError(CN_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(endErr));
        }
        CN_CUDA(cudaGraphInstantiate(&sv->graphExec, sv->graph, 0));
        sv->graphDt = frameDt;
        size_t count = 0;
        cudaGraphGetNodes(sv->graph, nullptr, &count);
        std::vector<cudaGraphNode_t> nodes(count);
        cudaGraphGetNodes(sv->graph, nodes.data(), &count);
        uint32_t kernels = 0;
        for (cudaGraphNode_t n : nodes) {
            cudaGraphNodeType type;
            if (cudaGraphNodeGetType(n, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
        }
        sv->graphNodes = uint32_t(count);
        sv->graphKernelNodes = kernels;
    }
    for (uint32_t f = 0; f < frames; ++f) CN_CUDA(cudaGraphLaunch(sv->graphExec, st));
    CN_CUDA(cudaGetLastError());
    return CN_OK;
}

} // namespace

extern "C" {

CN_API const char *cn_last_error(void) { return cn::g_lastError.c_str(); }
CN_API const char *cn_version(void) { return "cressim-neo-b200 0.1.0 (sm_100a)"; }

CN_API void cn_solver_desc_defaults(cn_solver_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->gravity[1] = -9.81f;
    d->substeps = 1;
    d->default_iterations = 20;
    d->contact = cn_contact_settings{1.0e-3f, 4.0f, 0.95f, 0.05f, 0.5f, 2.0f, 0.0f, 1.0e-5f};
    d->rigid = cn_rigid_settings{0.25f, 0.90f, 0.10f, 1.0f, 0.01f, 0.10f, 0.8f, 0.5f};
    d->joints = cn_joint_settings{0.95f, 0.7f, 0.05f, 0.02f, 0.12f, 1.0e-5f, 5.0e-5f, 1.0e-5f};
    d->soft.internal_relaxation = 0.2f;
    d->fluid.constraint_relaxation = 0.7f;
    d->fluid.position_relaxation = 1.0f;
    d->fluid.boundary_density_scale = 0.12f;
    d->fluid.boundary_delta_scale = 0.08f;
    d->fluid.max_under_density_ratio = 0.0f;
    d->enable_blocking_readback = 1u;
    d->max_fluid_neighborhood = 128u;
    d->particle_rigid_pairs_per_particle = 8u;
}

CN_API cn_status cn_solver_create(const cn_solver_desc *desc, int device, cn_solver **out)
{
    if (!desc || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_create: null argument");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return setError(CN_ERR_NO_DEVICE, "cn_solver_create: no CUDA device");
    }
    if (device < 0 || device >= count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_create: bad device");
    CN_CUDA(cudaSetDevice(device));
    cn_solver *sv = new cn_solver();
    sv->desc = *desc;
    sv->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&sv->ownStream, cudaStreamNonBlocking);
    for (cudaStream_t &x : sv->side)
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
    for (cudaEvent_t *ev : {&sv->fork, &sv->joinFluid, &sv->joinStrands, &sv->afterEdges, &sv->joinBends})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cn_solver_destroy(sv);
        return setError(CN_ERR_CUDA, std::string("cn_solver_create: ") + cudaGetErrorString(e));
    }
    *out = sv;
    return CN_OK;
}

CN_API void cn_solver_destroy(cn_solver *sv)
{
    if (!sv) return;
    cudaSetDevice(sv->device);
    if (sv->ownStream) cudaStreamSynchronize(sv->ownStream);
    releaseBuffers(sv);
    if (sv->ownStream) cudaStreamDestroy(sv->ownStream);
    for (cudaStream_t x : sv->side)
        if (x) cudaStreamDestroy(x);
    for (cudaEvent_t ev : {sv->fork, sv->joinFluid, sv->joinStrands, sv->afterEdges, sv->joinBends})
        if (ev) cudaEventDestroy(ev);
    delete sv;
}

// FNV-1a over the particle (segment) indices of every constraint record: the incidence tables,
// gather slots and colourings of the synced world are built from them.
static uint64_t topologyHash(const cn_world_soa &w)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint32_t v) {
        for (int k = 0; k < 4; ++k) {
            h ^= (v >> (8 * k)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    for (uint32_t c = 0; c < w.edge_count; ++c) { mix(w.edges[c].particle_a); mix(w.edges[c].particle_b); }
    for (uint32_t c = 0; c < w.bend_count; ++c) { mix(w.bends[c].particle0); mix(w.bends[c].particle1); mix(w.bends[c].particle2); }
    for (uint32_t c = 0; c < w.dihedral_count; ++c) {
        const cn_cloth_dihedral &d = w.dihedrals[c];
        mix(d.edge_particle0); mix(d.edge_particle1); mix(d.opposite_particle0); mix(d.opposite_particle1);
    }
    for (uint32_t c = 0; c < w.tet_count; ++c)
        for (int k = 0; k < 4; ++k) mix(w.tets[c].particle_indices[k]);
    for (uint32_t c = 0; c < w.strand_segment_count; ++c) { mix(w.strand_segments[c].particle_a); mix(w.strand_segments[c].particle_b); }
    for (uint32_t c = 0; c < w.strand_joint_count; ++c) { mix(w.strand_joints[c].segment_a); mix(w.strand_joints[c].segment_b); }
    for (uint32_t c = 0; c < w.strand_distance_count; ++c) { mix(w.strand_distances[c].particle_a); mix(w.strand_distances[c].particle_b); }
    return h;
}

// The structural choices that the particle attributes make at sync: particle-particle contacts
// possible (a self-colliding solid particle or several solid groups), vorticity confinement, and the
// fluid kernels built with the cohesion / surface-tension terms.
static uint32_t attributeStructure(const cn_world_soa &w)
{
    bool anyFluid = false, anySelf = false;
    uint32_t firstGroup = 0xffffffffu, groups = 0;
    for (uint32_t i = 0; i < w.particle_count; ++i) {
        if (w.kinds[i] == CN_PARTICLE_FLUID) {
            anyFluid = true;
            continue;
        }
        const uint32_t ph = w.metadata[4 * i + 1];
        if (ph & CN_PHASE_SELF_COLLIDE) anySelf = true;
        const uint32_t g = ph & CN_PHASE_GROUP_MASK;
        if (groups == 0) {
            firstGroup = g;
            groups = 1;
        } else if (g != firstGroup) {
            groups = 2;
        }
    }
    uint32_t bits = (anySelf || groups > 1) ? 1u : 0u;
    for (uint32_t m = 0; m < w.fluid_material_count; ++m) {
        const cn_fluid_material &fm = w.fluid_materials[m];
        if (anyFluid && fm.vorticity_confinement > 1.0e-6f) bits |= 2u;
        if (fm.cohesion > 0.0f || fm.surface_tension > 1.0e-6f) bits |= 4u;
    }
    return bits;
}

// The edges and tets in colour order, for the coloured schedules.
static cudaError_t uploadColourOrdered(cn_solver *sv, const cn_world_soa &w, cudaStream_t st)
{
    const cn::Scene &s = sv->s;
    if (s.edgesC) {
        const std::vector<uint32_t> &order = sv->colouring[cn::kFamEdges].order;
        sv->edgesC.resize(order.size());
        for (size_t i = 0; i < order.size(); ++i) sv->edgesC[i] = cn::packEdge(w.edges[order[i]]);
        const cudaError_t e = cudaMemcpyAsync(const_cast<cn::PackedEdge *>(s.edgesC), sv->edgesC.data(),
                                              sizeof(cn::PackedEdge) * order.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
    }
    if (s.tetsC) {
        const std::vector<uint32_t> &order = sv->colouring[cn::kFamTets].order;
        sv->tetsC.resize(order.size());
        for (size_t i = 0; i < order.size(); ++i) sv->tetsC[i] = w.tets[order[i]];
        const cudaError_t e = cudaMemcpyAsync(const_cast<cn_soft_tet *>(s.tetsC), sv->tetsC.data(),
                                              sizeof(cn_soft_tet) * order.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

CN_API cn_status cn_solver_sync_world(cn_solver *sv, const cn_world_soa *w)
{
    if (!sv || !w) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_sync_world: null argument");
    const uint32_t N = w->particle_count;
    if (N && (!w->positions_inv_mass || !w->velocities || !w->radii || !w->kinds || !w->metadata ||
              !w->material_indices || !w->fluid_material_indices || !w->owner_types || !w->owner_indices ||
              !w->adjacency_offsets || !w->adjacency_counts))
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_sync_world: missing particle array");
    if (N > (1u << 29)) return setError(CN_ERR_CAPACITY, "cn_solver_sync_world: more than 2^29 particles");
    if (sv->desc.max_fluid_neighborhood > 1024u)
        return setError(CN_ERR_INVALID_ARGUMENT, "max_fluid_neighborhood above 1024");
    if (sv->desc.particle_rigid_pairs_per_particle > 256u ||
        uint64_t(N) * cn::rigidPairsPerParticle(sv->desc) >= (uint64_t(1) << 32))
        return setError(CN_ERR_INVALID_ARGUMENT, "particle_rigid_pairs_per_particle above 256 or 2^32 pairs");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaStreamSynchronize(sv->ownStream));
    releaseBuffers(sv);

    // Structural flags (physics_solver.cpp:472-496), plus which contact families can have pairs.
    const cn_solver_desc &d = sv->desc;
    sv->substeps = std::max<uint32_t>(d.substeps, 1u);
    const uint32_t defIt = std::max<uint32_t>(d.default_iterations, 1u);
    sv->fluidIt = cn::resolveIter(d.fluid_iterations, defIt);
    sv->softIt = cn::resolveIter(d.soft_internal_iterations, defIt);
    sv->contactIt = cn::resolveIter(d.soft_contact_iterations, defIt);
    const uint32_t jointIt = cn::resolveIter(d.rigid_joint_iterations, defIt);
    const uint32_t rrIt = cn::resolveIter(d.rigid_rigid_contact_iterations, defIt);
    sv->jointIt = jointIt;
    sv->rrIt = rrIt;
    sv->maxIt = std::max(std::max(std::max(sv->fluidIt, sv->softIt), sv->contactIt), std::max(jointIt, rrIt));
    bool anyFluid = false, anySolid = false, anySelf = false;
    std::vector<uint32_t> solidGroups;
    for (uint32_t i = 0; i < N; ++i) {
        if (w->kinds[i] == CN_PARTICLE_FLUID) anyFluid = true;
        else {
            anySolid = true;
            const uint32_t ph = w->metadata[4 * i + 1];
            if (ph & CN_PHASE_SELF_COLLIDE) anySelf = true;
            const uint32_t g = ph & CN_PHASE_GROUP_MASK;
            if (solidGroups.size() < 2 && std::find(solidGroups.begin(), solidGroups.end(), g) == solidGroups.end())
                solidGroups.push_back(g);
        }
    }
    bool anyDynamic = false;
    for (uint32_t b = 0; b < w->rigid_body_count; ++b)
        if (w->body_types[b] == CN_BODY_DYNAMIC) anyDynamic = true;
    sv->vorticity = false;
    for (uint32_t m = 0; m < w->fluid_material_count; ++m)
        if (w->fluid_materials[m].vorticity_confinement > 1.0e-6f) sv->vorticity = anyFluid;
    sv->hasFluid = anyFluid;
    sv->hasDynamic = anyDynamic;
    if (anyFluid && (uint64_t(N) * std::max<uint32_t>(d.max_fluid_neighborhood, 160u) >= (uint64_t(1) << 32)))
        return setError(CN_ERR_UNSUPPORTED, "fluid scene too large for 32-bit neighbour list offsets");
    const bool contactWork = sv->contactIt > 0;
    sv->ppPossible = contactWork && N > 1 && anySolid && (anyFluid || anySelf || solidGroups.size() > 1);
    // particle-rigid contacts: solid particles against every body, fluid particles against dynamic
    // ones (physics_particle_count_particle_rigid_candidates.cs.hlsl:113-151)
    sv->rigidPossible = contactWork && N > 0 && w->collider_count > 0 && (anySolid || (anyFluid && anyDynamic));
    // Fluid x then also moves between the fluid iterations (contacts with dynamic bodies, or with
    // other particles): the positions are gathered every iteration, not double-buffered.
    sv->fluidXMoves = sv->ppPossible || (anyFluid && anyDynamic && sv->rigidPossible);
    sv->hasBroadphase = N > 0 && ((contactWork && N > 1) || anyFluid || w->collider_count > 0);

    // Fluid filter groups: dense ids of the distinct (environment, layer, mask) triples.
    std::vector<uint32_t> fluidGroup(N, 0u);
    {
        std::vector<std::array<uint32_t, 3>> groups;
        for (uint32_t i = 0; i < N; ++i) {
            if (w->kinds[i] != CN_PARTICLE_FLUID) continue;
            const std::array<uint32_t, 3> key{w->metadata[4 * i], w->metadata[4 * i + 2], w->metadata[4 * i + 3]};
            auto it = std::find(groups.begin(), groups.end(), key);
            if (it == groups.end()) {
                if (groups.size() >= 0xffffu)
                    return setError(CN_ERR_UNSUPPORTED, "more than 65535 fluid (environment, layer, mask) groups");
                groups.push_back(key);
                it = groups.end() - 1;
            }
            fluidGroup[i] = uint32_t(it - groups.begin());
        }
        for (uint32_t m = 0; m < N; ++m)
            if (w->kinds[m] == CN_PARTICLE_FLUID && w->fluid_material_indices[m] > 0x7fffu)
                return setError(CN_ERR_UNSUPPORTED, "fluid material index above 32767");
    }

    {
        const std::string err = checkSurfaceRender(*w);
        if (!err.empty()) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_sync_world: " + err);
    }

    // Collider query order: moving (kinematic, dynamic) colliders, then static, ascending index.
    // Rigid proxy particles: PhysicsWorld packs them before every other particle
    // (physics_world.cpp:4931-5023), which the passes rely on.
    uint32_t nProxy = 0;
    while (nProxy < N && w->owner_types[nProxy] == CN_OWNER_RIGID_BODY) ++nProxy;
    for (uint32_t i = nProxy; i < N; ++i)
        if (w->owner_types[i] == CN_OWNER_RIGID_BODY)
            return setError(CN_ERR_UNSUPPORTED, "rigid proxy particles must lead the particle order");
    if (nProxy) {
        if (!w->rigid_proxy_local_positions || !w->body_proxy_contact_materials)
            return setError(CN_ERR_INVALID_ARGUMENT, "rigid proxy particles without local positions or materials");
        for (uint32_t i = 0; i < nProxy; ++i)
            if (w->owner_indices[i] >= w->rigid_body_count)
                return setError(CN_ERR_INVALID_ARGUMENT, "rigid proxy particle of a body out of range");
    }
    sv->nProxy = nProxy;

    std::vector<uint32_t> order;
    const uint32_t moving = cn::colliderQueryOrder(*w, order);
    sv->queryOrder = order;
    // useInitialRigidContactSolve (physics_solver.cpp:512-514) for scenes where a body can move:
    // collider pairs of the rigid broadphase, or proxy particles against colliders
    sv->rigidRigid = anyDynamic && rrIt > 0 && ((order.size() >= 2 && moving > 0) || (nProxy > 0 && w->collider_count > 0));
    sv->proxyContacts = sv->rigidRigid && nProxy > 0 && w->collider_count > 0;
    if (sv->rigidRigid && uint64_t(w->rigid_body_count) * w->rigid_body_count >= 0xffffffffull)
        return setError(CN_ERR_UNSUPPORTED, "more than 65535 rigid bodies in a scene with dynamic bodies");
    // More colliders than the boundary mask holds: per-particle candidate lists over a collider LBVH
    sv->fluidBoundaryLists = anyFluid && order.size() > cn::kMaxBoundaryColliders;

    // Incidence tables.
    const cn::Incidence edgeI = cn::buildIncidence(N, w->edge_count, 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? w->edges[c].particle_a : w->edges[c].particle_b;
    });
    const uint32_t nb = w->bend_count;
    const cn::Incidence bendI = cn::buildIncidence(N, nb + w->dihedral_count, 4, [&](uint32_t c, uint32_t k) -> uint32_t {
        if (c < nb) {
            if (k == 3) return 0xffffffffu;
            const cn_soft_bend &b = w->bends[c];
            return k == 0 ? b.particle0 : (k == 1 ? b.particle1 : b.particle2);
        }
        const cn_cloth_dihedral &h = w->dihedrals[c - nb];
        const uint32_t p[4] = {h.edge_particle0, h.edge_particle1, h.opposite_particle0, h.opposite_particle1};
        return p[k];
    });
    const cn::Incidence tetI = cn::buildIncidence(N, w->tet_count, 4, [&](uint32_t c, uint32_t k) {
        return w->tets[c].particle_indices[k];
    });
    const cn::Incidence segI = cn::buildIncidence(N, w->strand_segment_count, 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? w->strand_segments[c].particle_a : w->strand_segments[c].particle_b;
    });
    const uint32_t S = w->strand_segment_count;
    const cn::Incidence jointI = cn::buildIncidence(S, w->strand_joint_count, 2, [&](uint32_t c, uint32_t k) -> uint32_t {
        const cn_strand_joint &j = w->strand_joints[c];
        if (j.segment_a >= S || j.segment_b >= S) return 0xffffffffu;
        return k == 0 ? j.segment_a : j.segment_b;
    });

    // XPBD schedule: the coloured schedules colour every family (elements: particles; segments
    // for the joints, whose corrections move orientations)
    const uint32_t schedule = d.soft.xpbd_schedule;
    if (schedule > CN_XPBD_COLOUR_GAUSS_SEIDEL)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_sync_world: unknown soft.xpbd_schedule");
    if (d.soft.fused_iterations > CN_FUSED_ON)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_sync_world: unknown soft.fused_iterations");
    sv->plan = cn::XpbdPlan{};
    sv->plan.schedule = schedule;
    for (cn::Colouring &col : sv->colouring) col = cn::Colouring{};
    if (schedule != CN_XPBD_GATHER) {
        // the gather applies strand distance records through the strand-segment incidence; the
        // colour schedules apply them to the distance's own particles, the same ones when each
        // distance constraint spans its segment (as cn_world authors strands)
        if (w->strand_distance_count &&
            (w->strand_distance_count != w->strand_segment_count ||
             !std::equal(w->strand_distances, w->strand_distances + w->strand_distance_count, w->strand_segments,
                         [](const cn_strand_distance &dc, const cn_strand_segment &sg) {
                             return dc.particle_a == sg.particle_a && dc.particle_b == sg.particle_b;
                         })))
            return setError(CN_ERR_UNSUPPORTED,
                            "coloured XPBD schedules need each strand distance constraint on its segment's particles");
        sv->colouring[cn::kFamEdges] = cn::colourGreedy(N, w->edge_count, 2, [&](uint32_t c, uint32_t k) {
            return k == 0 ? w->edges[c].particle_a : w->edges[c].particle_b;
        });
        sv->colouring[cn::kFamSegments] = cn::colourGreedy(N, S, 2, [&](uint32_t c, uint32_t k) {
            return k == 0 ? w->strand_segments[c].particle_a : w->strand_segments[c].particle_b;
        });
        sv->colouring[cn::kFamBends] = cn::colourGreedy(N, nb + w->dihedral_count, 4, [&](uint32_t c, uint32_t k) -> uint32_t {
            if (c < nb) {
                if (k == 3) return 0xffffffffu;
                const cn_soft_bend &b = w->bends[c];
                return k == 0 ? b.particle0 : (k == 1 ? b.particle1 : b.particle2);
            }
            const cn_cloth_dihedral &h = w->dihedrals[c - nb];
            const uint32_t p[4] = {h.edge_particle0, h.edge_particle1, h.opposite_particle0, h.opposite_particle1};
            return p[k];
        });
        sv->colouring[cn::kFamJoints] = cn::colourGreedy(S, w->strand_joint_count, 2, [&](uint32_t c, uint32_t k) {
            return k == 0 ? w->strand_joints[c].segment_a : w->strand_joints[c].segment_b;
        });
        sv->colouring[cn::kFamDistances] = cn::colourGreedy(N, w->strand_distance_count, 2, [&](uint32_t c, uint32_t k) {
            return k == 0 ? w->strand_distances[c].particle_a : w->strand_distances[c].particle_b;
        });
        sv->colouring[cn::kFamTets] = cn::colourGreedy(N, w->tet_count, 4, [&](uint32_t c, uint32_t k) {
            return w->tets[c].particle_indices[k];
        });
        for (uint32_t f = 0; f < cn::kFamilies; ++f) {
            sv->plan.colours[f] = sv->colouring[f].colours();
            sv->plan.hostStarts[f] = sv->colouring[f].starts.empty() ? nullptr : sv->colouring[f].starts.data();
        }
    }

    cn::Arena a;
    a.reset(nullptr);
    layout(sv, a, *w, edgeI, bendI, tetI, segI, jointI);
    sv->arenaBytes = a.size();
    {
        const cudaError_t e = cudaMalloc(&sv->arena, sv->arenaBytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            sv->arena = nullptr;
            return setError(CN_ERR_OUT_OF_MEMORY, "cn_solver_sync_world: cannot allocate " +
                                                      std::to_string(sv->arenaBytes) + " bytes");
        }
    }
    a.reset(static_cast<uint8_t *>(sv->arena));
    layout(sv, a, *w, edgeI, bendI, tetI, segI, jointI);
    cn::Scene &s = sv->s;
    s.cellSize = w->particle_grid_cell_size;
    s.fluidExtras = 0;
    for (uint32_t m = 0; m < w->fluid_material_count; ++m)
        if (w->fluid_materials[m].cohesion > 0.0f || w->fluid_materials[m].surface_tension > 1.0e-6f) s.fluidExtras = 1;
    s.solidEnd = 0;
    for (uint32_t i = N; i > 0; --i)
        if (w->kinds[i - 1] != CN_PARTICLE_FLUID) {
            s.solidEnd = i;
            break;
        }
    s.colQueryCount = uint32_t(order.size());
    s.activeMovingCount = moving;
    cudaStream_t st = sv->ownStream;
    CN_CUDA(cudaMemsetAsync(sv->arena, 0, sv->arenaBytes, st));
    CN_CUDA(up(s.x, w->positions_inv_mass, size_t(N) * 1, st));
    CN_CUDA(up(s.v, w->velocities, N, st));
    {
        std::vector<float4> xp(N);
        for (uint32_t i = 0; i < N; ++i)
            xp[i] = make_float4(w->positions_inv_mass[4 * i], w->positions_inv_mass[4 * i + 1],
                                w->positions_inv_mass[4 * i + 2], 0.0f);
        CN_CUDA(up(s.xprev, xp.data(), N, st));
        CN_CUDA(cudaStreamSynchronize(st));
    }
    CN_CUDA(up(s.radii, w->radii, N, st));
    CN_CUDA(up(s.kinds, w->kinds, N, st));
    CN_CUDA(up(s.meta, w->metadata, N, st));
    CN_CUDA(up(s.matIdx, w->material_indices, N, st));
    CN_CUDA(up(s.fluidMatIdx, w->fluid_material_indices, N, st));
    CN_CUDA(up(s.ownerTypes, w->owner_types, N, st));
    CN_CUDA(up(s.ownerIdx, w->owner_indices, N, st));
    CN_CUDA(up(s.fluidGroup, fluidGroup.data(), N, st));
    CN_CUDA(up(s.adjOff, w->adjacency_offsets, N, st));
    CN_CUDA(up(s.adjCnt, w->adjacency_counts, N, st));
    CN_CUDA(up(s.adjIdx, w->adjacency_indices, w->adjacency_index_count, st));
    CN_CUDA(up(s.contactMaterials, w->contact_materials, w->contact_material_count, st));
    CN_CUDA(up(s.fluidMaterials, w->fluid_materials, w->fluid_material_count, st));
    CN_CUDA(up(s.edges, w->edges, s.E, st));
    CN_CUDA(up(s.bends, w->bends, s.Bn, st));
    CN_CUDA(up(s.dihedrals, w->dihedrals, s.D, st));
    CN_CUDA(up(s.tets, w->tets, s.T, st));
    CN_CUDA(up(s.segs, w->strand_segments, s.S, st));
    CN_CUDA(up(s.joints, w->strand_joints, s.J, st));
    CN_CUDA(up(s.dists, w->strand_distances, s.SD, st));
    CN_CUDA(up(s.segOrient, w->strand_segment_orientations, s.S, st));
    s.edgeWin = cn::incidenceWindow(edgeI);
    s.bendWin = cn::incidenceWindow(bendI);
    s.tetWin = cn::incidenceWindow(tetI);
    s.segWin = cn::incidenceWindow(segI);
    CN_CUDA(up(s.edgeRanges, edgeI.ranges.data(), edgeI.ranges.size(), st));
    CN_CUDA(up(s.bendRanges, bendI.ranges.data(), bendI.ranges.size(), st));
    CN_CUDA(up(s.tetRanges, tetI.ranges.data(), tetI.ranges.size(), st));
    CN_CUDA(up(s.segRanges, segI.ranges.data(), segI.ranges.size(), st));
    CN_CUDA(up(s.segInc, segI.inc.data(), segI.inc.size(), st));
    CN_CUDA(up(s.segJointRanges, jointI.ranges.data(), jointI.ranges.size(), st));
    CN_CUDA(up(s.segJointInc, jointI.inc.data(), jointI.inc.size(), st));
    CN_CUDA(up(const_cast<uint32_t *>(s.edgeDst), edgeI.dst.data(), edgeI.dst.size(), st));
    CN_CUDA(up(const_cast<uint32_t *>(s.bendDst), bendI.dst.data(), bendI.dst.size(), st));
    CN_CUDA(up(const_cast<uint32_t *>(s.tetDst), tetI.dst.data(), tetI.dst.size(), st));
    {
        // strand distance c's records go to segment c's gather slots (none past the segments)
        std::vector<uint32_t> distDst(size_t(s.SD) * 2, 0xffffffffu);
        for (uint32_t c = 0; c < std::min(s.SD, s.S); ++c) {
            distDst[2 * size_t(c)] = segI.dst[2 * size_t(c)];
            distDst[2 * size_t(c) + 1] = segI.dst[2 * size_t(c) + 1];
        }
        CN_CUDA(up(const_cast<uint32_t *>(s.distDst), distDst.data(), distDst.size(), st));
    }
    for (uint32_t f = 0; f < cn::kFamilies; ++f) {
        const cn::Colouring &col = sv->colouring[f];
        if (!col.colours()) continue;
        CN_CUDA(up(const_cast<uint32_t *>(s.colOrder[f]), col.order.data(), col.order.size(), st));
        CN_CUDA(up(const_cast<uint32_t *>(sv->plan.devStarts[f]), col.starts.data(), col.starts.size(), st));
    }
    CN_CUDA(uploadColourOrdered(sv, *w, st));
    CN_CUDA(up(s.bodyPos, w->body_positions_inv_mass, s.B, st));
    CN_CUDA(up(s.bodyRot, w->body_orientations, s.B, st));
    CN_CUDA(up(s.bodyLin, w->body_linear_velocities, s.B, st));
    CN_CUDA(up(s.bodyAng, w->body_angular_velocities, s.B, st));
    CN_CUDA(up(s.bodyScale, w->body_scales, s.B, st));
    CN_CUDA(up(s.bodyInvInertia, w->body_inverse_inertia, s.B, st));
    CN_CUDA(up(s.bodyType, w->body_types, s.B, st));
    CN_CUDA(up(s.bodyKinPos, w->body_kinematic_target_positions, s.B, st));
    CN_CUDA(up(s.bodyKinRot, w->body_kinematic_target_orientations, s.B, st));
    CN_CUDA(up(s.bodyKinFlags, w->body_kinematic_target_flags, s.B, st));
    CN_CUDA(up(s.bodyColRanges, w->body_collider_ranges, s.B, st));
    CN_CUDA(up(s.bodyColIdx, w->body_collider_indices, w->body_collider_index_count, st));
    CN_CUDA(up(s.colGeo, w->collider_geometry, s.C, st));
    CN_CUDA(up(s.colBp, w->collider_broadphase, s.C, st));
    CN_CUDA(up(s.colMat, w->collider_materials, s.C, st));
    CN_CUDA(up(s.colQueryOrder, order.data(), order.size(), st));
    if (nProxy) {
        CN_CUDA(up(s.proxyLocal, w->rigid_proxy_local_positions, nProxy, st));
        CN_CUDA(up(s.bodyProxyMat, w->body_proxy_contact_materials, s.B, st));
    }
    {
        const cn_status r = uploadSurfaceRender(sv, *w, st);
        if (r != CN_OK) return r;
    }
    CN_CUDA(cudaStreamSynchronize(st));

    sv->cfg = cn::configFromDesc(d);
    // Fused iterations: soft bodies against static and kinematic colliders only, each phase at
    // most kFusedRounds passes of the cluster's threads over its elements
    sv->fused = false;
    if (d.soft.fused_iterations == CN_FUSED_ON && N > 0 && !sv->hasFluid && !sv->ppPossible && !sv->hasDynamic &&
        !sv->rigidRigid && nProxy == 0 && (s.E || s.Bn || s.D || s.T || s.S || s.J || s.SD)) {
        if (!sv->fusedShapeQueried) {
            sv->fusedShape = cn::fusedIterationsShape();
            sv->fusedShapeQueried = true;
        }
        constexpr uint32_t kFusedRounds = 4u;
        const uint64_t cap = uint64_t(sv->fusedShape.ctas) * sv->fusedShape.threads * kFusedRounds;
        const uint64_t most = std::max({uint64_t(N), uint64_t(s.E), uint64_t(s.Bn) + s.D, uint64_t(s.T), uint64_t(s.S),
                                        uint64_t(s.J), uint64_t(s.SD)});
        sv->fused = cap > 0 && most <= cap;
    }
    // Concurrent branches (per-phase gather schedule): the strand families beside the others, the
    // cloth bends beside the tets once the edges are applied, and the fluid chain beside the soft
    // families, whenever the particle windows they write are disjoint.
    {
        auto disjoint = [](uint2 a, uint2 b) { return a.y <= a.x || b.y <= b.x || a.y <= b.x || b.y <= a.x; };
        const bool perPhase = sv->plan.schedule == CN_XPBD_GATHER && !sv->fused;
        const bool strands = s.S || s.J || s.SD, others = s.E || s.Bn || s.D || s.T;
        sv->branchStrands = perPhase && strands && others && disjoint(s.segWin, s.edgeWin) &&
                            disjoint(s.segWin, s.bendWin) && disjoint(s.segWin, s.tetWin);
        sv->branchBends = perPhase && (s.Bn || s.D) && s.T && disjoint(s.bendWin, s.tetWin) &&
                          (!strands || sv->branchStrands);
        uint2 fluidWin = make_uint2(N, 0u);
        for (uint32_t i = 0; i < N; ++i)
            if (w->kinds[i] == CN_PARTICLE_FLUID) {
                fluidWin.x = std::min(fluidWin.x, i);
                fluidWin.y = i + 1;
            }
        sv->branchFluid = perPhase && sv->hasFluid && (strands || others) && disjoint(fluidWin, s.edgeWin) &&
                          disjoint(fluidWin, s.bendWin) && disjoint(fluidWin, s.tetWin) &&
                          disjoint(fluidWin, s.segWin);
    }
    sv->hostX = w->positions_inv_mass;
    sv->hostV = w->velocities;
    sv->contactMaterialCapacity = w->contact_material_count;
    sv->fluidMaterialCapacity = w->fluid_material_count;
    sv->surfIdxCapacity = w->surface_render ? w->surface_render->vertex_triangle_index_count : 0u;
    sv->cellRangeCapacity = cn::nextPow2(std::max<uint32_t>(N * 2u, 1u));
    sv->topologyHash = topologyHash(*w);
    sv->attributeStructure = attributeStructure(*w);
    sv->bodyTypes.assign(w->body_types, w->body_types + w->rigid_body_count);
    sv->synced = true;
    ++sv->bindingGeneration;
    cn::clearError();
    return CN_OK;
}

CN_API cn_status cn_solver_step(cn_solver *sv, float frame_dt, void *stream)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_step: null solver");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : sv->ownStream;
    const cn_status r = runFrames(sv, frame_dt, 1, st);
    if (r != CN_OK) return r;
    if (sv->desc.enable_blocking_readback && sv->hostX) {
        CN_CUDA(cudaMemcpyAsync(sv->hostX, sv->s.x, sizeof(float4) * sv->s.N, cudaMemcpyDeviceToHost, st));
        CN_CUDA(cudaMemcpyAsync(sv->hostV, sv->s.v, sizeof(float4) * sv->s.N, cudaMemcpyDeviceToHost, st));
        CN_CUDA(cudaStreamSynchronize(st));
    }
    return CN_OK;
}

CN_API cn_status cn_solver_step_many(cn_solver *sv, float frame_dt, uint32_t steps, void *stream)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_step_many: null solver");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : sv->ownStream;
    return runFrames(sv, frame_dt, steps, st);
}

CN_API cn_status cn_solver_validate_meta(cn_solver *sv, cn_meta *out)
{
    if (!sv || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_validate_meta: null argument");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_validate_meta: no world synced");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    cn::DeviceMeta m{};
    CN_CUDA(cudaMemcpy(&m, sv->s.meta_, sizeof(m), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->particle_rigid_candidate_count = m.rigidPairCount;
    out->required_particle_rigid_candidate_count = m.requiredRigidPairs;
    out->particle_rigid_candidate_overflow = m.requiredRigidPairs > sv->s.rigidPairCapacity ? 1u : 0u;
    out->particle_particle_candidate_count = m.particlePairCount;
    out->required_particle_particle_candidate_count = m.requiredParticlePairs;
    out->particle_particle_candidate_overflow = m.requiredParticlePairs > sv->s.particlePairCapacity ? 1u : 0u;
    out->fluid_boundary_candidate_overflow = m.boundaryMaskOverflow;
    out->active_particle_contact_count = m.activeParticleContactsLast;
    out->fluid_neighbor_truncations = m.neighborTruncations;
    out->device_wait_timeouts = m.waitTimeouts;
    out->rigid_rigid_candidate_count = m.rigidRigidPairCount;
    out->required_rigid_rigid_candidate_count = m.requiredRigidRigidPairs;
    out->rigid_rigid_candidate_overflow = m.requiredRigidRigidPairs > sv->s.rrCapacity ? 1u : 0u;
    out->proxy_rigid_contact_count = m.proxyContactSlots;
    out->required_proxy_rigid_contact_count = m.requiredProxyContacts;
    out->proxy_rigid_contact_overflow = m.requiredProxyContacts > sv->s.proxyCapacity ? 1u : 0u;
    if (m.waitTimeouts) return setError(CN_ERR_DEVICE_TIMEOUT, "a bounded device wait gave up (sort look-back)");
    if (out->particle_rigid_candidate_overflow || out->particle_particle_candidate_overflow ||
        out->fluid_boundary_candidate_overflow || out->rigid_rigid_candidate_overflow ||
        out->proxy_rigid_contact_overflow)
        return setError(CN_ERR_CAPACITY, "candidate buffer overflow");
    return CN_OK;
}

CN_API cn_status cn_solver_set_gravity(cn_solver *sv, float x, float y, float z)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_set_gravity: null solver");
    sv->desc.gravity[0] = x; sv->desc.gravity[1] = y; sv->desc.gravity[2] = z;
    sv->cfg.gravity[0] = x; sv->cfg.gravity[1] = y; sv->cfg.gravity[2] = z;
    releaseGraph(sv);
    return CN_OK;
}

CN_API cn_status cn_solver_set_kinematic_target(cn_solver *sv, uint32_t body, const float position[3],
                                                const float orientation[4])
{
    if (!sv || !position || !orientation) return setError(CN_ERR_INVALID_ARGUMENT, "set_kinematic_target: null argument");
    if (!sv->synced || body >= sv->s.B) return setError(CN_ERR_INVALID_ARGUMENT, "set_kinematic_target: bad body");
    const float4 p = make_float4(position[0], position[1], position[2], 0.0f);
    const float4 q = make_float4(orientation[0], orientation[1], orientation[2], orientation[3]);
    const uint32_t flag = 1u;
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaMemcpyAsync(sv->s.bodyKinPos + body, &p, sizeof(p), cudaMemcpyHostToDevice, sv->ownStream));
    CN_CUDA(cudaMemcpyAsync(sv->s.bodyKinRot + body, &q, sizeof(q), cudaMemcpyHostToDevice, sv->ownStream));
    CN_CUDA(cudaMemcpyAsync(sv->s.bodyKinFlags + body, &flag, sizeof(flag), cudaMemcpyHostToDevice, sv->ownStream));
    CN_CUDA(cudaStreamSynchronize(sv->ownStream));
    return CN_OK;
}

CN_API cn_status cn_solver_scene_view(cn_solver *sv, cn_scene_view *v)
{
    if (!sv || !v) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_scene_view: null argument");
    std::memset(v, 0, sizeof(*v));
    const cn::Scene &s = sv->s;
    v->positions_inv_mass = s.x; v->previous_positions = s.xprev; v->velocities = s.v;
    v->radii = const_cast<float *>(s.radii); v->kinds = const_cast<uint32_t *>(s.kinds);
    v->edges = const_cast<cn_soft_edge *>(s.edges); v->bends = const_cast<cn_soft_bend *>(s.bends);
    v->dihedrals = const_cast<cn_cloth_dihedral *>(s.dihedrals); v->tets = const_cast<cn_soft_tet *>(s.tets);
    v->strand_segments = const_cast<cn_strand_segment *>(s.segs);
    v->strand_joints = const_cast<cn_strand_joint *>(s.joints);
    v->strand_distances = const_cast<cn_strand_distance *>(s.dists);
    v->strand_segment_states = s.segOrient;
    v->particle_count = s.N; v->edge_count = s.E; v->bend_count = s.Bn; v->dihedral_count = s.D;
    v->tet_count = s.T; v->strand_segment_count = s.S; v->strand_joint_count = s.J; v->strand_distance_count = s.SD;
    v->binding_generation = sv->bindingGeneration;
    v->device = sv->device;
    return CN_OK;
}

CN_API cn_status cn_solver_surface_render_view(cn_solver *sv, cn_surface_render_view *v)
{
    if (!sv || !v) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_surface_render_view: null argument");
    std::memset(v, 0, sizeof(*v));
    const cn::Scene &s = sv->s;
    v->render_positions = s.surfPos;
    v->render_normals = s.surfNrm;
    v->triangle_normals = s.surfTriN;
    v->chunk_aabbs = s.surfChunkAabb;
    v->world_aabbs = s.surfWorldAabb;
    v->vertex_count = s.surfV;
    v->triangle_count = s.surfT;
    v->chunk_count = s.surfChunks;
    v->surface_count = s.surfS;
    v->binding_generation = sv->bindingGeneration;
    return CN_OK;
}

CN_API cn_status cn_solver_read_surface_render(cn_solver *sv, float *positions, float *normals, float *world_aabbs)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_read_surface_render: null solver");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_read_surface_render: no world synced");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    const cn::Scene &s = sv->s;
    if (positions && s.surfV) CN_CUDA(cudaMemcpy(positions, s.surfPos, sizeof(float4) * s.surfV, cudaMemcpyDeviceToHost));
    if (normals && s.surfV) CN_CUDA(cudaMemcpy(normals, s.surfNrm, sizeof(float4) * s.surfV, cudaMemcpyDeviceToHost));
    if (world_aabbs && s.surfS)
        CN_CUDA(cudaMemcpy(world_aabbs, s.surfWorldAabb, sizeof(float4) * 2 * s.surfS, cudaMemcpyDeviceToHost));
    return CN_OK;
}

namespace {
struct DlHolder {
    cn_dl_managed_tensor t{};
    int64_t shape[2] = {0, 0};
};
void dlDelete(cn_dl_managed_tensor *self)
{
    delete static_cast<DlHolder *>(self->manager_ctx);
}
} // namespace

CN_API cn_status cn_solver_export_dlpack(cn_solver *sv, const char *buffer, cn_dl_managed_tensor **out)
{
    if (!sv || !buffer || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_export_dlpack: null argument");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_export_dlpack: no world synced");
    const cn::Scene &s = sv->s;
    const std::string name(buffer);
    void *data = nullptr;
    int64_t rows = s.N, cols = 4;
    uint8_t code = 2; // float
    if (name == "positions_inv_mass") data = s.x;
    else if (name == "previous_positions") data = s.xprev;
    else if (name == "velocities") data = s.v;
    else if (name == "radii") { data = const_cast<float *>(s.radii); cols = 1; }
    else if (name == "kinds") { data = const_cast<uint32_t *>(s.kinds); cols = 1; code = 1; }
    else if (name == "strand_segment_states") { data = s.segOrient; rows = s.S; }
    else if (name == "render_positions") { data = s.surfPos; rows = s.surfV; }
    else if (name == "render_normals") { data = s.surfNrm; rows = s.surfV; }
    else if (name == "surface_world_aabbs") { data = s.surfWorldAabb; rows = s.surfS; cols = 8; }
    else return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_export_dlpack: unknown buffer '" + name + "'");
    auto *h = new DlHolder();
    h->shape[0] = rows;
    h->shape[1] = cols;
    cn_dl_tensor &t = h->t.dl_tensor;
    t.data = data;
    t.device_type = 2; // kDLCUDA
    t.device_id = sv->device;
    t.ndim = cols == 1 ? 1 : 2;
    t.dtype_code = code;
    t.dtype_bits = 32;
    t.dtype_lanes = 1;
    t.shape = h->shape;
    t.strides = nullptr;
    t.byte_offset = 0;
    h->t.manager_ctx = h;
    h->t.deleter = dlDelete;
    *out = &h->t;
    return CN_OK;
}

CN_API cn_status cn_solver_update_world(cn_solver *sv, const cn_world_soa *w, uint32_t flags)
{
    if (!sv || !w) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: null argument");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_update_world: no world synced");
    const cn::Scene &s = sv->s;
    if (w->particle_count != s.N || w->edge_count != s.E || w->bend_count != s.Bn || w->dihedral_count != s.D ||
        w->tet_count != s.T || w->strand_segment_count != s.S || w->strand_joint_count != s.J ||
        w->strand_distance_count != s.SD || w->rigid_body_count != s.B || w->collider_count != s.C)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: element counts changed; use cn_solver_sync_world");
    if (flags & CN_SYNC_SURFACE_RENDER) {
        const cn_surface_render_data *sr = w->surface_render;
        uint32_t chunks = 0;
        for (uint32_t k = 0; sr && k < sr->surface_count; ++k) chunks += (sr->surface_particle_ranges[2 * k + 1] + 63u) / 64u;
        if ((sr ? sr->vertex_count : 0u) != s.surfV || (sr ? sr->triangle_count : 0u) != s.surfT ||
            (sr ? sr->surface_count : 0u) != s.surfS || chunks != s.surfChunks)
            return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: surface render counts changed; use cn_solver_sync_world");
        const std::string err = checkSurfaceRender(*w);
        if (!err.empty()) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: " + err);
    }
    // everything that is refused is refused before anything is uploaded
    if (flags & CN_SYNC_PARTICLE_ATTRIBUTES) {
        if (w->contact_material_count > std::max<uint32_t>(sv->contactMaterialCapacity, 1u) ||
            w->fluid_material_count > std::max<uint32_t>(sv->fluidMaterialCapacity, 1u))
            return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: more materials than synced; use cn_solver_sync_world");
        if (s.nProxy && !w->rigid_proxy_local_positions)
            return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: rigid proxy local positions missing");
    }
    if ((flags & CN_SYNC_RIGID_BODIES) && s.nProxy && !w->body_proxy_contact_materials)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: proxy contact materials missing");
    if ((flags & CN_SYNC_SURFACE_RENDER) && w->surface_render &&
        w->surface_render->vertex_triangle_index_count > sv->surfIdxCapacity)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: more incident-triangle indices than synced");
    if ((flags & CN_SYNC_PARTICLE_ATTRIBUTES) && attributeStructure(*w) != sv->attributeStructure)
        return setError(CN_ERR_INVALID_ARGUMENT,
                        "cn_solver_update_world: the attributes change which contact or fluid terms run "
                        "(self-collision, solid groups, vorticity, cohesion / surface tension); use cn_solver_sync_world");
    if (flags & CN_SYNC_COLLIDERS) {
        std::vector<uint32_t> order;
        cn::colliderQueryOrder(*w, order);
        if (order != sv->queryOrder)
            return setError(CN_ERR_INVALID_ARGUMENT,
                            "cn_solver_update_world: colliders enabled, disabled or moved to other bodies; use cn_solver_sync_world");
    }
    if ((flags & CN_SYNC_CONSTRAINTS) && topologyHash(*w) != sv->topologyHash)
        return setError(CN_ERR_INVALID_ARGUMENT,
                        "cn_solver_update_world: constraint particle indices changed; use cn_solver_sync_world");
    if ((flags & CN_SYNC_RIGID_BODIES) && (s.B && (!w->body_types ||
                                                   !std::equal(sv->bodyTypes.begin(), sv->bodyTypes.end(), w->body_types))))
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_update_world: body types changed; use cn_solver_sync_world");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize()); // frames in flight read these buffers
    cudaStream_t st = sv->ownStream;
    const uint32_t N = s.N;
    if (flags & CN_SYNC_PARTICLE_STATE) {
        CN_CUDA(up(s.x, w->positions_inv_mass, N, st));
        CN_CUDA(up(s.v, w->velocities, N, st));
    }
    if (flags & CN_SYNC_PARTICLE_ATTRIBUTES) {
        CN_CUDA(up(s.radii, w->radii, N, st));
        CN_CUDA(up(s.meta, w->metadata, N, st));
        CN_CUDA(up(s.matIdx, w->material_indices, N, st));
        CN_CUDA(up(s.fluidMatIdx, w->fluid_material_indices, N, st));
        CN_CUDA(up(s.contactMaterials, w->contact_materials, w->contact_material_count, st));
        CN_CUDA(up(s.fluidMaterials, w->fluid_materials, w->fluid_material_count, st));
        if (s.nProxy) CN_CUDA(up(s.proxyLocal, w->rigid_proxy_local_positions, s.nProxy, st));
    }
    if (flags & CN_SYNC_CONSTRAINTS) {
        // records only: incidence tables depend on the particle indices, which must not change
        CN_CUDA(up(s.edges, w->edges, s.E, st));
        CN_CUDA(up(s.bends, w->bends, s.Bn, st));
        CN_CUDA(up(s.dihedrals, w->dihedrals, s.D, st));
        CN_CUDA(up(s.tets, w->tets, s.T, st));
        CN_CUDA(up(s.segs, w->strand_segments, s.S, st));
        CN_CUDA(up(s.joints, w->strand_joints, s.J, st));
        CN_CUDA(up(s.dists, w->strand_distances, s.SD, st));
        CN_CUDA(uploadColourOrdered(sv, *w, st)); // the coloured schedules' copies of the records
    }
    if (flags & CN_SYNC_RIGID_BODIES) {
        CN_CUDA(up(s.bodyPos, w->body_positions_inv_mass, s.B, st));
        CN_CUDA(up(s.bodyRot, w->body_orientations, s.B, st));
        CN_CUDA(up(s.bodyLin, w->body_linear_velocities, s.B, st));
        CN_CUDA(up(s.bodyAng, w->body_angular_velocities, s.B, st));
        CN_CUDA(up(s.bodyScale, w->body_scales, s.B, st));
        CN_CUDA(up(s.bodyInvInertia, w->body_inverse_inertia, s.B, st));
        CN_CUDA(up(s.bodyKinPos, w->body_kinematic_target_positions, s.B, st));
        CN_CUDA(up(s.bodyKinRot, w->body_kinematic_target_orientations, s.B, st));
        CN_CUDA(up(s.bodyKinFlags, w->body_kinematic_target_flags, s.B, st));
        if (s.nProxy) CN_CUDA(up(s.bodyProxyMat, w->body_proxy_contact_materials, s.B, st));
    }
    if (flags & CN_SYNC_COLLIDERS) {
        CN_CUDA(up(s.colGeo, w->collider_geometry, s.C, st));
        CN_CUDA(up(s.colBp, w->collider_broadphase, s.C, st));
        CN_CUDA(up(s.colMat, w->collider_materials, s.C, st));
    }
    if (flags & CN_SYNC_SURFACE_RENDER) {
        // the index-array length may differ at equal vertex counts (checked above to fit the synced one)
        const cn_status r = uploadSurfaceRender(sv, *w, st);
        if (r != CN_OK) return r;
    }
    CN_CUDA(cudaStreamSynchronize(st));
    return CN_OK;
}

CN_API cn_status cn_solver_read_particles(cn_solver *sv, float *x, float *v, float *xprev, uint32_t count)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_read_particles: null solver");
    if (count > sv->s.N) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_read_particles: count > particles");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    if (x) CN_CUDA(cudaMemcpy(x, sv->s.x, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    if (v) CN_CUDA(cudaMemcpy(v, sv->s.v, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    if (xprev) CN_CUDA(cudaMemcpy(xprev, sv->s.xprev, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    return CN_OK;
}

CN_API cn_status cn_solver_write_particles(cn_solver *sv, const float *x, const float *v, uint32_t count)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_write_particles: null solver");
    if (count > sv->s.N) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_write_particles: count > particles");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize()); // frames stepped on a caller stream may still be running
    if (x) CN_CUDA(cudaMemcpyAsync(sv->s.x, x, sizeof(float4) * count, cudaMemcpyHostToDevice, sv->ownStream));
    if (v) CN_CUDA(cudaMemcpyAsync(sv->s.v, v, sizeof(float4) * count, cudaMemcpyHostToDevice, sv->ownStream));
    CN_CUDA(cudaStreamSynchronize(sv->ownStream));
    return CN_OK;
}

CN_API cn_status cn_solver_read_rigid_bodies(cn_solver *sv, float *pos, float *rot, float *lin, float *ang,
                                             uint32_t count)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_read_rigid_bodies: null solver");
    if (count > sv->s.B) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_read_rigid_bodies: count > bodies");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    const size_t bytes = sizeof(float4) * count;
    if (!count) return CN_OK;
    if (pos) CN_CUDA(cudaMemcpy(pos, sv->s.bodyPos, bytes, cudaMemcpyDeviceToHost));
    if (rot) CN_CUDA(cudaMemcpy(rot, sv->s.bodyRot, bytes, cudaMemcpyDeviceToHost));
    if (lin) CN_CUDA(cudaMemcpy(lin, sv->s.bodyLin, bytes, cudaMemcpyDeviceToHost));
    if (ang) CN_CUDA(cudaMemcpy(ang, sv->s.bodyAng, bytes, cudaMemcpyDeviceToHost));
    return CN_OK;
}

CN_API cn_status cn_solver_step_io(cn_solver *sv, float frame_dt, const float *x_in, const float *v_in, float *x_out,
                                   float *v_out, void *stream)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_step_io: null solver");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_step_io: no world synced");
    CN_CUDA(cudaSetDevice(sv->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : sv->ownStream;
    const size_t bytes = sizeof(float4) * sv->s.N;
    if (x_in) CN_CUDA(cudaMemcpyAsync(sv->s.x, x_in, bytes, cudaMemcpyHostToDevice, st));
    if (v_in) CN_CUDA(cudaMemcpyAsync(sv->s.v, v_in, bytes, cudaMemcpyHostToDevice, st));
    const cn_status r = runFrames(sv, frame_dt, 1, st);
    if (r != CN_OK) return r;
    if (x_out) CN_CUDA(cudaMemcpyAsync(x_out, sv->s.x, bytes, cudaMemcpyDeviceToHost, st));
    if (v_out) CN_CUDA(cudaMemcpyAsync(v_out, sv->s.v, bytes, cudaMemcpyDeviceToHost, st));
    CN_CUDA(cudaStreamSynchronize(st));
    return CN_OK;
}

CN_API cn_status cn_solver_read_strand_orientations(cn_solver *sv, float *q, uint32_t count)
{
    if (!sv || !q) return setError(CN_ERR_INVALID_ARGUMENT, "read_strand_orientations: null argument");
    if (count > sv->s.S) return setError(CN_ERR_INVALID_ARGUMENT, "read_strand_orientations: count > segments");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    if (count) CN_CUDA(cudaMemcpy(q, sv->s.segOrient, sizeof(float4) * count, cudaMemcpyDeviceToHost));
    return CN_OK;
}

CN_API cn_status cn_solver_set_debug(cn_solver *sv, uint32_t flags)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_set_debug: null solver");
    sv->writeFluidDebug = (flags & 1u) != 0u;
    sv->postUpdateNeighbors = (flags & 2u) != 0u;
    sv->forceBroadphase = (flags & 4u) != 0u;
    sv->walkCells = (flags & 8u) != 0u;
    releaseGraph(sv);
    return CN_OK;
}

CN_API cn_status cn_solver_set_timing(cn_solver *sv, uint32_t enable)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_set_timing: null solver");
    sv->timing = enable != 0u;
    releaseGraph(sv);
    return CN_OK;
}

CN_API cn_status cn_solver_kernel_times(cn_solver *sv, cn_kernel_time *out, uint32_t capacity, uint32_t *count)
{
    if (!sv || !count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_kernel_times: null argument");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    std::vector<cn_kernel_time> acc;
    for (const auto &p : sv->probes) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.begin, p.end) != cudaSuccess) {
            cudaGetLastError();
            return setError(CN_ERR_CUDA, "cn_solver_kernel_times: events not recorded yet");
        }
        auto it = std::find_if(acc.begin(), acc.end(), [&](const cn_kernel_time &k) { return std::strcmp(k.name, p.name) == 0; });
        if (it == acc.end()) {
            cn_kernel_time k{};
            std::strncpy(k.name, p.name, sizeof(k.name) - 1);
            acc.push_back(k);
            it = acc.end() - 1;
        }
        it->milliseconds += ms;
        it->launches += 1;
    }
    *count = uint32_t(acc.size());
    if (out)
        for (uint32_t i = 0; i < capacity && i < acc.size(); ++i) out[i] = acc[i];
    return CN_OK;
}

CN_API cn_status cn_solver_graph_stats(cn_solver *sv, uint32_t *kernel_nodes, uint32_t *nodes)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_graph_stats: null solver");
    if (kernel_nodes) *kernel_nodes = sv->graphKernelNodes;
    if (nodes) *nodes = sv->graphNodes;
    return CN_OK;
}

CN_API cn_status cn_solver_schedule_info(cn_solver *sv, cn_schedule_info *out)
{
    if (!sv || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_schedule_info: null argument");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_schedule_info: no world synced");
    std::memset(out, 0, sizeof(*out));
    out->xpbd_schedule = sv->plan.schedule;
    out->fused_iterations = sv->fused ? 1u : 0u;
    out->cluster_ctas = sv->fused ? sv->fusedShape.ctas : 0u;
    out->threads_per_cta = sv->fused ? sv->fusedShape.threads : 0u;
    for (uint32_t f = 0; f < cn::kFamilies; ++f) out->colours[f] = sv->plan.colours[f];
    out->branches = (sv->branchFluid ? 1u : 0u) | (sv->branchStrands ? 2u : 0u) | (sv->branchBends ? 4u : 0u);
    return CN_OK;
}

CN_API cn_status cn_colour_constraints(const uint32_t *elements, uint32_t constraint_count, uint32_t per_constraint,
                                       uint32_t element_count, uint32_t *order, uint32_t *colour_starts,
                                       uint32_t colour_capacity, uint32_t *colours)
{
    if (!colours || (constraint_count && (!elements || !order || !colour_starts || per_constraint == 0)))
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_colour_constraints: null argument");
    const cn::Colouring col = cn::colourGreedy(element_count, constraint_count, per_constraint, [&](uint32_t c, uint32_t k) {
        return elements[size_t(c) * per_constraint + k];
    });
    *colours = col.colours();
    if (constraint_count) std::copy(col.order.begin(), col.order.end(), order);
    const size_t keep = std::min<size_t>(col.starts.size(), size_t(colour_capacity) + 1u);
    if (colour_starts) std::copy(col.starts.begin(), col.starts.begin() + keep, colour_starts);
    if (col.colours() > colour_capacity)
        return setError(CN_ERR_CAPACITY, "cn_colour_constraints: more colours than colour_capacity");
    cn::clearError();
    return CN_OK;
}

CN_API cn_status cn_solver_debug_read(cn_solver *sv, cn_debug_buffer which, void *dst, size_t cap, size_t *outBytes)
{
    if (!sv) return setError(CN_ERR_INVALID_ARGUMENT, "cn_solver_debug_read: null solver");
    if (!sv->synced) return setError(CN_ERR_NOT_INITIALIZED, "cn_solver_debug_read: no world synced");
    CN_CUDA(cudaSetDevice(sv->device));
    CN_CUDA(cudaDeviceSynchronize());
    const cn::Scene &s = sv->s;
    const uint32_t N = s.N;
    std::vector<uint8_t> buf;
    auto fetch = [&](const void *src, size_t bytes, std::vector<uint8_t> &into) -> cudaError_t {
        into.resize(bytes);
        if (!bytes || !src) return cudaSuccess;
        return cudaMemcpy(into.data(), src, bytes, cudaMemcpyDeviceToHost);
    };
    std::vector<uint8_t> rankB, valsB;
    const bool needRank = which == CN_DEBUG_FLUID_NEIGHBOR_COUNTS || which == CN_DEBUG_FLUID_NEIGHBORS ||
                          which == CN_DEBUG_FLUID_SUPERSET_COUNTS ||
                          which == CN_DEBUG_FLUID_CONSTRAINTS || which == CN_DEBUG_FLUID_DELTA;
    if (needRank) {
        if (!s.rank || !s.hasFluid) return setError(CN_ERR_INVALID_ARGUMENT, "debug_read: scene has no fluid");
        CN_CUDA(fetch(s.rank, sizeof(uint32_t) * N, rankB));
        CN_CUDA(fetch(s.cvals, sizeof(uint32_t) * N, valsB));
    }
    const uint32_t *rank = reinterpret_cast<const uint32_t *>(rankB.data());
    const uint32_t *vals = reinterpret_cast<const uint32_t *>(valsB.data());
    std::vector<uint8_t> kindsB;
    switch (which) {
    case CN_DEBUG_CELL_ENTRIES:
        if (!s.entries) return setError(CN_ERR_INVALID_ARGUMENT, "debug_read: no broadphase");
        CN_CUDA(fetch(s.entries, sizeof(int4) * N, buf));
        break;
    case CN_DEBUG_SORTED_KEYS: {
        if (!s.keysA) return setError(CN_ERR_INVALID_ARGUMENT, "debug_read: no broadphase");
        std::vector<uint8_t> k, v;
        CN_CUDA(fetch(s.keysA, sizeof(uint32_t) * N, k));
        CN_CUDA(fetch(s.valsA, sizeof(uint32_t) * N, v));
        buf.resize(size_t(N) * 8);
        uint32_t *o = reinterpret_cast<uint32_t *>(buf.data());
        for (uint32_t i = 0; i < N; ++i) {
            o[2 * i] = reinterpret_cast<uint32_t *>(k.data())[i];
            o[2 * i + 1] = reinterpret_cast<uint32_t *>(v.data())[i];
        }
        break;
    }
    case CN_DEBUG_CELL_RANGES: {
        if (!s.keysA) return setError(CN_ERR_INVALID_ARGUMENT, "debug_read: no broadphase");
        const uint32_t capR = sv->cellRangeCapacity;
        uint4 *tmp = nullptr;
        CN_CUDA(cudaMalloc(&tmp, sizeof(uint4) * capR));
        std::vector<uint4> init(capR, make_uint4(0xffffffffu, 0u, 0u, 0u));
        cudaMemcpy(tmp, init.data(), sizeof(uint4) * capR, cudaMemcpyHostToDevice);
        cn::launchExportCellRanges(s, tmp, capR, sv->scanScratch, sv->scanScratchBytes, sv->ownStream);
        cudaStreamSynchronize(sv->ownStream);
        const cudaError_t e = fetch(tmp, sizeof(uint4) * capR, buf);
        cudaFree(tmp);
        CN_CUDA(e);
        break;
    }
    case CN_DEBUG_FLUID_NEIGHBOR_COUNTS: {
        std::vector<uint8_t> c;
        CN_CUDA(fetch(s.nbrCount, sizeof(uint32_t) * N, c));
        CN_CUDA(fetch(s.kinds, sizeof(uint32_t) * N, kindsB));
        buf.assign(size_t(N) * 4, 0);
        uint32_t *o = reinterpret_cast<uint32_t *>(buf.data());
        const uint32_t *cc = reinterpret_cast<const uint32_t *>(c.data());
        const uint32_t *kk = reinterpret_cast<const uint32_t *>(kindsB.data());
        for (uint32_t p = 0; p < N; ++p) o[p] = kk[p] == CN_PARTICLE_FLUID ? cc[rank[p]] : 0u;
        break;
    }
    case CN_DEBUG_FLUID_SUPERSET_COUNTS: {
        buf.assign(size_t(N) * 4, 0);
        if (!s.supCount) break;
        std::vector<uint8_t> c;
        CN_CUDA(fetch(s.supCount, sizeof(uint32_t) * N, c));
        CN_CUDA(fetch(s.kinds, sizeof(uint32_t) * N, kindsB));
        uint32_t *o = reinterpret_cast<uint32_t *>(buf.data());
        const uint32_t *cc = reinterpret_cast<const uint32_t *>(c.data());
        const uint32_t *kk = reinterpret_cast<const uint32_t *>(kindsB.data());
        for (uint32_t p = 0; p < N; ++p) o[p] = kk[p] == CN_PARTICLE_FLUID ? cc[rank[p]] : 0u;
        break;
    }
    case CN_DEBUG_FLUID_NEIGHBORS: {
        std::vector<uint8_t> c, l;
        CN_CUDA(fetch(s.nbrCount, sizeof(uint32_t) * N, c));
        CN_CUDA(fetch(s.nbr, sizeof(uint32_t) * size_t(N) * s.maxNbr, l));
        CN_CUDA(fetch(s.kinds, sizeof(uint32_t) * N, kindsB));
        buf.assign(size_t(N) * s.maxNbr * 4, 0);
        uint32_t *o = reinterpret_cast<uint32_t *>(buf.data());
        const uint32_t *cc = reinterpret_cast<const uint32_t *>(c.data());
        const uint32_t *ll = reinterpret_cast<const uint32_t *>(l.data());
        const uint32_t *kk = reinterpret_cast<const uint32_t *>(kindsB.data());
        for (uint32_t p = 0; p < N; ++p) {
            if (kk[p] != CN_PARTICLE_FLUID) continue;
            const uint32_t r = rank[p];
            const uint32_t n = std::min(cc[r], s.maxNbr);
            const bool inter = cn::fluidListsInterleaved();
            for (uint32_t k = 0; k < n; ++k)
                o[size_t(p) * s.maxNbr + k] = vals[ll[inter ? size_t(k) * N + r : size_t(r) * s.maxNbr + k]];
        }
        break;
    }
    case CN_DEBUG_FLUID_CONSTRAINTS:
    case CN_DEBUG_FLUID_DELTA: {
        std::vector<uint8_t> c;
        CN_CUDA(fetch(which == CN_DEBUG_FLUID_CONSTRAINTS ? s.Cs : s.Dx, sizeof(float4) * N, c));
        buf.assign(size_t(N) * 16, 0);
        float4 *o = reinterpret_cast<float4 *>(buf.data());
        const float4 *cc = reinterpret_cast<const float4 *>(c.data());
        for (uint32_t p = 0; p < N; ++p) o[p] = cc[rank[p]];
        break;
    }
    case CN_DEBUG_RIGID_CONTACTS: {
        if (!s.rigidContacts) { buf.clear(); break; }
        std::vector<uint8_t> c, cnt, off;
        CN_CUDA(fetch(s.rigidContacts, sizeof(cn::RigidContact) * s.rigidPairCapacity, c));
        CN_CUDA(fetch(s.candCount, sizeof(uint32_t) * N, cnt));
        CN_CUDA(fetch(s.candOffset, sizeof(uint32_t) * N, off));
        const cn::RigidContact *cc = reinterpret_cast<const cn::RigidContact *>(c.data());
        const uint32_t *pc = reinterpret_cast<const uint32_t *>(cnt.data());
        const uint32_t *po = reinterpret_cast<const uint32_t *>(off.data());
        // particle-major pair order; the pairs of a particle sit at its offset in either layout
        // (scanned offsets or fixed slots)
        for (uint32_t p = 0; p < N; ++p)
            for (uint32_t k = 0; k < pc[p]; ++k) {
                const uint32_t pi = po[p] + k;
                if (pi >= s.rigidPairCapacity) break; // dropped by a full pair buffer
                if (!cc[pi].active) continue;
                const uint8_t *b = reinterpret_cast<const uint8_t *>(&cc[pi]);
                buf.insert(buf.end(), b, b + sizeof(cn::RigidContact));
            }
        break;
    }
    default:
        return setError(CN_ERR_INVALID_ARGUMENT, "debug_read: unknown buffer");
    }
    if (outBytes) *outBytes = buf.size();
    if (dst && cap) std::memcpy(dst, buf.data(), std::min(cap, buf.size()));
    return CN_OK;
}

} // extern "C"
