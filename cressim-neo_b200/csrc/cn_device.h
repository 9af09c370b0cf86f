// cn_device.h -- device-resident scene layout and kernel launchers of the particle substep.
//
// One Scene value holds every device pointer and count the kernels need; it is passed by
// value to each launch so a captured CUDA graph replays with stable arguments.  Per-particle
// state stays in the reference's particle order (float4 x/invMass, x_prev, v: the layout
// PhysicsGpuSceneView exports, include/physics/physics_gpu_scene_view.h:114-169).  The fluid
// solve runs in cell order: after the broadphase sort every fluid quantity of an iteration
// (position, accumulated delta, density constraint, neighbour list) lives at the particle's
// sorted slot, so neighbour gathers touch contiguous cell runs.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cn_physics.h"

namespace cn {

// GpuParticleRigidContact (physics_particle_types.hlsli:74-83), 64 B.
struct RigidContact {
    uint32_t particle, body, collider, active;
    float4 normalPenetration;
    float4 rigidLocalPoint;
    float4 material;
};
// GpuParticleContact (physics_particle_types.hlsli:85-92), 48 B.
struct ParticleContact {
    uint32_t a, b, active, reserved;
    float4 normalPenetration;
    float4 material;
};

// Device counters (mirrors GpuParticleNeighborMeta plus this build's own counters).
struct DeviceMeta {
    uint32_t rigidPairCount;          // min(required, capacity)
    uint32_t requiredRigidPairs;
    uint32_t particlePairCount;
    uint32_t requiredParticlePairs;
    uint32_t activeRigidContacts;
    uint32_t activeParticleContacts;
    uint32_t boundaryMaskOverflow;
    uint32_t neighborTruncations;
    uint32_t waitTimeouts;
    uint32_t rigidRigidPairCount;     // min(required, capacity) collider pairs of the rigid broadphase
    uint32_t requiredRigidRigidPairs;
    uint32_t rigidGroupCount;         // body pairs with active contacts (velocity-solve groups)
    uint32_t rigidContactSlots;       // kRigidPairContacts x rigidRigidPairCount + proxy contact slots
    uint32_t proxyContactSlots;       // min(required, capacity) proxy particle -> body contact slots
    uint32_t requiredProxyContacts;   // proxy candidates (GpuProxyRigidContactMeta.requiredContactCount)
    uint32_t activeParticleContactsLast; // activeParticleContacts of the last completed contact pass
};

// Rigid-rigid contact point of a collider pair (GpuRigidContact, physics_rigid_types.hlsli):
// kRigidPairContacts slots per pair (box-box manifolds fill up to 4, other shapes one), 80 B.
constexpr uint32_t kRigidPairContacts = 4u; // kRigidContactsPerPair
struct RigidPairContact {
    uint32_t bodyA, bodyB, active, reserved;
    float4 normalPenetration;   // normal A -> B, penetration
    float4 localPointA, localPointB;
    float4 material;            // friction, restitution, static friction
};
// Velocity-solve slot of a contact in its body-pair group
// (GpuRigidBodyPairContactAggregateSlot): normal (w kinetic friction), local points (A.w static
// friction), solver state (accumulated normal impulse, restitution target, tangent accumulation).
struct RigidSlot {
    float4 normal, localA, localB, state;
};
constexpr uint32_t kRigidGroupContacts = 16u; // kRigidBodyPairAggregateContacts

constexpr uint32_t kMaxBoundaryColliders = 64u;  // bits of the per-particle boundary mask
constexpr uint32_t kRigidDedup = 16u;            // kParticleRigidDedupCacheSize
constexpr uint32_t kColliderIterationCap = 64u;  // kParticleRigidColliderIterationCap
constexpr float kBroadPhaseMargin = 0.05f;       // physics_shape_common.hlsli:10

// A batch's per-tick work: `tiles` are element ranges [x, y) of the scenes stepped this tick,
// `count` the number of tiles (device word); kernels launched with a work list run `grid` blocks
// that stride over the tiles.  A null list means "all elements [0, n)" (a single world).
struct WorkList {
    const uint2 *tiles = nullptr;
    const uint32_t *count = nullptr;
    uint32_t grid = 0;
};

// XPBD families in the order a soft iteration solves them (physics_solver.cpp:915-1019).
constexpr uint32_t kFamilies = 6u;
enum : uint32_t { kFamEdges = 0u, kFamSegments = 1u, kFamBends = 2u, kFamJoints = 3u, kFamDistances = 4u, kFamTets = 5u };

// An edge as the solves read it, 16 bytes instead of the record's 32: particle b's top bit marks a
// disabled edge (particle indices stay below 2^29).
struct PackedEdge {
    uint32_t a, b;
    float rest, compliance;
};
__host__ __device__ inline PackedEdge packEdge(const cn_soft_edge &e)
{
    return PackedEdge{e.particle_a, e.particle_b | (e.enabled ? 0u : 0x80000000u), e.rest_length, e.compliance};
}

struct Scene {
    // per-tick work lists of a batch (all null for a single world)
    WorkList wP, wE, wT, wB, wC;      // particles, edges, tets, rigid bodies, colliders
    const uint2 *pColRange = nullptr; // per particle: its scene's range of colQueryOrder
    uint32_t N = 0;
    uint32_t solidEnd = 0;            // 1 + the largest index of a non-fluid particle
    uint32_t fluidExtras = 0;         // a fluid material has cohesion or surface tension
    // ---- particles (reference order) ----
    float4 *x = nullptr, *xprev = nullptr, *v = nullptr;
    const float *radii = nullptr;
    const uint32_t *kinds = nullptr;
    const uint4 *meta = nullptr;            // (environment, phase, layer, mask)
    const uint32_t *matIdx = nullptr;
    const uint32_t *fluidMatIdx = nullptr;
    const uint32_t *ownerTypes = nullptr;
    const uint32_t *ownerIdx = nullptr;
    const uint32_t *fluidGroup = nullptr;   // dense id of (environment, layer, mask) for fluid particles
    const uint32_t *adjOff = nullptr, *adjCnt = nullptr, *adjIdx = nullptr;
    const float4 *contactMaterials = nullptr;
    const cn_fluid_material *fluidMaterials = nullptr;
    float cellSize = 1.0f;

    // ---- soft constraints ----
    uint32_t E = 0, Bn = 0, D = 0, T = 0, S = 0, J = 0, SD = 0;
    const cn_soft_edge *edges = nullptr;
    const cn_soft_bend *bends = nullptr;
    const cn_cloth_dihedral *dihedrals = nullptr;
    const cn_soft_tet *tets = nullptr;
    const cn_strand_segment *segs = nullptr;
    const cn_strand_joint *joints = nullptr;
    const cn_strand_distance *dists = nullptr;
    float4 *segOrient = nullptr;
    // incidence: per-particle (start, count) of its entries in ascending constraint order
    // (physics_scene_gpu_state.cpp:3255-3420); the (constraint, slot) lists themselves are kept
    // for the strand segments and joints, whose applies read them
    const uint2 *edgeRanges = nullptr;
    const uint2 *bendRanges = nullptr;
    const uint2 *tetRanges = nullptr;
    const uint2 *segRanges = nullptr, *segInc = nullptr;
    const uint2 *segJointRanges = nullptr, *segJointInc = nullptr;
    // gather slots: for each constraint entry (edge 2, bend / dihedral 4, tet 4, strand distance 2)
    // the index in its particle's incidence list, where the solve writes that entry's correction
    // record (0xffffffff: no particle); the gathers read each particle's records contiguously.
    // Strand distances use the strand-segment incidence (the reference applies distance c's
    // records to segment c's particles).
    const uint32_t *edgeDst = nullptr, *bendDst = nullptr, *tetDst = nullptr, *distDst = nullptr;
    // per family: the particles [x, y) with records (a single world's apply window)
    uint2 edgeWin{0u, 0u}, bendWin{0u, 0u}, tetWin{0u, 0u}, segWin{0u, 0u};
    // lambdas and per-constraint correction records
    float *edgeLambda = nullptr, *bendLambda = nullptr, *tetLambda = nullptr, *distLambda = nullptr;
    float4 *segLambda = nullptr, *jointLambda = nullptr;
    float4 *edgeCorr = nullptr;   // per edge incidence entry (gather slot)
    float4 *bendCorr = nullptr;   // per bend / dihedral incidence entry
    float4 *tetCorr = nullptr;    // per tet incidence entry
    float4 *segCorr = nullptr;    // 3 per segment
    float4 *jointCorr = nullptr;  // 2 per joint (twistRotationA, twistRotationB)
    float4 *distCorr = nullptr;   // per strand-segment incidence entry
    float4 *posCorr = nullptr, *velCorr = nullptr;
    // coloured XPBD schedules: per family (kFam*) the constraint indices grouped by colour,
    // the colour-Jacobi per-particle sum of a family's corrections (zero between families) and
    // the per-segment sum of the joint family's orientation corrections
    const uint32_t *colOrder[kFamilies] = {};
    float4 *softAcc = nullptr;
    float4 *orientAcc = nullptr;
    // a batch's colour tables, per admitted scene and family (edges, then tets) a run of words:
    // colours, the family's particle window [lo, hi), then colours + 1 starts (scene-local)
    uint32_t *batchColStarts = nullptr;
    // a coloured batch's edges and tets in colour order (pool position e0 + i holds the scene's
    // i-th constraint in colour order; lambdas share that indexing under a coloured schedule) and
    // each tet's last corrections in the same order
    const PackedEdge *edgesC = nullptr;
    const cn_soft_tet *tetsC = nullptr;
    // a batch's edges, packed (its pool has no scene view that would need the record layout)
    const PackedEdge *edgesP = nullptr;
    float4 *tetRecC = nullptr;

    // ---- rigid bodies / colliders ----
    uint32_t B = 0, C = 0;
    float4 *bodyPos = nullptr, *bodyRot = nullptr, *bodyLin = nullptr, *bodyAng = nullptr;
    const float4 *bodyScale = nullptr, *bodyInvInertia = nullptr;
    const uint32_t *bodyType = nullptr;
    float4 *bodyKinPos = nullptr, *bodyKinRot = nullptr;
    uint32_t *bodyKinFlags = nullptr;
    const uint2 *bodyColRanges = nullptr;
    const uint32_t *bodyColIdx = nullptr;
    const cn_collider_geometry *colGeo = nullptr;
    const cn_collider_broadphase *colBp = nullptr;
    const float4 *colMat = nullptr;
    float4 *prevBodyPos = nullptr, *prevBodyRot = nullptr;
    float4 *predBodyPos = nullptr, *predBodyRot = nullptr, *predBodyLin = nullptr, *predBodyAng = nullptr;
    float4 *colAabbMin = nullptr, *colAabbMax = nullptr;
    // rigid-rigid contacts (scenes with dynamic bodies): LBVH over the query-order colliders, the
    // moving colliders' candidate pairs, one contact per pair, body-pair groups for the velocities
    uint32_t rrCapacity = 0;
    uint32_t *rrCount = nullptr, *rrOffset = nullptr;     // per moving collider
    uint2 *rrPairs = nullptr;                              // (collider A, collider B), canonical
    uint2 *rrStage = nullptr;                              // per moving collider: its first pairs
    RigidPairContact *rrContacts = nullptr;
    RigidSlot *rrSlots = nullptr;                          // per sorted contact
    uint32_t *rrKeyA = nullptr, *rrValA = nullptr, *rrKeyB = nullptr, *rrValB = nullptr;
    uint32_t *rrHead = nullptr, *rrGroupOf = nullptr;      // per sorted contact
    uint2 *rrGroups = nullptr;                             // (first sorted contact, contacts)
    uint32_t *bvhKeyA = nullptr, *bvhValA = nullptr, *bvhKeyB = nullptr, *bvhValB = nullptr;
    uint2 *bvhChildren = nullptr;                          // per internal node
    uint32_t *bvhParent = nullptr, *bvhVisits = nullptr;   // per node / internal node
    float4 *bvhMin = nullptr, *bvhMax = nullptr;           // per node
    float4 *bvhWide = nullptr;                             // per internal node: both child boxes (4)
    float4 *bvhBounds = nullptr;                           // scene centre bounds (2)
    // Contact slots: kRigidPairContacts per collider pair, then one per proxy candidate
    // (physics_rigid_generate_proxy_contacts.cs.hlsl appends after the pair contacts)
    uint32_t proxyCapacity = 0, rrSlotCapacity = 0;
    // rigid proxy particles: the first nProxy particles, owned by rigid bodies
    // (physics_particle_sync_rigid_proxy_particles.cs.hlsl)
    uint32_t nProxy = 0;
    const float4 *proxyLocal = nullptr;    // per proxy: scaled body-frame position
    const float4 *bodyProxyMat = nullptr;  // per body: its proxies' contact material
    // dynamic bodies: corrections summed (float atomics) over a pass, applied per body after it
    uint32_t hasDynamic = 0;
    // the particle-rigid contact pass writes its contact records (read by the velocity passes after
    // the iterations): the iteration loops set it for their last contact iteration only
    uint32_t storeRigidContacts = 1;
    float4 *bodyTransCorr = nullptr, *bodyRotCorr = nullptr, *bodyLinVelCorr = nullptr, *bodyAngVelCorr = nullptr;
    // Per collider, the world frame the fluid boundary queries use this substep (4 float4:
    // centre + shape/enabled word, orientation, shape extents, capsule end).
    float4 *colFrame = nullptr;
    const uint32_t *colQueryOrder = nullptr; // moving colliders first, then static
    uint32_t colQueryCount = 0, activeMovingCount = 0;

    // ---- surface render passes (physics/soft/render/*), once per frame ----
    uint32_t surfV = 0, surfT = 0, surfS = 0, surfChunks = 0;
    const uint4 *surfBind = nullptr;        // 2 per vertex: particle indices, then weights (bits)
    const float4 *surfFallback = nullptr;   // per vertex
    const uint4 *surfRanges = nullptr;      // per vertex (start, count, 0, 0) into surfIdx
    const uint32_t *surfIdx = nullptr;      // incident triangles
    const uint4 *surfTri = nullptr;         // per triangle (a, b, c, 0)
    const uint4 *surfChunk = nullptr;       // per 64-particle chunk (surface, start, count, 0)
    const uint2 *surfChunkRange = nullptr;  // per surface (first chunk, chunk count)
    float4 *surfPos = nullptr, *surfNrm = nullptr, *surfTriN = nullptr;
    float4 *surfChunkAabb = nullptr, *surfWorldAabb = nullptr; // (min, max) pairs

    // ---- broadphase ----
    int4 *entries = nullptr;          // (cellX, cellY, cellZ, key) per particle
    uint32_t *keysA = nullptr, *keysB = nullptr, *valsA = nullptr, *valsB = nullptr;
    uint32_t *rank = nullptr;         // particle -> sorted slot
    uint32_t tableMask = 0;           // cell hash table capacity - 1
    uint32_t *tableKeys = nullptr, *tableStart = nullptr;
    uint32_t *cellEnd = nullptr;      // at a run start: end | (mixed-coordinate flag << 31)
    uint32_t *runFlag = nullptr;      // 1 at a run start (fluid scenes)
    uint32_t *runIdx = nullptr;       // exclusive scan of runFlag
    // Fluid scenes solve in "compute order": the runs of the key sort re-ordered along a Morton
    // curve of their cells, each run's particles kept in sorted order.  Runs are numbered r in
    // key order and j in compute order.
    uint32_t *runStartOf = nullptr;   // per run j: compute start | (mixed << 31)
    uint2 *runNbr = nullptr;          // per run j: 27 neighbour runs (compute start | check << 31, end)
    uint32_t *runKey = nullptr, *runVal = nullptr, *runKeyB = nullptr, *runValB = nullptr; // run sort (j -> r)
    uint32_t *runTotal = nullptr;     // number of runs (device word)
    uint32_t *runHashStart = nullptr; // per run r: key-order start | (mixed << 31)
    uint32_t *runLen = nullptr;       // per run r: particle count
    uint32_t *runLenSorted = nullptr; // per run j: particle count (0 past the last run)
    uint32_t *runCompStart = nullptr; // per run j: compute start (exclusive scan of runLenSorted)
    uint32_t *runComp = nullptr;      // per run r: compute start
    uint32_t *runPos = nullptr;       // per run r: j
    uint32_t *cvals = nullptr;        // compute slot -> particle
    int4 *cCell = nullptr;            // compute slot -> cell coordinates
    uint32_t *cRun = nullptr;         // compute slot -> run j

    // ---- fluid (cell order) ----
    uint32_t hasFluid = 0;
    float4 *Xs = nullptr;             // x at the sorted slot (w = invMass)
    float4 *P = nullptr;              // x + accumulated delta, w = tag word (fluid bit, material, group)
    float4 *Pb = nullptr;             // second position buffer (odd iterations) when x is fixed over them
    float4 *P0 = nullptr;             // positions at the superset build when contacts also move fluid x
    float4 *Da = nullptr, *Db = nullptr; // accumulated delta ping-pong
    float4 *Cs = nullptr;             // surface normal xyz, density constraint w
    float4 *Dx = nullptr;             // packed delta + interaction weight (last iteration)
    int4 *sCell = nullptr;            // cell entry at the sorted slot
    uint4 *sMeta = nullptr;           // metadata at the sorted slot
    uint32_t *sInfo = nullptr;        // kind (bit 31 = fluid) | fluid material index
    unsigned long long *sBoundary = nullptr; // boundary-collider candidate mask (query order)
    // Scenes with more colliders than the mask has bits keep per-slot candidate lists instead
    // (physics_particle_count/emit_fluid_boundary_candidates.cs.hlsl): bCount / bOffset per
    // compute slot, bList the colliders' query positions in ascending order (bList == nullptr:
    // the mask is used).
    uint32_t *bCount = nullptr, *bOffset = nullptr, *bList = nullptr;
    uint32_t bListCap = 0;
    uint32_t colBvh = 0;              // the collider LBVH is built every substep (boundary queries)
    uint32_t maxNbr = 128;
    uint32_t *nbr = nullptr;          // [N][maxNbr] sorted slots
    uint32_t *nbrCount = nullptr;     // per sorted slot
    uint32_t supCap = 0;              // superset list slots per particle (0: superset lists off)
    float supMargin = 0.25f;          // superset radius = h * (1 + supMargin)
    uint32_t *sup = nullptr;          // [N][supCap] candidates within the superset radius, traversal order
    uint32_t *supCount = nullptr;     // per sorted slot (> supCap: overflowed)
    uint32_t *fluidMaxDelta = nullptr; // [64] float bits of max |accumulated delta| per iteration
    float4 *fluidVort = nullptr;      // curl xyz + magnitude per sorted slot (vorticity confinement)

    // ---- contact candidates ----
    uint32_t *candCount = nullptr, *candOffset = nullptr; // per particle
    uint32_t *ppCount = nullptr, *ppOffset = nullptr;
    uint2 *rigidPairs = nullptr;      // (particle, body)
    uint32_t rigidPairCapacity = 0;
    RigidContact *rigidContacts = nullptr;
    uint2 *particlePairs = nullptr;   // (a, b)
    uint2 *ppStage = nullptr;         // per particle: its first pairs, staged by the count pass
    uint32_t particlePairCapacity = 0;
    ParticleContact *particleContacts = nullptr;
    DeviceMeta *meta_ = nullptr;
};

// Settings the kernels read (PhysicsSolverConfigBuffer, physics_solver_config.hlsli:5-51).
struct Config {
    float slop, softContactRelaxation, softMaxCorrection, restitutionVelocityThreshold;
    float restitutionPenetrationThreshold, positionFrictionMinDistance;
    float softInternalRelaxation;
    float fluidSolveCoefficient, fluidRelaxation, fluidBoundaryDensityScale, fluidBoundaryDeltaScale;
    float fluidMaxUnderDensityRatio;
    float gravity[3];
    // per-iteration caps on a dynamic body's summed corrections (physics_solver_config.hlsli:31-34)
    float maxTranslationCorrection, maxRotationCorrection, maxLinearVelocityCorrection, maxAngularVelocityCorrection;
    // rigid-rigid contacts (physics_solver_config.hlsli:23-30)
    float rigidRestitutionThreshold, baumgarte, depenetrationRelaxation, maxDepenetration, velocityPenetrationStiffness;
    float manifoldMergeDistance; // manifold_merge_slop_multiplier x slop
};

// A kinematic target staged for a batch tick: pos.xyz, pos.w = the body index (bits); rot = xyzw.
struct BodyTarget {
    float4 pos;
    float4 rot;
};

#ifdef __CUDACC__
// Programmatic dependent launch: a kernel launched with programmatic stream serialization may
// start while the previous kernel of its stream finishes; it waits here until that kernel has
// completed and its writes are visible, then lets the next kernel of the stream launch.  For a
// kernel launched without the attribute both instructions return at once.
__device__ __forceinline__ void pdlEnter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Walks the LBVH over the query-order colliders (colQueryCount >= 2) and calls leaf(j) for every
// sorted leaf j whose box overlaps [qmin, qmax]; leaf returns false to stop the walk.  Each visit
// reads one internal node's record of both child boxes, so only overlapping subtrees are entered.
// Returns false when a push found the kStack-entry stack full (that subtree was skipped).
template <uint32_t kStack, class V, class F>
__device__ __forceinline__ bool bvhQuery(const Scene &s, V qmin, V qmax, F &&leaf)
{
    const uint32_t inner = s.colQueryCount - 1u;
    auto hit = [&](const float4 &lo, const float4 &hi) {
        return qmin.x <= hi.x && qmax.x >= lo.x && qmin.y <= hi.y && qmax.y >= lo.y && qmin.z <= hi.z &&
               qmax.z >= lo.z;
    };
    uint32_t stack[kStack];
    uint32_t sp = 0;
    bool complete = true;
    stack[sp++] = 0u;
    while (sp > 0u) {
        const float4 *w = s.bvhWide + size_t(stack[--sp]) * 4u;
        const float4 l0 = w[0], l1 = w[1], r0 = w[2], r1 = w[3];
        const uint32_t lc = __float_as_uint(l0.w), rc = __float_as_uint(r0.w);
        const bool lo = hit(l0, l1), ro = hit(r0, r1);
        if (lo && lc >= inner && !leaf(lc - inner)) return complete;
        if (ro && rc >= inner && !leaf(rc - inner)) return complete;
        if (ro && rc < inner) {
            if (sp < kStack) stack[sp++] = rc;
            else complete = false;
        }
        if (lo && lc < inner) {
            if (sp < kStack) stack[sp++] = lc;
            else complete = false;
        }
    }
    return complete;
}
#endif

// ------------------------------------------------------------------ launchers (cn_kernels.cu)
// Writes `*count` staged kinematic targets (what cn_solver_set_kinematic_target writes for one).
void launchApplyBodyTargets(const Scene &s, const BodyTarget *list, const uint32_t *count, uint32_t capacity,
                            cudaStream_t st);
void launchRigidPredict(const Scene &s, float dt, float gx, float gy, float gz, cudaStream_t st);
// The LBVH over the query-order colliders' world AABBs (cn_rigid.cu), after the rigid predict.
void launchColliderBvh(const Scene &s, void *scratch, cudaStream_t st);
void launchPredictAndKeys(const Scene &s, float dt, const Config &c, cudaStream_t st);
void launchCellSetup(const Scene &s, uint32_t *scanTmp, void *sortScratch, cudaStream_t st);
// Neighbour and superset lists: entry k of compute slot i at k * N + i (true) or i * cap + k.
bool fluidListsInterleaved();
void launchRigidCandidates(const Scene &s, uint32_t *scanTmp, size_t scanTmpBytes, cudaStream_t st);
void launchParticleCandidates(const Scene &s, uint32_t *scanTmp, size_t scanTmpBytes, cudaStream_t st);
void launchFluidIteration(const Scene &s, uint32_t iter, float dt, const Config &c, bool writeDebug,
                          cudaStream_t st);
void launchFluidGather(const Scene &s, uint32_t iter, cudaStream_t st);
// False when the positions are double-buffered: the gather then runs at the first iteration only.
bool fluidGatherEachIteration(const Scene &s);
// walkCells: every iteration walks the 27 cells (no superset lists).
void launchFluidNeighborsDensity(const Scene &s, const Config &c, uint32_t iter, bool walkCells, cudaStream_t st);
void launchFluidDeltaApplyClamp(const Scene &s, uint32_t iter, float dt, const Config &c, bool writeDebug,
                                cudaStream_t st);
void launchFluidNeighborsOnly(const Scene &s, cudaStream_t st);
// Vorticity confinement (after launchFluidNeighborsOnly's post-update lists): curl, then force.
void launchFluidVorticity(const Scene &s, float dt, cudaStream_t st);
// One iteration of the soft families (gather schedule).  With `rigidContacts` (an iteration whose
// particle-rigid contacts follow the soft families directly: no particle-particle contacts) and
// a tet family, those contacts run in the tet gather's pass; returns true when they did, and the
// caller launches them itself otherwise.
bool launchSoftIteration(const Scene &s, float dt, const Config &c, cudaStream_t st, bool rigidContacts = false);
// The same for the families whose bit (1 << kFam*) is set in `families`, in the family order.
bool launchSoftFamilies(const Scene &s, float dt, const Config &c, cudaStream_t st, uint32_t families,
                        bool rigidContacts = false);
constexpr uint32_t kAllFamilies = (1u << kFamilies) - 1u;
// The XPBD schedule of a solver: CN_XPBD_* and, for the coloured schedules, each family's colour
// count and colour start offsets into Scene::colOrder (host copies for the per-colour launches,
// device copies for the fused kernel).
struct XpbdPlan {
    uint32_t schedule = 0;
    uint32_t colours[kFamilies] = {};
    const uint32_t *hostStarts[kFamilies] = {};
    const uint32_t *devStarts[kFamilies] = {};
};
bool launchSoftIteration(const Scene &s, float dt, const Config &c, const XpbdPlan &plan, cudaStream_t st,
                         bool rigidContacts = false);
// Fused iterations: one thread-block cluster runs every iteration of a substep (soft families in
// `plan`'s schedule, then the particle-rigid contacts when `rigid`), phases separated by cluster
// barriers.  fusedIterationsShape() is {0, 0} when the cluster launch is unavailable.
struct FusedShape {
    uint32_t ctas = 0, threads = 0;
};
FusedShape fusedIterationsShape();
// A batch tick's stepped scenes: kSceneListStride uint2 per scene -- its particle, edge and tet
// ranges [x, y), then the word offsets of its edge and tet colour tables in Scene::batchColStarts.
constexpr uint32_t kSceneListStride = 4u;
constexpr uint32_t kBatchMaxColours = 256u;
constexpr uint32_t kColWordsHeader = 3u; // colours, window lo, window hi
// A batch tick's iterations as one persistent kernel (cn_batch): `clusters` clusters of `ctas`
// CTAs, each taking stepped scenes from `next` (zero at the tick's start) until `sceneCount`.
struct BatchFusedPlan {
    uint32_t iterations, softIterations, contactIterations;
    const uint2 *scenes;
    const uint32_t *sceneCount;
    uint32_t *next;
};
// Clusters of `ctas` CTAs that fit on the device at once (0: unavailable).
uint32_t batchFusedClusters(uint32_t ctas);
void launchBatchFusedIterations(const Scene &s, const Config &c, float dt, const BatchFusedPlan &plan, uint32_t ctas,
                                uint32_t clusters, cudaStream_t st);
// One iteration of a batch's edge and tet families under a coloured schedule: per family and
// colour k < maxColours[family] one kernel over the stepped scenes (`scenes`, `sceneCount`), the
// grid's blocks split evenly over the scenes' colour-k constraints; colour Jacobi then adds each
// scene's sums to x over the family's particle window.
void launchBatchColourIteration(const Scene &s, float dt, const Config &c, uint32_t schedule, const uint32_t maxColours[2],
                                const uint2 *scenes, const uint32_t *sceneCount, uint32_t grid, cudaStream_t st);
void launchFusedIterations(const Scene &s, const Config &c, float dt, const XpbdPlan &plan, uint32_t iterations,
                           uint32_t softIterations, uint32_t contactIterations, bool rigid, const FusedShape &shape,
                           cudaStream_t st);
void launchContacts(const Scene &s, const Config &c, bool particleContacts, bool rigidContacts,
                    cudaStream_t st);
void launchUpdateVelocities(const Scene &s, float dt, const float4 *fluidDelta, cudaStream_t st);
void launchFluidBoundaryVelocities(const Scene &s, float dt, const Config &c, cudaStream_t st);
void launchRigidContactVelocities(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st);
void launchParticleContactVelocities(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st);
void launchCopyPredictedRigid(const Scene &s, cudaStream_t st);
// Dynamic bodies: summed position corrections applied (physics_rigid_apply_corrections), velocities
// from the pose change (physics_rigid_update_velocities), and the particle-rigid velocity
// iterations with the bodies' velocity corrections applied after each.
void launchApplyRigidCorrections(const Scene &s, const Config &c, cudaStream_t st);
void launchUpdateRigidVelocities(const Scene &s, float dt, cudaStream_t st);
void launchRigidContactVelocitiesDynamic(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st);
// Rigid proxy particles placed at their bodies' predicted poses
// (physics_particle_sync_rigid_proxy_particles.cs.hlsl; the predict does it for the first time).
void launchSyncRigidProxies(const Scene &s, cudaStream_t st);

// ---------------------------------------------------------------- batch admission (cn_batch.cpp)
// A scene's upload image: every per-element array a batch pool holds for it, with the scene's own
// (0-based) indices, each segment 16-byte aligned in one host buffer.  Admission copies the image
// to a device staging buffer in one transfer and k_admitScene scatters it into the pool ranges,
// adding the scene's range offsets to every index field.
enum AdmitSegment : uint32_t {
    kAdmX, kAdmV, kAdmRadii, kAdmKinds, kAdmMeta, kAdmMatIdx, kAdmOwnerTypes, kAdmOwnerIdx, kAdmEdgeRanges,
    kAdmTetRanges, kAdmEdges, kAdmEdgeDst, kAdmTets, kAdmTetDst, kAdmMaterials, kAdmBodyPos, kAdmBodyRot,
    kAdmBodyLin, kAdmBodyAng, kAdmBodyScale, kAdmBodyInvI, kAdmBodyType, kAdmKinPos, kAdmKinRot, kAdmKinFlags,
    kAdmBodyColRanges, kAdmBodyColIdx, kAdmColGeo, kAdmColBp, kAdmColMat, kAdmQueryOrder, kAdmEdgeColOrder,
    kAdmTetColOrder, kAdmColStarts, kAdmSegments
};
struct AdmitImage {
    const uint8_t *img = nullptr;          // the staging copy on the device
    uint64_t off[kAdmSegments] = {};       // byte offset of each segment
    uint32_t N = 0, E = 0, T = 0, B = 0, C = 0, CI = 0, M = 0, queryCount = 0;
    uint32_t p0 = 0, e0 = 0, t0 = 0, ei0 = 0, ti0 = 0, b0 = 0, c0 = 0, ci0 = 0, m0 = 0; // pool offsets
    uint32_t colWords = 0, k0 = 0;         // colour-table words (0: none) and their pool offset
};
void launchAdmitScene(const Scene &s, const AdmitImage &a, cudaStream_t st);

// ---------------------------------------------------------------- rigid-rigid contacts (cn_rigid.cu)
// Scratch of the rigid broadphase and grouping (sort + scan), in bytes, for C colliders and
// `pairs` candidate pairs.
size_t rigidScratchBytes(uint32_t colliders, uint32_t pairs);
// LBVH over the colliders' world AABBs, the moving colliders' candidate pairs, and one contact
// per pair (physics_rigid_bvh_*, physics_rigid_count/emit_pairs, physics_rigid_generate_contacts).
void launchRigidBroadphaseAndContacts(const Scene &s, const Config &c, void *scratch, cudaStream_t st);
// One contact slot per proxy candidate after the pair contacts: a proxy particle as a sphere of
// its body against the candidate body's colliders (physics_rigid_generate_proxy_contacts).
void launchProxyRigidContacts(const Scene &s, cudaStream_t st);
// Body-pair groups of the active contacts and their velocity slots
// (physics_rigid_init_contact_velocities).
void launchRigidVelocityInit(const Scene &s, const Config &c, void *scratch, cudaStream_t st);
// Position-level depenetration of every contact (physics_rigid_depenetrate_contacts).
void launchRigidDepenetration(const Scene &s, const Config &c, cudaStream_t st);
// `iterations` rounds of the group velocity solve, the body corrections applied after each
// (physics_rigid_solve_contact_velocities + apply_contact_velocities); rounds past
// `contactIterations` only apply.
void launchRigidContactVelocitySolve(const Scene &s, const Config &c, uint32_t iterations, uint32_t contactIterations,
                                     cudaStream_t st);
// Skinning, triangle and vertex normals, chunk and surface AABBs from the current positions.
void launchSurfaceRender(const Scene &s, cudaStream_t st);
// debug export of the compacted cell-range table (reference layout)
void launchExportCellRanges(const Scene &s, uint4 *out, uint32_t capacity, uint32_t *scanTmp,
                            size_t scanTmpBytes, cudaStream_t st);

// ------------------------------------------------------------------ sort / scan (cn_sort.cu)
// Stable LSD radix sort of (key, index) pairs, 8-bit digits, onesweep passes with
// decoupled look-back.  keys/vals A hold the input keys (vals ignored: the input index is
// implied) and receive the sorted result; B is the ping-pong buffer.
size_t radixSortScratchBytes(uint32_t n);
// With `count` (device word), only the first min(n, *count) pairs are sorted; the rest of A is
// left as it was.
void radixSortPairs(uint32_t *keysA, uint32_t *valsA, uint32_t *keysB, uint32_t *valsB, uint32_t n,
                    void *scratch, uint32_t *waitTimeouts, cudaStream_t st, const uint32_t *count = nullptr);
// Exclusive scan of n uint32 values; *total (device) receives the sum.
size_t scanScratchBytes(uint32_t n);
void exclusiveScan(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *total, void *scratch,
                   cudaStream_t st);

} // namespace cn
