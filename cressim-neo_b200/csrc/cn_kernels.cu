// cn_kernels.cu -- sm_100a kernels of the CRESSim-Neo particle physics substep.
//
// Each kernel cites the reference HLSL pass (paths relative to the reference project root)
// whose result it reproduces.  The reference dispatches ~20 passes per solver iteration, each
// a 64-thread-group 1-D dispatch over particles or constraints.  Here:
//  * predict + cell key + sort key are one pass over particles;
//  * the cell-range table is a hash map keyed by the reference's 32-bit cell key, with the
//    reference's "skip a cell whose key is 0xffffffff" and coordinate-compare semantics;
//  * the fluid solve runs in cell order (sorted slots): one kernel builds the neighbour list
//    and the density constraint, one kernel computes the position delta, applies it and
//    clamps against the boundary (the reference's four fluid passes per iteration);
//  * particle-rigid contacts are generated, solved and summed per particle in candidate-pair
//    order, so their sums are deterministic (the reference uses float atomics).
// Arithmetic follows the reference's expression order; the library is built with
// --fmad=false so float32 results match a CPU evaluation of the same order.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <utility>
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "cn_device.h"
#include "cn_math.cuh"

namespace cn {
namespace {

constexpr int kThreads = 256;
#ifndef CN_LIST_ROW_MAJOR
constexpr bool kInterleavedLists = true;
#else
constexpr bool kInterleavedLists = false;
#endif
inline unsigned blocksFor(size_t n) { return n == 0 ? 1u : unsigned((n + kThreads - 1) / kThreads); }
// Block size of the fluid neighbour and delta kernels.
constexpr uint32_t kFluidThreads = 128u;
inline unsigned fluidBlocksFor(size_t n) { return n == 0 ? 1u : unsigned((n + kFluidThreads - 1) / kFluidThreads); }
// Grid of a kernel that strides over a device-counted list of capacity n: 16 blocks per SM at most.
inline unsigned pairGrid(size_t n) { return std::min<unsigned>(blocksFor(n), 148u * 16u); }
// Per-slot fluid word: bit 31 = fluid particle, bits 16..30 = fluid material, bits 0..15 = filter
// group (a dense id of the particle's (environment, layer, mask) triple).  P.w carries the same
// word with bit 31 meaning "fluid and invMass > kEps" (the neighbour candidate filter).
constexpr uint32_t kFluidBit = 0x80000000u;
constexpr uint32_t kMaxTrackedIterations = 64u; // fluid iterations whose max |delta| is tracked
__host__ __device__ __forceinline__ uint32_t infoMaterial(uint32_t info) { return (info >> 16) & 0x7fffu; }
__host__ __device__ __forceinline__ uint32_t infoGroup(uint32_t info) { return info & 0xffffu; }

__device__ __forceinline__ float4 ld4(const float4 *p) { return __ldg(p); }

// One element per thread over [0, n) (a single world), or -- with a work list -- a fixed grid
// striding over the list's tiles: each tile is an element range [x, y) of one resident scene of
// a batch, so a launch covers exactly the scenes stepped this tick.
template <class F> __device__ __forceinline__ void forEachElem(const WorkList &w, uint32_t n, F &&f)
{
    if (w.tiles == nullptr) {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < n) f(i);
        return;
    }
    const uint32_t count = *w.count;
    for (uint32_t t = blockIdx.x; t < count; t += gridDim.x) {
        const uint2 r = w.tiles[t];
        for (uint32_t i = r.x + threadIdx.x; i < r.y; i += blockDim.x) f(i);
    }
}
inline unsigned gridFor(const WorkList &w, size_t n) { return w.tiles ? w.grid : blocksFor(n); }

// The soft families' solves and gathers, the colour passes and the particle-rigid contacts run in
// small blocks: a single world's few hundred to few thousand elements then spread over more SMs
// (64 threads: the 16^3 cube's frame 3.30 -> 2.94 ms), a batch's work-list grid in blocks of 128
// (its tick is 8 % slower with 64).
constexpr int kSoftThreads = 64;
constexpr int kSoftBatchThreads = 128;
inline unsigned softThreads(const Scene &s) { return s.wP.tiles ? kSoftBatchThreads : kSoftThreads; }
inline unsigned softBlocksFor(size_t n) { return n == 0 ? 1u : unsigned((n + kSoftThreads - 1) / kSoftThreads); }
inline unsigned softGridFor(const WorkList &w, size_t n) { return w.tiles ? w.grid : softBlocksFor(n); }
inline unsigned softApplyGrid(const Scene &s, uint2 win)
{
    return s.wP.tiles ? gridFor(s.wP, s.N) : softBlocksFor(win.y > win.x ? win.y - win.x : 0u);
}

// Launches `k` with programmatic stream serialization (the kernel starts with pdlEnter()), so its
// launch and CTA dispatch overlap the previous kernel's tail; CN_PDL=0 in the environment turns
// it off.  Used for the kernels of the solver iterations, which run back to back in thousands.
bool pdlEnabled()
{
    static const bool on = [] {
        const char *e = std::getenv("CN_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}
template <class... P, class... A>
void launchPdl(void (*k)(P...), unsigned grid, unsigned block, cudaStream_t st, A &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(block, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdlEnabled() ? 1u : 0u;
    cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}
// The same for loops that one block runs over a small family (rigid bodies, colliders).
template <class F> __device__ __forceinline__ void forEachInBlock(const WorkList &w, uint32_t n, F &&f)
{
    if (w.tiles == nullptr) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) f(i);
        return;
    }
    // body / collider tiles are one scene's few elements: one thread per tile
    const uint32_t count = *w.count;
    for (uint32_t t = threadIdx.x; t < count; t += blockDim.x) {
        const uint2 r = w.tiles[t];
        for (uint32_t i = r.x; i < r.y; ++i) f(i);
    }
}

// ------------------------------------------------------------------------------------------
// Rigid predict (static, kinematic and dynamic branches)
// physics_rigid_predict.cs.hlsl:20-81, collider world AABBs physics_rigid_update_world_aabbs.cs.hlsl
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ void rigidPredictBody(const Scene &s, float dt, float gx, float gy, float gz, uint32_t b)
{
    const float4 p = s.bodyPos[b];
    const float4 q = qNormalize(s.bodyRot[b]);
    const float4 lin = s.bodyLin[b], ang = s.bodyAng[b];
    const bool kin = (s.bodyKinFlags[b] & 1u) != 0u;
    const float4 kq = qNormalize(s.bodyKinRot[b]);
    s.prevBodyPos[b] = p;
    s.prevBodyRot[b] = q;
    const uint32_t type = s.bodyType[b];
    if (type == CN_BODY_STATIC) {
        s.predBodyPos[b] = p;
        s.predBodyRot[b] = q;
        s.predBodyLin[b] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.predBodyAng[b] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else if (type == CN_BODY_KINEMATIC) {
        const f3 pp = kin ? xyz(s.bodyKinPos[b]) : xyz(p);
        const float4 pq = kin ? kq : q;
        const f3 l = (pp - xyz(p)) / mx(dt, kEps);
        const f3 a = angularVelocityFromQuaternionDelta(q, pq, mx(dt, kEps));
        s.predBodyPos[b] = mk4(pp, p.w);
        s.predBodyRot[b] = pq;
        s.predBodyLin[b] = mk4(l, lin.w);
        s.predBodyAng[b] = mk4(a, ang.w);
    } else {
        const f3 l = xyz(lin) + f3{gx, gy, gz} * dt;
        s.predBodyPos[b] = mk4(xyz(p) + l * dt, p.w);
        s.predBodyRot[b] = integrateOrientation(q, xyz(ang), dt);
        s.predBodyLin[b] = mk4(l, lin.w);
        s.predBodyAng[b] = ang;
    }
}

__device__ __forceinline__ void colliderAabb(const Scene &s, uint32_t c)
{
    const cn_collider_broadphase bp = s.colBp[c];
    const uint32_t ob = bp.owner_body;
    if (ob >= s.B || bp.enabled_flag == 0u) {
        s.colAabbMin[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.colAabbMax[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 sc = s.bodyScale[ob];
    const cn_collider_geometry cg = s.colGeo[c];
    const float4 params = make_float4(cg.shape_params[0], cg.shape_params[1], cg.shape_params[2],
                                      cg.shape_params[3]);
    const f3 lp = f3{cg.local_position[0], cg.local_position[1], cg.local_position[2]} * xyz(sc);
    const float4 lq = qNormalize(make_float4(cg.local_orientation[0], cg.local_orientation[1],
                                             cg.local_orientation[2], cg.local_orientation[3]));
    const float4 bq = qNormalize(s.predBodyRot[ob]);
    const float4 pbq = qNormalize(s.prevBodyRot[ob]);
    const f3 cp = xyz(s.predBodyPos[ob]) + qRotate(bq, lp);
    const float4 cq = qNormalize(qMul(bq, lq));
    const f3 pcp = xyz(s.prevBodyPos[ob]) + qRotate(pbq, lp);
    const float4 pcq = qNormalize(qMul(pbq, lq));
    f3 a0, a1, b0, b1;
    computeBodyAabb(bp.shape_type, cp, cq, params, sc, a0, a1);
    computeBodyAabb(bp.shape_type, pcp, pcq, params, sc, b0, b1);
    const f3 lo = min3(a0, b0) - f3{kBroadPhaseMargin, kBroadPhaseMargin, kBroadPhaseMargin};
    const f3 hi = max3(a1, b1) + f3{kBroadPhaseMargin, kBroadPhaseMargin, kBroadPhaseMargin};
    s.colAabbMin[c] = mk4(lo, 0.f);
    s.colAabbMax[c] = mk4(hi, 0.f);
}

__device__ __forceinline__ void colliderFrame(const Scene &s, uint32_t c)
{
    const cn_collider_broadphase bp = s.colBp[c];
    float4 *fr = s.colFrame + size_t(c) * 4;
    const uint32_t b = bp.owner_body;
    if (bp.enabled_flag == 0u || b >= s.B) {
        fr[0] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
        return;
    }
    const f3 bpos = xyz(s.predBodyPos[b]);
    const float4 bq = qNormalize(s.predBodyRot[b]);
    const float4 sc = s.bodyScale[b];
    const cn_collider_geometry cg = s.colGeo[c];
    const f3 cwp = bpos + qRotate(bq, f3{cg.local_position[0], cg.local_position[1], cg.local_position[2]});
    const float4 cwq = qNormalize(qMul(bq, qNormalize(make_float4(cg.local_orientation[0], cg.local_orientation[1],
                                                                  cg.local_orientation[2], cg.local_orientation[3]))));
    const float4 sp = make_float4(cg.shape_params[0], cg.shape_params[1], cg.shape_params[2], cg.shape_params[3]);
    float4 e0 = make_float4(0.f, 0.f, 0.f, 0.f), e1 = e0;
    if (bp.shape_type == CN_COLLIDER_SPHERE) {
        e0.x = sphereRadius(sp, sc);
    } else if (bp.shape_type == CN_COLLIDER_BOX) {
        e0 = mk4(boxHalfExtents(sp, sc), 0.f);
    } else {
        f3 a, b2;
        float cr = 0.0f;
        capsuleSegment(cwp, cwq, sp, sc, a, b2, cr);
        e0 = mk4(a, cr);
        e1 = mk4(b2, 0.f);
    }
    fr[0] = mk4(cwp, __uint_as_float(1u | (bp.shape_type << 8)));
    fr[1] = cwq;
    fr[2] = e0;
    fr[3] = e1;
}

__global__ void __launch_bounds__(kThreads) k_rigidPredict(Scene s, float dt, float gx, float gy, float gz)
{
    forEachInBlock(s.wB, s.B, [&](uint32_t b) { rigidPredictBody(s, dt, gx, gy, gz, b); });
    __syncthreads();
    forEachInBlock(s.wC, s.C, [&](uint32_t c) { colliderAabb(s, c); });
    // Collider frames for the fluid boundary queries, with the arithmetic of
    // physics_fluid_boundary_common.hlsli:11-40 (unscaled local offset), done once per collider.
    forEachInBlock(s.wC, s.C, [&](uint32_t c) { colliderFrame(s, c); });
}

// The same in two grid-wide launches (bodies, then colliders), for a single world with many bodies:
// one block would walk them all in turn.
__global__ void __launch_bounds__(kThreads) k_rigidPredictBodies(Scene s, float dt, float gx, float gy, float gz)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < s.B) rigidPredictBody(s, dt, gx, gy, gz, b);
}

__global__ void __launch_bounds__(kThreads) k_colliderBoundsFrames(Scene s)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= s.C) return;
    colliderAabb(s, c);
    colliderFrame(s, c);
}

__global__ void k_applyBodyTargets(Scene s, const BodyTarget *list, const uint32_t *count)
{
    const uint32_t n = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const BodyTarget bt = list[t];
        const uint32_t b = __float_as_uint(bt.pos.w);
        if (b >= s.B) continue;
        s.bodyKinPos[b] = make_float4(bt.pos.x, bt.pos.y, bt.pos.z, 0.0f);
        s.bodyKinRot[b] = bt.rot;
        s.bodyKinFlags[b] = 1u;
    }
}

// physics_rigid_update_velocities (copyPredictedRigidBodiesToPersistentState)
__device__ __forceinline__ void copyPredictedBody(const Scene &s, uint32_t b)
{
    s.bodyPos[b] = s.predBodyPos[b];
    s.bodyRot[b] = s.predBodyRot[b];
    s.bodyLin[b] = s.predBodyLin[b];
    s.bodyAng[b] = s.predBodyAng[b];
}

__global__ void k_copyPredictedRigid(Scene s)
{
    forEachInBlock(s.wB, s.B, [&](uint32_t b) { copyPredictedBody(s, b); });
}

// ------------------------------------------------------------------------------------------
// Predict + broadphase entry + sort key.
// physics_soft_predict.cs.hlsl:12-47, physics_particle_build_broad_phase_entries.cs.hlsl:9-35,
// physics_particle_build_broad_phase_keys.cs.hlsl:8-23
// ------------------------------------------------------------------------------------------
// physics_particle_sync_rigid_proxy_particles.cs.hlsl: a proxy particle at its body's predicted pose
__device__ __forceinline__ f3 proxyWorldPosition(const Scene &s, uint32_t i)
{
    const uint32_t b = s.ownerIdx[i];
    const float4 q = qNormalize(s.predBodyRot[b]);
    return xyz(s.predBodyPos[b]) + qRotate(q, xyz(s.proxyLocal[i]));
}

__device__ __forceinline__ void predictParticle(const Scene &s, float dt, float gx, float gy, float gz, bool writeKeys, uint32_t i)
{
    const float4 pim = s.x[i];
    const float4 v0 = s.v[i];            // loaded with x (not after the mass test):
    const uint32_t kind = s.kinds[i];    // one round trip fewer
    const f3 pos = xyz(pim);
    s.xprev[i] = mk4(pos, 0.0f);
    f3 pp = pos;
    if (pim.w <= kEps) {
        s.v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        f3 vel = xyz(v0);
        float gs = 1.0f;
        if (kind == CN_PARTICLE_FLUID) gs = s.fluidMaterials[s.fluidMatIdx[i]].gravity_scale;
        vel = vel + f3{gx, gy, gz} * (dt * gs);
        pp = pos + vel * dt;
        s.v[i] = mk4(vel, 0.0f);
        s.x[i] = mk4(pp, pim.w);
    }
    if (i < s.nProxy) { // the proxy sync that follows the predict (physics_solver.cpp:587-592)
        pp = proxyWorldPosition(s, i);
        s.x[i] = mk4(pp, pim.w);
    }
    if (!writeKeys) return;
    const float safe = mx(s.cellSize, 1.0e-4f);
    const float inv = 1.0f / safe;
    const int cx = int(floorf(pp.x * inv));
    const int cy = int(floorf(pp.y * inv));
    const int cz = int(floorf(pp.z * inv));
    const uint32_t key = cellKey(cx, cy, cz);
    s.entries[i] = make_int4(cx, cy, cz, int(key));
    s.keysA[i] = key;
}

__global__ void __launch_bounds__(kThreads) k_predictKeys(Scene s, float dt, float gx, float gy, float gz,
                                                          bool writeKeys)
{
    forEachElem(s.wP, s.N, [&](uint32_t i) { predictParticle(s, dt, gx, gy, gz, writeKeys, i); });
}

// ------------------------------------------------------------------------------------------
// Cell table + cell-order gathers (one thread per sorted slot).
// physics_particle_mark_cell_range_starts.cs.hlsl, physics_particle_build_cell_ranges.cs.hlsl
// (the reference compacts runs into a sorted table searched by binary search; the same
// (key -> run) mapping is stored here as an open-addressing hash map), plus the fluid
// boundary candidate query (physics_particle_count/emit_fluid_boundary_candidates.cs.hlsl).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fluidBoundaryMaskFor(const Scene &s, uint32_t p, f3 pos,
                                                         unsigned long long &mask)
{
    mask = 0ull;
    const float pr = mx(s.radii[p], 0.0f);
    const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[p]];
    const float support = mx(fm.smoothing_radius, pr);
    const float reuse = mx(mx(fm.cfl_radius, pr), support);
    const float qr = support + reuse;
    const f3 qmin = pos - f3{qr, qr, qr}, qmax = pos + f3{qr, qr, qr};
    const uint4 m = s.meta[p];
    uint32_t overflow = 0;
    for (uint32_t k = 0; k < s.colQueryCount; ++k) {
        const uint32_t c = s.colQueryOrder[k];
        if (!aabbOverlaps(qmin, qmax, xyz(s.colAabbMin[c]), xyz(s.colAabbMax[c]))) continue;
        const cn_collider_broadphase bp = s.colBp[c];
        const uint32_t bt = s.bodyType[bp.owner_body];
        if (bp.enabled_flag != 0u && bp.environment_index == m.x && bt != CN_BODY_DYNAMIC &&
            (m.w & bp.collision_layer) != 0u && (bp.collision_mask & m.z) != 0u) {
            if (k < kMaxBoundaryColliders) mask |= 1ull << k;
            else overflow = 1;
        }
    }
    return overflow;
}

// The same query for scenes with more colliders than the mask holds: counts (kEmit false) or
// writes (kEmit true, at most `room` entries) the candidates' query positions in ascending order.
// With the collider LBVH built this substep, the overlapping leaves come from the tree (sorted
// back into query order; more than kCandidateHits of them fall back to the scan); the filters
// are those of the mask query.
template <bool kEmit>
__device__ uint32_t fluidBoundaryListFor(const Scene &s, uint32_t p, f3 pos, uint32_t *out, uint32_t room);

__global__ void __launch_bounds__(kThreads) k_cellSetup(Scene s)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t p = s.valsA[slot];
    const uint32_t key = s.keysA[slot];
    if (!s.hasFluid) s.rank[p] = slot; // fluid scenes rank particles in compute order
    const int4 e = s.entries[p];
    s.sCell[slot] = e;
    const bool start = slot == 0 || s.keysA[slot - 1] != key;
    if (s.runFlag) s.runFlag[slot] = start ? 1u : 0u;
    if (!start) return;
    uint32_t end = slot + 1;
    uint32_t mixed = 0;
    while (end < s.N && s.keysA[end] == key) {
        const int4 o = s.entries[s.valsA[end]];
        if (o.x != e.x || o.y != e.y || o.z != e.z) mixed = 1;
        ++end;
    }
    s.cellEnd[slot] = end | (mixed << 31);
    if (key == kInvalid) return; // a run keyed 0xffffffff is never found by the reference lookup
    uint32_t h = mixKey(key) & s.tableMask;
    for (uint32_t probe = 0; probe <= s.tableMask; ++probe) {
        const uint32_t prev = atomicCAS(&s.tableKeys[h], kInvalid, key);
        if (prev == kInvalid || prev == key) {
            s.tableStart[h] = slot;
            return;
        }
        h = (h + 1) & s.tableMask;
    }
}

// Returns the run [start, end) of cell key `key`, or false (FindCellRange semantics).
__device__ __forceinline__ bool findRun(const Scene &s, uint32_t key, uint32_t &start, uint32_t &end,
                                        bool &mixed)
{
    if (key == kInvalid) return false;
    uint32_t h = mixKey(key) & s.tableMask;
    for (uint32_t probe = 0; probe <= s.tableMask; ++probe) {
        const uint32_t k = __ldg(&s.tableKeys[h]);
        if (k == key) {
            start = __ldg(&s.tableStart[h]);
            const uint32_t ce = __ldg(&s.cellEnd[start]);
            end = ce & 0x7fffffffu;
            mixed = (ce >> 31) != 0u;
            return true;
        }
        if (k == kInvalid) return false;
        h = (h + 1) & s.tableMask;
    }
    return false;
}

// Compute order (fluid scenes).  The key sort groups each cell's particles into a run but
// scatters neighbouring cells over the whole array (the key is a hash).  The fluid kernels
// instead walk the runs along a Morton curve of their cells, so a warp's particles share
// neighbour cells and their gathers hit in L1.  Inside a run the particles keep their sorted
// order, which is all the reference's neighbour order depends on (cells in (dz, dy, dx) order,
// each cell's particles in sorted order), so results are unchanged.
__device__ __forceinline__ uint32_t spreadBits3(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// 30-bit Morton code of the low 10 bits of each cell coordinate (wrapping only costs locality).
__device__ __forceinline__ uint32_t cellMorton(int4 e)
{
    return spreadBits3(uint32_t(e.x)) | (spreadBits3(uint32_t(e.y)) << 1) | (spreadBits3(uint32_t(e.z)) << 2);
}

__device__ __forceinline__ uint32_t runOfSlot(const Scene &s, uint32_t slot)
{
    return s.runIdx[slot] + s.runFlag[slot] - 1u;
}

// Per run r (at its key-order start): sort key, start and length.
__global__ void __launch_bounds__(kThreads) k_runKeys(Scene s)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N || s.runFlag[slot] == 0u) return;
    const uint32_t r = s.runIdx[slot];
    const uint32_t ce = s.cellEnd[slot];
    s.runKey[r] = cellMorton(s.sCell[slot]);
    s.runHashStart[r] = slot | (ce & 0x80000000u);
    s.runLen[r] = (ce & 0x7fffffffu) - slot;
}

// Per sorted run j: its length (0 for the padding past the last run).
__global__ void __launch_bounds__(kThreads) k_runLengths(Scene s)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.N) return;
    s.runLenSorted[j] = s.runKey[j] != kInvalid ? s.runLen[s.runVal[j]] : 0u;
}

// Per sorted run j: compute start, and the r -> (compute start, j) maps.
__global__ void __launch_bounds__(kThreads) k_runPlace(Scene s)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.N || s.runKey[j] == kInvalid) return;
    const uint32_t r = s.runVal[j];
    const uint32_t cs = s.runCompStart[j];
    s.runComp[r] = cs;
    s.runPos[r] = j;
    s.runStartOf[j] = cs | (s.runHashStart[r] & 0x80000000u);
}

// Per key-order slot: its compute slot, and the per-particle data the fluid kernels read there.
__global__ void __launch_bounds__(kThreads) k_computeOrderSetup(Scene s)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t r = runOfSlot(s, slot);
    const uint32_t cslot = s.runComp[r] + (slot - (s.runHashStart[r] & 0x7fffffffu));
    const uint32_t p = s.valsA[slot];
    s.cvals[cslot] = p;
    s.rank[p] = cslot;
    s.cCell[cslot] = s.sCell[slot];
    s.cRun[cslot] = s.runPos[r];
    const bool fluid = s.kinds[p] == CN_PARTICLE_FLUID;
    s.sMeta[cslot] = s.meta[p];
    s.sInfo[cslot] = fluid ? (kFluidBit | ((s.fluidMatIdx[p] & 0x7fffu) << 16) | (s.fluidGroup[p] & 0xffffu)) : 0u;
    unsigned long long mask = 0ull;
    if (s.bList) {
        s.bCount[cslot] = fluid && s.colQueryCount > 0 ? fluidBoundaryListFor<false>(s, p, xyz(s.x[p]), nullptr, 0u) : 0u;
    } else if (fluid && s.colQueryCount > 0) {
        if (fluidBoundaryMaskFor(s, p, xyz(s.x[p]), mask)) atomicAdd(&s.meta_->boundaryMaskOverflow, 1u);
    }
    s.sBoundary[cslot] = mask;
}

// Per compute slot: its boundary candidates at its offset (after the count above and a scan).
__global__ void __launch_bounds__(kThreads) k_fluidBoundaryEmit(Scene s)
{
    const uint32_t cslot = blockIdx.x * blockDim.x + threadIdx.x;
    if (cslot >= s.N) return;
    const uint32_t n = s.bCount[cslot];
    if (n == 0u) return;
    const uint32_t off = s.bOffset[cslot];
    const uint32_t room = off < s.bListCap ? s.bListCap - off : 0u;
    if (room < n) atomicAdd(&s.meta_->boundaryMaskOverflow, 1u);
    if (room == 0u) return;
    const uint32_t p = s.cvals[cslot];
    fluidBoundaryListFor<true>(s, p, xyz(s.x[p]), s.bList + off, room < n ? room : n);
}

// The run of cell key `key` in compute slots (FindCellRange semantics).
__device__ __forceinline__ bool findRunCompute(const Scene &s, uint32_t key, uint32_t &start, uint32_t &end,
                                               bool &mixed)
{
    uint32_t hs, he;
    if (!findRun(s, key, hs, he, mixed)) return false;
    start = __ldg(&s.runComp[__ldg(&s.runIdx[hs])]);
    end = start + (he - hs);
    return true;
}

// Per run j: the 27 neighbour runs in the reference's traversal order (dz, dy, dx), looked up
// once per substep.  Entry k = (compute start | checkCoordinates << 31, end); empty when the
// target cell has no run or its (uniform) run holds another cell that hashes to the same key.
__device__ __forceinline__ void runNeighborAt(const Scene &s, uint32_t j, uint32_t k)
{
    const uint32_t r = s.runVal[j];
    const int4 e = s.sCell[s.runHashStart[r] & 0x7fffffffu];
    const int dz = int(k / 9u) - 1, dy = int((k / 3u) % 3u) - 1, dx = int(k % 3u) - 1;
    const int tx = e.x + dx, ty = e.y + dy, tz = e.z + dz;
    uint32_t hs = 0, he = 0;
    bool mixed = false;
    uint2 rg = make_uint2(0u, 0u);
    if (findRun(s, cellKey(tx, ty, tz), hs, he, mixed)) {
        const uint32_t cs = s.runComp[s.runIdx[hs]];
        if (mixed) {
            rg = make_uint2(cs | 0x80000000u, cs + (he - hs));
        } else {
            const int4 ce = s.sCell[hs];
            if (ce.x == tx && ce.y == ty && ce.z == tz) rg = make_uint2(cs, cs + (he - hs));
        }
    }
    s.runNbr[size_t(j) * 27u + k] = rg;
}

__global__ void __launch_bounds__(kThreads) k_runNeighbors(Scene s)
{
    // one thread per (run j, neighbour k), striding over the runs that exist (a device count):
    // the 27 hash probes of a run proceed in parallel
    const uint64_t items = uint64_t(__ldg(s.runTotal)) * 27u;
    for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < items;
         t += uint64_t(gridDim.x) * blockDim.x)
        runNeighborAt(s, uint32_t(t / 27u), uint32_t(t % 27u));
}

// ------------------------------------------------------------------------------------------
// Particle-rigid candidate pairs (solid particles vs static/kinematic bodies, dedup 16)
// physics_particle_count_particle_rigid_candidates.cs.hlsl:113-151, emit, finalize.
// ------------------------------------------------------------------------------------------
// Query-order positions of the colliders whose AABB overlaps [qmin, qmax], ascending, from this
// substep's LBVH over the query-order colliders (built for scenes with dynamic bodies); false when
// more than kCandidateHits overlap or the walk outgrows its stack -- the caller then scans.
constexpr uint32_t kCandidateHits = 32u, kCandidateStack = 64u;
__device__ __forceinline__ bool bvhOverlaps(const Scene &s, f3 qmin, f3 qmax, uint32_t *hits, uint32_t &nh)
{
    nh = 0;
    bool room = true;
    const bool complete = bvhQuery<kCandidateStack>(s, qmin, qmax, [&](uint32_t leaf) -> bool {
        if (nh == kCandidateHits) return room = false;
        hits[nh++] = s.bvhValA[leaf];
        return true;
    });
    if (!complete || !room) return false;
    for (uint32_t a = 1; a < nh; ++a) { // insertion sort: a handful of hits
        const uint32_t v = hits[a];
        uint32_t b = a;
        while (b > 0u && hits[b - 1] > v) {
            hits[b] = hits[b - 1];
            --b;
        }
        hits[b] = v;
    }
    return true;
}

template <bool kEmit>
__device__ uint32_t fluidBoundaryListFor(const Scene &s, uint32_t p, f3 pos, uint32_t *out, uint32_t room)
{
    const float pr = mx(s.radii[p], 0.0f);
    const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[p]];
    const float support = mx(fm.smoothing_radius, pr);
    const float reuse = mx(mx(fm.cfl_radius, pr), support);
    const float qr = support + reuse;
    const f3 qmin = pos - f3{qr, qr, qr}, qmax = pos + f3{qr, qr, qr};
    const uint4 m = s.meta[p];
    uint32_t count = 0;
    auto consider = [&](uint32_t k) {
        const uint32_t c = s.colQueryOrder[k];
        if (!aabbOverlaps(qmin, qmax, xyz(s.colAabbMin[c]), xyz(s.colAabbMax[c]))) return;
        const cn_collider_broadphase bp = s.colBp[c];
        const uint32_t bt = s.bodyType[bp.owner_body];
        if (bp.enabled_flag != 0u && bp.environment_index == m.x && bt != CN_BODY_DYNAMIC &&
            (m.w & bp.collision_layer) != 0u && (bp.collision_mask & m.z) != 0u) {
            if (kEmit && count < room) out[count] = k;
            ++count;
        }
    };
    uint32_t hits[kCandidateHits], nh = 0;
    if (s.colBvh && s.colQueryCount >= 2u && bvhOverlaps(s, qmin, qmax, hits, nh)) {
        for (uint32_t i = 0; i < nh; ++i) consider(hits[i]);
    } else {
        for (uint32_t k = 0; k < s.colQueryCount; ++k) consider(k);
    }
    return count;
}

// kMode 0 counts the particle's candidate bodies, 1 emits its pairs from `write` (its offset
// after the count pass and the scan); both return the count.  Colliders are taken in query order
// (moving, then static): by a linear scan, or -- with many colliders and an LBVH this substep --
// from the tree's overlaps sorted back into query order, the same sequence.
template <uint32_t kMode>
__device__ __forceinline__ uint32_t rigidCandidatesAt(const Scene &s, uint32_t i, uint32_t write)
{
    const f3 p = xyz(s.x[i]);
    const float r = s.radii[i];
    const f3 qmin = p - f3{r, r, r}, qmax = p + f3{r, r, r};
    const uint4 m = s.meta[i];
    const uint32_t kind = s.kinds[i];
    const bool proxyOwner = s.ownerTypes[i] == CN_OWNER_RIGID_BODY;
    const uint32_t owner = s.ownerIdx[i];
    uint32_t seen[kRigidDedup];
    uint32_t seenCount = 0, count = 0;
    // one overlapping collider (query position k): filter, dedup by body, count / emit; false
    // when the emission buffer is full
    auto consider = [&](uint32_t k) -> bool {
        const uint32_t c = s.colQueryOrder[k];
        const cn_collider_broadphase bp = s.colBp[c];
        const uint32_t b = bp.owner_body;
        if (proxyOwner && b == owner) return true;
        const uint32_t bt = s.bodyType[b];
        if (!(bp.enabled_flag != 0u && bp.environment_index == m.x && (m.w & bp.collision_layer) != 0u &&
              (bp.collision_mask & m.z) != 0u && (kind == CN_PARTICLE_SOLID || bt == CN_BODY_DYNAMIC) &&
              s.bodyColRanges[b].y > 0u))
            return true;
        bool fresh = true;
        for (uint32_t q = 0; q < seenCount; ++q)
            if (seen[q] == b) { fresh = false; break; }
        if (!fresh) return true;
        if (seenCount < kRigidDedup) seen[seenCount++] = b;
        if (kMode != 0u) {
            if (write >= s.rigidPairCapacity) return false;
            s.rigidPairs[write++] = make_uint2(i, b);
        }
        ++count;
        return true;
    };
    if (s.rrCapacity != 0u && s.activeMovingCount != 0u && s.colQueryCount > kCandidateHits && !s.pColRange) {
        uint32_t hits[kCandidateHits], nh;
        if (bvhOverlaps(s, qmin, qmax, hits, nh)) {
            for (uint32_t j = 0; j < nh; ++j)
                if (!consider(hits[j])) break;
            return count;
        }
    }
    const uint2 cq = s.pColRange ? s.pColRange[i] : make_uint2(0u, s.colQueryCount);
    for (uint32_t k = cq.x; k < cq.y; ++k) {
        const uint32_t c = s.colQueryOrder[k];
        if (!aabbOverlaps(qmin, qmax, xyz(s.colAabbMin[c]), xyz(s.colAabbMax[c]))) continue;
        if (!consider(k)) break;
    }
    return count;
}

template <bool kEmit>
__global__ void __launch_bounds__(kThreads) k_rigidCandidates(Scene s, const uint32_t *total)
{
    if (kEmit && blockIdx.x == 0 && threadIdx.x == 0) {
        s.meta_->requiredRigidPairs = *total;
        s.meta_->rigidPairCount = min(*total, s.rigidPairCapacity);
    }
    forEachElem(s.wP, s.N, [&](uint32_t i) {
        if (!kEmit) {
            s.candCount[i] = rigidCandidatesAt<0u>(s, i, 0u);
        } else if (s.candCount[i] != 0u) {
            rigidCandidatesAt<1u>(s, i, s.candOffset[i]);
        }
    });
}

// ------------------------------------------------------------------------------------------
// Particle-particle candidate pairs (cross-body / self collision)
// physics_particle_count/emit_particle_particle_candidates.cs.hlsl,
// physics_particle_broad_phase_query.hlsli:50-117
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ bool isAdjacent(const Scene &s, uint32_t p, uint32_t c)
{
    const uint32_t o = s.adjOff[p], n = s.adjCnt[p];
    for (uint32_t k = 0; k < n; ++k)
        if (s.adjIdx[o + k] == c) return true;
    return false;
}

constexpr uint32_t kPairStageP = 8u; // staged particle-particle pairs per particle

template <bool kEmit>
__global__ void __launch_bounds__(kThreads) k_particleCandidates(Scene s, const uint32_t *total)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (kEmit && blockIdx.x == 0 && threadIdx.x == 0) {
        s.meta_->requiredParticlePairs = *total;
        s.meta_->particlePairCount = min(*total, s.particlePairCapacity);
    }
    if (i >= s.N) return;
    if (kEmit && s.ppCount[i] == 0u) return;
    // The count pass stages a particle's first kPairStageP pairs; the emit pass copies them to
    // their scanned offsets and walks again only for a particle with more.
    uint2 *stage = s.ppStage + size_t(i) * kPairStageP;
    if (kEmit && s.ppCount[i] <= kPairStageP) {
        uint32_t write = s.ppOffset[i];
        for (uint32_t k = 0; k < s.ppCount[i] && write < s.particlePairCapacity; ++k) s.particlePairs[write++] = stage[k];
        return;
    }
    const uint32_t kind = s.kinds[i];
    // Pairs go from the lower index up and fluid-fluid pairs are excluded: a fluid particle past
    // every solid (the world packs fluids last) has no candidate to walk for.
    if (!kEmit && kind == CN_PARTICLE_FLUID && i >= s.solidEnd) {
        s.ppCount[i] = 0u;
        return;
    }
    const int4 e = s.entries[i];
    const f3 pos = xyz(s.x[i]);
    const float r = s.radii[i];
    const uint4 m = s.meta[i];
    uint32_t count = 0;
    uint32_t write = kEmit ? s.ppOffset[i] : 0u;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int tx = e.x + dx, ty = e.y + dy, tz = e.z + dz;
                uint32_t start, end;
                bool mixed;
                if (!findRun(s, cellKey(tx, ty, tz), start, end, mixed)) continue;
                if (!mixed) {
                    const int4 ce = s.sCell[start];
                    if (ce.x != tx || ce.y != ty || ce.z != tz) continue;
                }
                for (uint32_t slot = start; slot < end; ++slot) {
                    if (mixed) {
                        const int4 ce = s.sCell[slot];
                        if (ce.x != tx || ce.y != ty || ce.z != tz) continue;
                    }
                    const uint32_t c = s.valsA[slot];
                    if (c <= i) continue;
                    // the filters are independent of one another: the distance test, which
                    // rejects most candidates, comes first, so the metadata loads and the
                    // adjacency scan run for the pairs in contact range only
                    const f3 op = xyz(s.x[c]);
                    const float cr = r + s.radii[c];
                    const f3 d = op - pos;
                    if (!(dot(d, d) <= cr * cr)) continue;
                    const uint4 om = s.meta[c];
                    if (om.x != m.x) continue;
                    if ((m.w & om.z) == 0u || (om.w & m.z) == 0u) continue;
                    const uint32_t ok = s.kinds[c];
                    if (kind == CN_PARTICLE_FLUID && ok == CN_PARTICLE_FLUID) continue;
                    if (kind == CN_PARTICLE_SOLID && ok == CN_PARTICLE_SOLID &&
                        (m.y & CN_PHASE_GROUP_MASK) == (om.y & CN_PHASE_GROUP_MASK)) {
                        const bool a = (m.y & CN_PHASE_SELF_COLLIDE) != 0u;
                        const bool b = (om.y & CN_PHASE_SELF_COLLIDE) != 0u;
                        if (!a || !b || isAdjacent(s, i, c)) continue;
                    }
                    if (kEmit) {
                        if (write >= s.particlePairCapacity) return;
                        s.particlePairs[write++] = make_uint2(i, c);
                    } else {
                        if (count < kPairStageP) stage[count] = make_uint2(i, c);
                        ++count;
                    }
                }
            }
    if (!kEmit) s.ppCount[i] = count;
}

// ------------------------------------------------------------------------------------------
// Fluid solve (cell order).
// ------------------------------------------------------------------------------------------
// Position of this fluid iteration: x + accumulated delta (iteration > 0), in sorted slots.
// With `P2` the first iteration writes a second copy: the other buffer of double-buffered
// positions (see k_fluidDeltaApplyClamp), so the tags of slots the iterations never rewrite are
// valid in each, or the superset build positions P0.  With `P0` (later iterations of a scene whose
// contacts also move fluid x) a particle's move is measured from P0, otherwise it is its
// accumulated delta.
__global__ void __launch_bounds__(kThreads) k_fluidGather(Scene s, float4 *Xs, const float4 *Dcur,
                                                          uint32_t iter, float4 *P2, const float4 *P0)
{
    pdlEnter();
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    float largest = 0.0f;
    if (slot < s.N) {
        const float4 xp = s.x[s.cvals[slot]];
        const f3 d = iter > 0 ? xyz(Dcur[slot]) : f3{0.f, 0.f, 0.f};
        const uint32_t info = s.sInfo[slot];
        const uint32_t tag = (info & 0x7fffffffu) | ((info & kFluidBit) && xp.w > kEps ? kFluidBit : 0u);
        const f3 p = xyz(xp) + d;
        Xs[slot] = xp;
        s.P[slot] = mk4(p, __uint_as_float(tag));
        if (P2) P2[slot] = mk4(p, __uint_as_float(tag));
        if (info & kFluidBit) {
            const f3 moved = P0 ? p - xyz(P0[slot]) : d;
            largest = sqrtf(dot(moved, moved));
        }
    }
    // largest move of this iteration: validity of the superset lists
    if (s.fluidMaxDelta && iter > 0 && iter < kMaxTrackedIterations) {
        for (int o = 16; o > 0; o >>= 1) largest = fmaxf(largest, __shfl_xor_sync(0xffffffffu, largest, o));
        if ((threadIdx.x & 31) == 0 && largest > 0.0f)
            atomicMax(&s.fluidMaxDelta[iter], __float_as_uint(largest));
    }
}

// physics_fluid_boundary_common.hlsli:11-83
__device__ bool fluidBoundaryContactInfo(const Scene &s, uint32_t c, f3 pos, float &sd, f3 &n)
{
    sd = 0.0f;
    n = f3{0.f, 1.f, 0.f};
    const float4 *fr = s.colFrame + size_t(c) * 4;
    const float4 f0 = __ldg(&fr[0]);
    const uint32_t word = __float_as_uint(f0.w);
    if ((word & 1u) == 0u) return false; // disabled collider
    const uint32_t shape = word >> 8;
    const f3 cwp = xyz(f0);
    if (shape == CN_COLLIDER_SPHERE) {
        const float r = __ldg(&fr[2].x);
        const f3 d = pos - cwp;
        const float dist = length(d);
        n = dist > kEps ? (d / dist) : f3{0.f, 1.f, 0.f};
        sd = dist - r;
    } else if (shape == CN_COLLIDER_BOX) {
        const float4 cwq = __ldg(&fr[1]);
        const f3 he = xyz(__ldg(&fr[2]));
        const f3 lp = qInvRotate(cwq, pos - cwp);
        const f3 cl = clamp3(lp, -he, he);
        const f3 d = lp - cl;
        const float dl = length(d);
        if (dl > kEps) {
            n = qRotate(cwq, d / dl);
            sd = dl;
        } else {
            const f3 ds = he - fabs3(lp);
            n = qRotate(cwq, closestFaceNormalLocal(lp, he));
            sd = -mn(ds.x, mn(ds.y, ds.z));
        }
    } else {
        const float4 e0 = __ldg(&fr[2]);
        const f3 a = xyz(e0), b2 = xyz(__ldg(&fr[3]));
        const float cr = e0.w;
        const f3 seg = b2 - a;
        const float l2 = dot(seg, seg);
        float t = 0.0f;
        if (l2 > kEps) t = saturate(dot(pos - a, seg) / l2);
        const f3 cl = lerp3(a, b2, t);
        const f3 d = pos - cl;
        const float dist = length(d);
        n = dist > kEps ? (d / dist) : f3{0.f, 1.f, 0.f};
        sd = dist - cr;
    }
    return true;
}

__device__ __forceinline__ bool fluidGhostDelta(const Scene &s, uint32_t c, f3 pos, float h, f3 &ghost)
{
    ghost = f3{0.f, 0.f, 0.f};
    float sd = 0.0f;
    f3 n{0.f, 1.f, 0.f};
    if (!fluidBoundaryContactInfo(s, c, pos, sd, n)) return false;
    if (sd < 0.0f || sd >= h) return false;
    ghost = n * (2.0f * sd);
    return true;
}

// Calls f(k) for every boundary candidate of compute slot `slot` (collider query positions k,
// ascending): from the mask, or from the slot's candidate list.
template <class F> __device__ __forceinline__ void forEachBoundary(const Scene &s, uint32_t slot, F &&f)
{
    if (!s.bList) {
        unsigned long long bm = s.sBoundary[slot];
        while (bm) {
            const uint32_t k = __ffsll(bm) - 1;
            bm &= bm - 1ull;
            f(k);
        }
    } else {
        const uint32_t off = s.bOffset[slot];
        const uint32_t n = s.bCount[slot];
        const uint32_t end = off + n < s.bListCap ? off + n : s.bListCap;
        for (uint32_t e = off; e < end; ++e) f(__ldg(&s.bList[e]));
    }
}
__device__ __forceinline__ bool hasBoundary(const Scene &s, uint32_t slot)
{
    return s.bList ? s.bCount[slot] != 0u : s.sBoundary[slot] != 0ull;
}

// Smallest float t with sqrtf(t) >= h: `length(d) >= h` (the reference's neighbour test) is exactly
// `dot(d, d) >= t` because the IEEE square root is correctly rounded and monotonic, so the square
// root is only taken for accepted neighbours.
__device__ __forceinline__ float sqrtThreshold(float h)
{
    float t = h * h;
    for (int k = 0; k < 4 && sqrtf(t) >= h; ++k) t = __uint_as_float(__float_as_uint(t) - 1u);
    for (int k = 0; k < 8 && sqrtf(t) < h; ++k) t = __uint_as_float(__float_as_uint(t) + 1u);
    return t;
}

// Candidate filter of physics_fluid_neighbor_build.hlsli:48-69 on the packed tag: fluid with
// invMass > kEps (bit 31), then environment / layer / mask.  Same-group candidates share the
// self particle's (environment, layer, mask), so the answer is the self-compatibility bit.
__device__ __forceinline__ bool neighborAllowed(const Scene &s, uint32_t tag, uint32_t myGroup, bool selfCompat,
                                                uint4 m, uint32_t c)
{
    if ((tag & kFluidBit) == 0u) return false;
    if ((tag & 0xffffu) == myGroup) return selfCompat;
    const uint4 om = __ldg(&s.sMeta[c]);
    return om.x == m.x && (m.w & om.z) != 0u && (om.w & m.z) != 0u;
}

// Neighbour list + density constraint.
// physics_fluid_build_neighbors.cs.hlsl:21-147 fused with
// physics_fluid_compute_density_lambda.cs.hlsl:26-115.  The density sum runs over the list in
// list order with the same distance values, so it equals the reference's second pass.
//
// mode 0: walk the 27 cells (runs from the per-run table of k_runNeighbors; a particle whose run
//         mixes several cells looks its runs up itself);
// mode 1: as mode 0, and also record every candidate within h * (1 + margin) ("superset", in
//         traversal order) for the later iterations of this substep;
// mode 3: record the superset only (no list, no density): the first iteration's list and density
//         then come from the mode 2 filter over it, which visits the same candidates in the same
//         order with the same distances, so the list and the sums are those of mode 1;
// mode 2: filter the superset instead of walking the cells.  Cells are fixed for the substep and
//         positions move only by the accumulated delta, so while 2 * max|delta| < margin * h every
//         neighbour of this iteration is in the superset, and filtering it in order yields exactly
//         the list the cell walk would build.  Otherwise (or if this particle's superset
//         overflowed) the particle walks the cells.
// One instantiation per mode, so the cell walk's register needs do not set the filter's occupancy;
// the filter is held to 64 registers (4 blocks of 256 per SM: 14 % faster than 65 registers and
// 3 blocks, measured; 48 registers and 5 blocks spill).
// With `Dk` (the accumulated delta this iteration starts from) the density constraint is also
// stored in Dk.w, so the delta kernel reads a neighbour's delta and constraint in one load.
// kExtras false: no fluid material has surface tension, so the colour-field normal is not summed
// (fewer live registers: the kernels then run at 5 blocks of 256 per SM without spills -- the
// filter 10 %, the superset build 5 % faster than the full build, measured).
template <uint32_t mode, bool kExtras>
__global__ void __launch_bounds__(kFluidThreads, (kExtras ? 4 : 5) * (256 / kFluidThreads)) k_fluidNeighborsDensity(Scene s, Config cfg, bool density,
                                                                                    uint32_t iter, float4 *Dk)
{
    pdlEnter();
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t info = s.sInfo[slot];
    if ((info & kFluidBit) == 0u) {
        if (density && mode != 3u) s.Cs[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 self = s.P[slot];
    if ((__float_as_uint(self.w) & kFluidBit) == 0u) { // invMass <= kEps
        if (mode == 1u || mode == 3u) s.supCount[slot] = 0u;
        if (mode == 3u) return;
        if (density) s.Cs[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.nbrCount[slot] = 0u;
        return;
    }
    const uint32_t maxN = s.maxNbr;
    const cn_fluid_material &fm = s.fluidMaterials[infoMaterial(info)];
    const float h = mx(fm.smoothing_radius, 1.0e-4f);
    const float h2 = sqrtThreshold(h);
    const float kW = spikyK(h);
    const float invH = 1.0f / h;
    const float st = kExtras ? mx(fm.surface_tension, 0.0f) : 0.0f;
    const f3 sp = xyz(self);
    // Lists are interleaved (entry k of slot i at k * N + i): a warp's k-th entries share lines.
    uint32_t *out = kInterleavedLists ? s.nbr + slot : s.nbr + size_t(slot) * maxN;
    const size_t lstr = kInterleavedLists ? size_t(s.N) : 1u;
    uint32_t count = 0, truncated = 0;
    float rho = 0.0f;
    f3 normal{0.f, 0.f, 0.f};

    bool useSuperset = false;
    if (mode == 2u) {
        const float maxDelta = __uint_as_float(s.fluidMaxDelta[iter < kMaxTrackedIterations ? iter : 0u]);
        useSuperset = iter < kMaxTrackedIterations && 2.0f * maxDelta < 0.99f * s.supMargin * h &&
                      s.supCount[slot] <= s.supCap;
    }
    if (useSuperset) {
        const uint32_t n = s.supCount[slot];
        const uint32_t *sup = kInterleavedLists ? s.sup + slot : s.sup + size_t(slot) * s.supCap;
        // Four entries in flight: their list words, then their positions, load before any is
        // used (the loop is bound by gather latency); they are consumed in list order.
        for (uint32_t k = 0; k < n; k += 4u) {
            uint32_t cc[4];
            float4 qq[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) cc[j] = (k + j < n) ? __ldcs(&sup[(k + j) * lstr]) : slot;
#pragma unroll
            for (int j = 0; j < 4; ++j) qq[j] = ld4(&s.P[cc[j]]);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (k + j >= n) break;
                const f3 delta = sp - xyz(qq[j]);
                const float d2 = dot(delta, delta);
                if (d2 >= h2) continue;
                if (count >= maxN) { truncated = 1; continue; }
                out[count++ * lstr] = cc[j];
                if (density) {
                    const float dist = sqrtf(d2);
                    rho += spikyWk(dist, h, invH, kW);
                    if (kExtras && st > kEps) normal += spikyGradK(delta, dist, h, invH, kW);
                }
            }
        }
    } else {
        const uint4 m = s.sMeta[slot];
        const uint32_t myGroup = infoGroup(info);
        const bool selfCompat = (m.w & m.z) != 0u;
        const int4 e = s.cCell[slot];
        const bool buildSup = mode == 1u || mode == 3u;
        const float supR = h * (1.0f + s.supMargin);
        const float sup2 = supR * supR;
        const float rec2 = buildSup ? (sup2 > h2 ? sup2 : h2) : h2;
        uint32_t *sup = buildSup ? (kInterleavedLists ? s.sup + slot : s.sup + size_t(slot) * s.supCap) : nullptr;
        uint32_t supN = 0;
        const uint32_t run = s.cRun[slot];
        const uint32_t runStart = s.runStartOf[run];
        const bool ownLookups = (runStart >> 31) != 0u;
        const uint2 *ranges = s.runNbr + size_t(run) * 27u;
        int k = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx, ++k) {
                    const int tx = e.x + dx, ty = e.y + dy, tz = e.z + dz;
                    uint32_t start, end;
                    bool check;
                    if (!ownLookups) {
                        const uint2 rg = __ldg(&ranges[k]);
                        start = rg.x & 0x7fffffffu;
                        end = rg.y;
                        check = (rg.x >> 31) != 0u;
                    } else {
                        bool mixed;
                        if (!findRunCompute(s, cellKey(tx, ty, tz), start, end, mixed)) continue;
                        check = true;
                    }
                    // A candidate beyond the recording radius (the superset's, else h; the superset's
                    // is the larger) records nothing whatever its filter says, so the distance test
                    // comes first; mixed runs also check the candidate's cell.
                    auto visit = [&](uint32_t c, const float4 &q) {
                        const f3 delta = sp - xyz(q);
                        const float d2 = dot(delta, delta);
                        if (d2 >= rec2) return;
                        if (c == slot || !neighborAllowed(s, __float_as_uint(q.w), myGroup, selfCompat, m, c)) return;
                        if (buildSup) {
                            if (supN < s.supCap) __stcs(&sup[supN * lstr], c); // written once, read later
                            ++supN;
                        }
                        if (mode == 3u || d2 >= h2) return;
                        if (count >= maxN) { truncated = 1; return; }
                        __stcs(&out[count++ * lstr], c);
                        if (density) {
                            const float dist = sqrtf(d2);
                            rho += spikyWk(dist, h, invH, kW);
                            if (kExtras && st > kEps) normal += spikyGradK(delta, dist, h, invH, kW);
                        }
                    };
                    if (!check) { // two candidates' positions in flight, visited in order
                        uint32_t c = start;
                        for (; c + 1u < end; c += 2u) {
                            const float4 q0 = ld4(&s.P[c]), q1 = ld4(&s.P[c + 1u]);
                            visit(c, q0);
                            visit(c + 1u, q1);
                        }
                        if (c < end) visit(c, ld4(&s.P[c]));
                    } else {
                        for (uint32_t c = start; c < end; ++c) {
                            const int4 ce = __ldg(&s.cCell[c]);
                            if (ce.x != tx || ce.y != ty || ce.z != tz) continue;
                            visit(c, ld4(&s.P[c]));
                        }
                    }
                }
        if (buildSup) s.supCount[slot] = supN; // > supCap marks an overflowed superset
        if (mode == 3u) return;
    }
    s.nbrCount[slot] = count;
    if (truncated) atomicAdd(&s.meta_->neighborTruncations, 1u);
    if (!density) return;
    forEachBoundary(s, slot, [&](uint32_t kk) {
        f3 ghost;
        if (!fluidGhostDelta(s, s.colQueryOrder[kk], sp, h, ghost)) return;
        const float dist = length(ghost);
        if (dist >= h) return;
        rho += spikyWk(dist, h, invH, kW) * cfg.fluidBoundaryDensityScale;
    });
    const float rho0 = mx(fm.rest_density, 1.0f);
    const float C = mx(rho - rho0, -rho0 * mx(cfg.fluidMaxUnderDensityRatio, 0.0f)) * fm.density_constraint_scale;
    if (kExtras && st > kEps) {
        normal = normal * st;
        s.Cs[slot] = mk4(normal, C);
    } else {
        s.Cs[slot] = make_float4(0.f, 0.f, 0.f, C);
    }
    if (Dk) reinterpret_cast<float *>(Dk + slot)[3] = C;
}

// Position delta, apply and boundary clamp.
// physics_fluid_compute_delta_positions.cs.hlsl:27-157, physics_fluid_apply_delta_positions.cs.hlsl:11-31,
// physics_fluid_clamp_boundary.cs.hlsl:23-80.  Reads the accumulated delta of iteration k (Dcur)
// and writes that of iteration k+1 (Dnext), so the neighbours' deltas stay those of iteration k.
//
// With `Pnext` (fluid x fixed over the iterations: no particle-particle contacts) the kernel also
// writes the next iteration's position x + accumulated delta -- what k_fluidGather would compute
// -- into the other position buffer, and records the largest accumulated delta for the superset
// test of the next iteration, so the gather runs once per substep.
//
// kExtras false: no fluid material of the scene has cohesion or surface tension, so those terms
// are zero for every pair and the kernel is built without them (fewer live registers).
template <bool kExtras>
__global__ void __launch_bounds__(kFluidThreads, (kExtras ? 4 : 5) * (256 / kFluidThreads)) k_fluidDeltaApplyClamp(Scene s, Config cfg, const float4 *Xs,
                                                                   const float4 *Dcur, float4 *Dnext,
                                                                   uint32_t iter, float dt, bool writeDx,
                                                                   float4 *Pnext)
{
    pdlEnter();
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t info = s.sInfo[slot];
    if ((info & kFluidBit) == 0u) {
        if (writeDx) s.Dx[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 self = s.P[slot];
    const f3 sdl = iter > 0 ? xyz(Dcur[slot]) : f3{0.f, 0.f, 0.f};
    const uint32_t myMat = infoMaterial(info);
    const cn_fluid_material &fm = s.fluidMaterials[myMat];
    f3 packed{0.f, 0.f, 0.f};
    float weight = 0.0f;
    if (__float_as_uint(self.w) & kFluidBit) {
        const f3 sp = xyz(self);
        const float4 snc = s.Cs[slot];
        const float sC = snc.w;
        const float h = mx(fm.smoothing_radius, 1.0e-4f);
        const float kW = spikyK(h);
        const float invH = 1.0f / h;
        const float cohesion = kExtras ? dt * mx(fm.cohesion, 0.0f) : 0.0f;
        const float visc = dt * mx(fm.viscosity, 0.0f);
        const float st = kExtras ? mx(fm.surface_tension, 0.0f) : 0.0f;
        const float cfl = mx(fm.cfl_radius, 0.0f);
        const bool needRel = visc > kEps || cfl > kEps;
        const f3 sn = st > kEps ? xyz(snc) : f3{0.f, 0.f, 0.f};
        f3 dp{0.f, 0.f, 0.f};
        const uint32_t cnt = s.nbrCount[slot];
        // 32-bit list offsets (N x max neighbours < 2^32 is checked at sync)
        const uint32_t *lst = kInterleavedLists ? s.nbr + slot : s.nbr + size_t(slot) * s.maxNbr;
        const uint32_t lstr = kInterleavedLists ? s.N : 1u;
        // Software-pipelined over the list: the next neighbour's slot, position word, constraint
        // and accumulated delta are in flight while the current pair term is computed.
        // A neighbour's accumulated delta (xyz, used from the second iteration on) and density
        // constraint (w, stored there by the density kernel) come in one load.
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t cN = cnt > 0 ? __ldcs(&lst[0]) : 0u; // list words are read once: streaming loads
        uint32_t cNN = cnt > 1 ? __ldcs(&lst[lstr]) : 0u;
        float4 npN = cnt > 0 ? ld4(&s.P[cN]) : zero4;
        float4 dN = cnt > 0 ? ld4(&Dcur[cN]) : zero4;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t c = cN;
            const float4 np = npN;
            const float ncw = dN.w;
            const float4 nd4 = dN;
            if (k + 1 < cnt) {
                cN = cNN;
                if (k + 2 < cnt) cNN = __ldcs(&lst[(k + 2) * lstr]);
                npN = ld4(&s.P[cN]);
                dN = ld4(&Dcur[cN]);
            }
            const uint32_t tag = __float_as_uint(np.w);
            if ((tag & kFluidBit) == 0u) continue;
            const f3 delta = sp - xyz(np);
            const float dist = length(delta);
            if (dist >= h || dist <= kEps) continue;
            const f3 nij = delta * (1.0f / dist);
            // spikyDW / spikyW of physics_fluid_common.hlsli:17-41 sharing 1 - dist / h
            const float om = 1.0f - dist * invH;
            const float dw = -2.0f * kW * om * invH;
            f3 pd = -0.5f * (sC + ncw) * dw * nij;
            if (infoMaterial(tag) == myMat) {
                if (kExtras && cohesion > kEps)
                    pd -= nij * (cohesion * cohesionW(dist, h, invH, fm.cohesion1, fm.cohesion2));
                if (needRel) {
                    const f3 nd = iter > 0 ? xyz(nd4) : f3{0.f, 0.f, 0.f};
                    const f3 rel = sdl - nd;
                    if (visc > kEps) {
                        const float vs = 1.0f - (1.0f / (1.0f + visc * (kW * om * om)));
                        pd -= vs * rel;
                    }
                    if (cfl > kEps) {
                        const float proj = dot(rel, nij);
                        if (proj < -cfl) pd -= nij * (proj + cfl) * 0.5f;
                    }
                }
                if (kExtras && st > kEps) pd -= dt * (sn - xyz(ld4(&s.Cs[c])));
            }
            dp += pd;
            weight += 1.0f;
        }
        f3 bd{0.f, 0.f, 0.f};
        forEachBoundary(s, slot, [&](uint32_t k) {
            f3 ghost;
            if (!fluidGhostDelta(s, s.colQueryOrder[k], sp, h, ghost)) return;
            const float dist = length(ghost);
            if (dist <= kEps || dist >= h) return;
            const f3 nij = ghost * (1.0f / dist);
            const float dw = spikyDWk(dist, h, invH, kW);
            bd += -mx(sC, 0.0f) * dw * nij;
        });
        bd = bd * cfg.fluidBoundaryDeltaScale;
        packed = dp * cfg.fluidSolveCoefficient + bd;
    }
    if (writeDx) s.Dx[slot] = mk4(packed, weight);
    // apply (physics_fluid_apply_delta_positions.cs.hlsl:21-30)
    const float w = mx(weight * cfg.fluidRelaxation, 1.0f);
    const f3 d = packed / w;
    const f3 acc = sdl + d;
    // clamp (physics_fluid_clamp_boundary.cs.hlsl:36-79)
    const f3 base = xyz(Xs[slot]);
    f3 cur = base + acc;
    if (hasBoundary(s, slot)) {
        const uint32_t p = s.cvals[slot];
        const float pr = mx(s.radii[p], 0.0f);
        for (uint32_t sweep = 0; sweep < 2u; ++sweep) {
            bool changed = false;
            forEachBoundary(s, slot, [&](uint32_t k) {
                float sd = 0.0f;
                f3 n{0.f, 1.f, 0.f};
                if (!fluidBoundaryContactInfo(s, s.colQueryOrder[k], cur, sd, n)) return;
                if (sd >= pr) return;
                cur += n * (pr - sd);
                changed = true;
            });
            if (!changed) break;
        }
    }
    const f3 dn = cur - base;
    Dnext[slot] = mk4(dn, 0.0f);
    if (Pnext) {
        Pnext[slot] = mk4(base + dn, self.w);
        const uint32_t next = iter + 1u;
        if (next < kMaxTrackedIterations) {
            // lanes that returned early are not in the mask; diverged groups reduce separately
            const unsigned mask = __activemask();
            const uint32_t big = __reduce_max_sync(mask, __float_as_uint(sqrtf(dot(dn, dn))));
            if (int(threadIdx.x & 31u) == __ffs(mask) - 1 && big > 0u) atomicMax(&s.fluidMaxDelta[next], big);
        }
    }
}

// Vorticity confinement over the lists of the post-update rebuild, in compute order (positions in
// s.P after the velocity update, velocities in particle order).
// physics_fluid_compute_vorticity.cs.hlsl:13-76: curl of the velocity field from same-material
// neighbours, with its magnitude in w.
__global__ void __launch_bounds__(kThreads) k_fluidVorticity(Scene s)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t info = s.sInfo[slot];
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 self = s.P[slot];
    const cn_fluid_material &fm = s.fluidMaterials[infoMaterial(info)];
    if ((info & kFluidBit) && mx(fm.vorticity_confinement, 0.0f) > kEps && (__float_as_uint(self.w) & kFluidBit)) {
        const f3 sp = xyz(self), sv = xyz(s.v[s.cvals[slot]]);
        const float h = mx(fm.smoothing_radius, 1.0e-4f);
        const float kW = spikyK(h), invH = 1.0f / h;
        const uint32_t mat = infoMaterial(info);
        f3 curl{0.f, 0.f, 0.f};
        const uint32_t cnt = s.nbrCount[slot];
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t c = s.nbr[size_t(k) * s.N + slot];
            const float4 q = s.P[c];
            if (infoMaterial(__float_as_uint(q.w)) != mat) continue;
            const f3 delta = sp - xyz(q);
            const float dist = length(delta);
            if (dist <= kEps || dist >= h) continue;
            curl += cross(xyz(s.v[s.cvals[c]]) - sv, spikyGradK(delta, dist, h, invH, kW));
        }
        out = mk4(curl, length(curl));
    }
    s.fluidVort[slot] = out;
}

// physics_fluid_apply_vorticity_confinement.cs.hlsl:13-92: the confinement force along the
// gradient of the curl magnitude, added to the particle's velocity (w cleared).
__global__ void __launch_bounds__(kThreads) k_fluidVorticityApply(Scene s, float dt)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    const uint32_t info = s.sInfo[slot];
    if ((info & kFluidBit) == 0u) return;
    const cn_fluid_material &fm = s.fluidMaterials[infoMaterial(info)];
    const float conf = mx(fm.vorticity_confinement, 0.0f);
    if (conf <= kEps) return;
    const float4 self = s.P[slot];
    if ((__float_as_uint(self.w) & kFluidBit) == 0u) return;
    const float4 sc = s.fluidVort[slot];
    if (sc.w <= kEps) return;
    const f3 sp = xyz(self);
    const float h = mx(fm.smoothing_radius, 1.0e-4f);
    const float kW = spikyK(h), invH = 1.0f / h;
    const uint32_t mat = infoMaterial(info);
    f3 grad{0.f, 0.f, 0.f};
    const uint32_t cnt = s.nbrCount[slot];
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t c = s.nbr[size_t(k) * s.N + slot];
        const float4 q = s.P[c];
        if (infoMaterial(__float_as_uint(q.w)) != mat) continue;
        const f3 delta = sp - xyz(q);
        const float dist = length(delta);
        if (dist <= kEps || dist >= h) continue;
        grad += s.fluidVort[c].w * spikyGradK(delta, dist, h, invH, kW);
    }
    const float gl = length(grad);
    if (gl <= kEps) return;
    const f3 force = conf * cross(grad / gl, xyz(sc));
    const uint32_t p = s.cvals[slot];
    s.v[p] = mk4(xyz(s.v[p]) + dt * force, 0.0f);
}

// ------------------------------------------------------------------------------------------
// XPBD families: Jacobi solve writes per-constraint records, apply gathers them per particle in
// ascending constraint order (the reference's incidence order).
// ------------------------------------------------------------------------------------------
// A constraint's correction record for one of its particles goes to that particle's gather slot
// (kNoSlot: the entry names no particle, e.g. slot 3 of a 3-point bend).
constexpr uint32_t kNoSlot = 0xffffffffu;
__device__ __forceinline__ void putRecord(float4 *corr, uint32_t slot, float4 v)
{
    if (slot != kNoSlot) corr[slot] = v;
}
__device__ __forceinline__ float4 recordAt(const float4 *corr, uint32_t slot)
{
    return slot != kNoSlot ? corr[slot] : make_float4(0.f, 0.f, 0.f, 0.f);
}

// physics_soft_solve_edge_constraints.cs.hlsl:10-74: one edge's corrections (zero when it is
// disabled or degenerate) and, when it returns true, its new lambda.
__device__ __forceinline__ bool edgeSolve(const Scene &s, float dt, float relax, const PackedEdge &ed, float lambda,
                                          float &newLambda, float4 &cA, float4 &cB)
{
    cA = make_float4(0.f, 0.f, 0.f, 0.f);
    cB = cA;
    if (ed.b >> 31) return false; // disabled
    const float4 a = s.x[ed.a], b = s.x[ed.b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    const f3 delta = xyz(b) - xyz(a);
    const float l2 = dot(delta, delta);
    if (!(wSum > kEps && l2 > kEps)) return false;
    const float len = sqrtf(l2);
    const f3 gA = -delta / len;
    const f3 gB = -gA;
    const float alpha = mx(ed.compliance, 0.0f) / mx(dt * dt, kEps);
    const float Cv = len - ed.rest;
    const float den = wSum + alpha;
    if (!(den > kEps)) return false;
    const float dl = -(Cv + alpha * lambda) / den;
    newLambda = lambda + dl;
    cA = mk4(wA * dl * gA * relax, 0.0f);
    cB = mk4(wB * dl * gB * relax, 0.0f);
    return true;
}

__device__ __forceinline__ void solveEdge(const Scene &s, float dt, float relax, uint32_t e)
{
    const PackedEdge ed = s.edgesP ? s.edgesP[e] : packEdge(s.edges[e]);
    const float lambda = s.edgeLambda[e]; // with the record: one round trip fewer
    float newLambda;
    float4 cA, cB;
    if (edgeSolve(s, dt, relax, ed, lambda, newLambda, cA, cB)) s.edgeLambda[e] = newLambda;
    const uint2 d = reinterpret_cast<const uint2 *>(s.edgeDst)[e];
    putRecord(s.edgeCorr, d.x, cA);
    putRecord(s.edgeCorr, d.y, cB);
}

__global__ void __launch_bounds__(kThreads) k_solveEdges(Scene s, float dt, float relax)
{
    pdlEnter();
    forEachElem(s.wE, s.E, [&](uint32_t e) { solveEdge(s, dt, relax, e); });
}

// Gather of the correction records: each particle's records sit contiguously at its incidence
// range, in ascending constraint order (the solves write each record to its gather slot), and are
// fetched kGatherBatch at a time before they are summed in list order -- the one-at-a-time sum,
// with the range and the records as the only dependent loads.
constexpr uint32_t kGatherBatch = 8u;

// x + the particle's records summed in list order (x itself for a particle without weight).
__device__ __forceinline__ float4 gatheredPosition(const uint2 *ranges, const float4 *corr, uint32_t i, const float4 p)
{
    const uint2 r = ranges[i];
    if (p.w <= kEps) return p;
    f3 total{0.f, 0.f, 0.f};
    for (uint32_t k = 0; k < r.y; k += kGatherBatch) {
        float4 c[kGatherBatch];
#pragma unroll
        for (uint32_t j = 0; j < kGatherBatch; ++j)
            if (k + j < r.y) c[j] = corr[r.x + k + j];
#pragma unroll
        for (uint32_t j = 0; j < kGatherBatch; ++j)
            if (k + j < r.y) total += xyz(c[j]);
    }
    return mk4(xyz(p) + total, p.w);
}

__device__ __forceinline__ void applyGatherAt(const Scene &s, const uint2 *ranges, const float4 *corr, uint32_t i)
{
    const float4 p = s.x[i];
    if (p.w > kEps) s.x[i] = gatheredPosition(ranges, corr, i, p);
}

// physics_soft_apply_edge_corrections.cs.hlsl:9-35, physics_soft_apply_tet_corrections.cs.hlsl:9-50,
// physics_soft_apply_bend_corrections.cs.hlsl:9-51, physics_strand_apply_distance_corrections.cs.hlsl:9-38.
// A single world applies over `win`, the particles [lo, hi) that the family touches (bodies are
// contiguous in the particle order; the others have no records and keep x); a batch over its tiles.
__global__ void __launch_bounds__(kThreads) k_applyGather(Scene s, const uint2 *ranges, const float4 *corr, uint2 win)
{
    pdlEnter();
    if (s.wP.tiles) {
        forEachElem(s.wP, s.N, [&](uint32_t i) { applyGatherAt(s, ranges, corr, i); });
        return;
    }
    const uint32_t i = win.x + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < win.y) applyGatherAt(s, ranges, corr, i);
}

// physics_soft_solve_tet_constraints.cs.hlsl:15-87: one tet's four corrections and its new
// lambda; false when the tet keeps its previous corrections (no weight, or a degenerate one).
__device__ __forceinline__ bool tetSolve(const Scene &s, float dt, float relax, const cn_soft_tet &tet, float lambda,
                                         float &newLambda, float4 c[4])
{
    const float4 q0 = s.x[tet.particle_indices[0]], q1 = s.x[tet.particle_indices[1]];
    const float4 q2 = s.x[tet.particle_indices[2]], q3 = s.x[tet.particle_indices[3]];
    const float w0 = q0.w, w1 = q1.w, w2 = q2.w, w3 = q3.w;
    if ((w0 + w1 + w2 + w3) <= kEps) return false;
    const f3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2), p3 = xyz(q3);
    const float sv = dot(cross(p1 - p0, p2 - p0), p3 - p0) / 6.0f;
    const float vs = (sv >= 0.0f) ? 1.0f : -1.0f;
    const float Cv = fabsf(sv) - mx(tet.rest_volume, 0.0f);
    const f3 g0 = cross(p3 - p1, p2 - p1) * (vs / 6.0f);
    const f3 g1 = cross(p2 - p0, p3 - p0) * (vs / 6.0f);
    const f3 g2 = cross(p3 - p0, p1 - p0) * (vs / 6.0f);
    const f3 g3 = cross(p1 - p0, p2 - p0) * (vs / 6.0f);
    const float sg = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2) + w3 * dot(g3, g3);
    const float alpha = mx(tet.compliance, 0.0f) / mx(dt * dt, kEps);
    const float den = sg + alpha;
    if (den <= kEps) return false;
    const float dl = -(Cv + alpha * lambda) / den;
    newLambda = lambda + dl;
    c[0] = mk4(w0 * dl * g0 * relax, 0.0f);
    c[1] = mk4(w1 * dl * g1 * relax, 0.0f);
    c[2] = mk4(w2 * dl * g2 * relax, 0.0f);
    c[3] = mk4(w3 * dl * g3 * relax, 0.0f);
    return true;
}

__device__ __forceinline__ void solveTet(const Scene &s, float dt, float relax, uint32_t t)
{
    const cn_soft_tet tet = s.tets[t];
    const float lambda = s.tetLambda[t]; // with the record: one round trip fewer
    float newLambda;
    float4 c[4];
    if (!tetSolve(s, dt, relax, tet, lambda, newLambda, c)) return; // keeps the previous records
    s.tetLambda[t] = newLambda;
    const uint4 d = reinterpret_cast<const uint4 *>(s.tetDst)[t];
    putRecord(s.tetCorr, d.x, c[0]);
    putRecord(s.tetCorr, d.y, c[1]);
    putRecord(s.tetCorr, d.z, c[2]);
    putRecord(s.tetCorr, d.w, c[3]);
}

__global__ void __launch_bounds__(kThreads) k_solveTets(Scene s, float dt, float relax)
{
    pdlEnter();
    forEachElem(s.wT, s.T, [&](uint32_t t) { solveTet(s, dt, relax, t); });
}

// physics_soft_solve_bend_constraints.cs.hlsl:20-86
__device__ __forceinline__ void solveBendAt(const Scene &s, float dt, float relax, uint32_t b)
{
    const cn_soft_bend bd = s.bends[b];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 o0 = z, o1 = z, o2 = z;
    const float4 q0 = s.x[bd.particle0], q1 = s.x[bd.particle1], q2 = s.x[bd.particle2];
    const float w0 = q0.w, w1 = q1.w, w2 = q2.w;
    const f3 e0 = xyz(q0) - xyz(q1), e1 = xyz(q2) - xyz(q1);
    const float l0s = dot(e0, e0), l1s = dot(e1, e1);
    if (w0 + w1 + w2 > kEps && l0s > kEps && l1s > kEps) {
        const float l0 = sqrtf(l0s), l1 = sqrtf(l1s);
        const f3 d0 = e0 / l0, d1 = e1 / l1;
        const float ct = mn(mx(dot(d0, d1), -1.0f + 1.0e-4f), 1.0f - 1.0e-4f);
        const float st2 = mx(1.0f - ct * ct, 1.0e-8f);
        const float st = sqrtf(st2);
        const float theta = acosf(ct);
        const f3 g0 = -(d1 - ct * d0) / mx(l0 * st, kEps);
        const f3 g2 = -(d0 - ct * d1) / mx(l1 * st, kEps);
        const f3 g1 = -(g0 + g2);
        const float den = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2);
        const float alpha = mx(bd.compliance, 0.0f) / mx(dt * dt, kEps);
        if (den + alpha > kEps) {
            const float Cv = theta - bd.rest_angle;
            const float lambda = s.bendLambda[b];
            const float dl = -(Cv + alpha * lambda) / (den + alpha);
            s.bendLambda[b] = lambda + dl;
            o0 = mk4(w0 * dl * g0 * relax, 0.0f);
            o1 = mk4(w1 * dl * g1 * relax, 0.0f);
            o2 = mk4(w2 * dl * g2 * relax, 0.0f);
        }
    }
    const uint4 d = reinterpret_cast<const uint4 *>(s.bendDst)[b];
    putRecord(s.bendCorr, d.x, o0);
    putRecord(s.bendCorr, d.y, o1);
    putRecord(s.bendCorr, d.z, o2);
    putRecord(s.bendCorr, d.w, z);
}

__global__ void __launch_bounds__(kThreads) k_solveBends(Scene s, float dt, float relax)
{
    pdlEnter();
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < s.Bn) solveBendAt(s, dt, relax, b);
}

// physics_cloth_solve_dihedral_constraints.cs.hlsl:20-95
__device__ __forceinline__ void solveDihedralAt(const Scene &s, float dt, float relax, uint32_t d)
{
    const uint32_t ci = s.Bn + d;
    const cn_cloth_dihedral h = s.dihedrals[d];
    const uint4 dst = reinterpret_cast<const uint4 *>(s.bendDst)[ci];
    auto put4 = [&](float4 a, float4 b, float4 c, float4 e) {
        putRecord(s.bendCorr, dst.x, a);
        putRecord(s.bendCorr, dst.y, b);
        putRecord(s.bendCorr, dst.z, c);
        putRecord(s.bendCorr, dst.w, e);
    };
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 e0m = s.x[h.edge_particle0], e1m = s.x[h.edge_particle1];
    const float4 o0m = s.x[h.opposite_particle0], o1m = s.x[h.opposite_particle1];
    const f3 p0 = xyz(o0m), p1 = xyz(o1m), p2 = xyz(e0m), p3 = xyz(e1m);
    const f3 edge = p3 - p2;
    const float el2 = dot(edge, edge);
    const f3 rn0 = cross(p2 - p0, p3 - p0);
    const f3 rn1 = cross(p3 - p1, p2 - p1);
    const float n0s = dot(rn0, rn0), n1s = dot(rn1, rn1);
    if (el2 <= kEps || n0s <= kEps || n1s <= kEps) {
        put4(z, z, z, z);
        return;
    }
    const float el = sqrtf(el2);
    const float iel = 1.0f / el;
    const f3 sn0 = rn0 / n0s, sn1 = rn1 / n1s;
    const f3 dO0 = el * sn0, dO1 = el * sn1;
    const f3 dE0 = dot(p0 - p3, edge) * iel * sn0 + dot(p1 - p3, edge) * iel * sn1;
    const f3 dE1 = dot(p2 - p0, edge) * iel * sn0 + dot(p2 - p1, edge) * iel * sn1;
    const f3 g0 = -dE0, g1 = -dE1, g2 = -dO0, g3 = -dO1;
    const f3 n0 = rn0 / sqrtf(n0s), n1 = rn1 / sqrtf(n1s);
    const float theta = atan2f(dot(edge * iel, cross(n0, n1)), mn(mx(dot(n0, n1), -1.0f), 1.0f));
    const float twoPi = 6.283185307179586f;
    float Cv = theta - h.rest_angle;
    Cv = Cv - twoPi * floorf((Cv + 3.141592653589793f) / twoPi);
    const float w0 = e0m.w, w1 = e1m.w, w2 = o0m.w, w3 = o1m.w;
    const float den = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2) + w3 * dot(g3, g3);
    const float alpha = mx(h.compliance, 0.0f) / mx(dt * dt, kEps);
    if (den + alpha <= kEps) {
        put4(z, z, z, z);
        return;
    }
    const float lambda = s.bendLambda[ci];
    const float dl = -(Cv + alpha * lambda) / (den + alpha);
    s.bendLambda[ci] = lambda + dl;
    put4(mk4(w0 * dl * g0 * relax, 0.0f), mk4(w1 * dl * g1 * relax, 0.0f), mk4(w2 * dl * g2 * relax, 0.0f),
         mk4(w3 * dl * g3 * relax, 0.0f));
}

__global__ void __launch_bounds__(kThreads) k_solveDihedrals(Scene s, float dt, float relax)
{
    pdlEnter();
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < s.D) solveDihedralAt(s, dt, relax, d);
}

// 3x3 helpers of physics_strand_solve_{segment,joint}_constraints.cs.hlsl:12-64
struct m3 { float m[3][3]; };
__device__ __forceinline__ void addOuter(m3 &acc, float sc, f3 a, f3 b)
{
    const float o[3][3] = {{a.x * b.x, a.x * b.y, a.x * b.z}, {a.y * b.x, a.y * b.y, a.y * b.z},
                           {a.z * b.x, a.z * b.y, a.z * b.z}};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc.m[r][c] = acc.m[r][c] + sc * o[r][c];
}
__device__ __forceinline__ f3 solve3(const m3 &M, f3 v)
{
    const float a00 = M.m[0][0], a01 = M.m[0][1], a02 = M.m[0][2];
    const float a10 = M.m[1][0], a11 = M.m[1][1], a12 = M.m[1][2];
    const float a20 = M.m[2][0], a21 = M.m[2][1], a22 = M.m[2][2];
    const float c00 = a11 * a22 - a12 * a21, c01 = a02 * a21 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const float c10 = a12 * a20 - a10 * a22, c11 = a00 * a22 - a02 * a20, c12 = a02 * a10 - a00 * a12;
    const float c20 = a10 * a21 - a11 * a20, c21 = a01 * a20 - a00 * a21, c22 = a00 * a11 - a01 * a10;
    const float det = a00 * c00 + a01 * c10 + a02 * c20;
    if (fabsf(det) <= kEps) return f3{0.f, 0.f, 0.f} * v.x + f3{0.f, 0.f, 0.f}; // zero inverse
    const float id = 1.0f / det;
    const f3 r0{c00 * id, c01 * id, c02 * id}, r1{c10 * id, c11 * id, c12 * id}, r2{c20 * id, c21 * id, c22 * id};
    return f3{dot(r0, v), dot(r1, v), dot(r2, v)};
}
__device__ __forceinline__ float strandOrientationInvMass(float wA, float wB, float rl)
{
    const float ws = mx(wA + wB, 0.0f);
    if (ws <= kEps || rl <= kEps) return 0.0f;
    const float avg = ws * 0.5f;
    return 12.0f * avg / mx(rl * rl, kEps);
}

// physics_strand_solve_segment_constraints.cs.hlsl:66-147
__device__ __forceinline__ void solveSegmentAt(const Scene &s, float dt, float relax, uint32_t g)
{
    const cn_strand_segment sg = s.segs[g];
    const float4 a = s.x[sg.particle_a], b = s.x[sg.particle_b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 o0 = z, o1 = z, o2 = z;
    const f3 delta = xyz(b) - xyz(a);
    if (wSum > kEps && dot(delta, delta) > kEps) {
        const float4 q = qNormalize(s.segOrient[g]);
        const f3 axis = qRotate(q, f3{1.f, 0.f, 0.f});
        const float irl = 1.0f / mx(sg.rest_length, kEps);
        const float oim = strandOrientationInvMass(wA, wB, sg.rest_length);
        const f3 Cv = delta * irl - axis;
        const float alpha = mx(sg.stretch_shear_compliance, 0.0f) / mx(dt * dt, kEps);
        const f3 lambda = xyz(s.segLambda[g]);
        const f3 qv = xyz(q);
        const float qw = q.w;
        const f3 gQw = 2.0f * f3{qw, qv.z, -qv.y};
        const f3 gQx = 2.0f * f3{0.0f, qv.y, qv.z};
        const f3 gQy = 2.0f * f3{-qv.y, 0.0f, -qw};
        const f3 gQz = 2.0f * f3{-qv.z, qw, 0.0f};
        const float dg = wSum * irl * irl + alpha;
        m3 sys{{{dg, 0.f, 0.f}, {0.f, dg, 0.f}, {0.f, 0.f, dg}}};
        addOuter(sys, oim, gQx, gQx);
        addOuter(sys, oim, gQy, gQy);
        addOuter(sys, oim, gQz, gQz);
        addOuter(sys, oim, gQw, gQw);
        const f3 rhs = -(Cv + alpha * lambda);
        const f3 dl = solve3(sys, rhs);
        if (dot(dl, dl) > 0.0f) {
            s.segLambda[g] = mk4(lambda + dl, 0.0f);
            o0 = mk4(-wA * irl * dl * relax, 0.0f);
            o1 = mk4(wB * irl * dl * relax, 0.0f);
            o2 = scale4(make_float4(-dot(gQx, dl), -dot(gQy, dl), -dot(gQz, dl), -dot(gQw, dl)), oim * relax);
        }
    }
    float4 *out = s.segCorr + 3 * size_t(g);
    out[0] = o0; out[1] = o1; out[2] = o2;
}

__global__ void __launch_bounds__(kThreads) k_solveSegments(Scene s, float dt, float relax)
{
    pdlEnter();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < s.S) solveSegmentAt(s, dt, relax, g);
}

// physics_strand_apply_segment_corrections.cs.hlsl:11-43.  Thread i applies particle segWin.x + i
// of the segments' particle window (the others have no segment records) and renormalises
// segment i's orientation.
__device__ __forceinline__ void applySegmentsAt(const Scene &s, uint32_t t)
{
    const uint32_t i = s.segWin.x + t;
    if (i < s.segWin.y) {
        const float4 p = s.x[i];
        if (p.w > kEps) {
            const uint2 r = s.segRanges[i];
            f3 total{0.f, 0.f, 0.f};
            for (uint32_t k = 0; k < r.y; ++k) {
                const uint2 ref = s.segInc[r.x + k];
                total += xyz(s.segCorr[3 * ref.x + (ref.y == 0u ? 0u : 1u)]);
            }
            s.x[i] = mk4(xyz(p) + total, p.w);
        }
    }
    if (t < s.S) s.segOrient[t] = qNormalize(add4(s.segOrient[t], s.segCorr[3 * size_t(t) + 2]));
}
__host__ __device__ __forceinline__ uint32_t segmentApplyThreads(const Scene &s)
{
    const uint32_t w = s.segWin.y > s.segWin.x ? s.segWin.y - s.segWin.x : 0u;
    return w > s.S ? w : s.S;
}

__global__ void __launch_bounds__(kThreads) k_applySegments(Scene s)
{
    pdlEnter();
    applySegmentsAt(s, blockIdx.x * blockDim.x + threadIdx.x);
}

// physics_strand_solve_joint_constraints.cs.hlsl:66-154
__device__ __forceinline__ void solveJointAt(const Scene &s, float dt, float relax, uint32_t j)
{
    const cn_strand_joint jt = s.joints[j];
    const cn_strand_segment sA = s.segs[jt.segment_a], sB = s.segs[jt.segment_b];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 tA = z, tB = z;
    const float4 oA = qNormalize(s.segOrient[jt.segment_a]);
    const float4 oB = qNormalize(s.segOrient[jt.segment_b]);
    const float imA = strandOrientationInvMass(s.x[sA.particle_a].w, s.x[sA.particle_b].w, sA.rest_length);
    const float imB = strandOrientationInvMass(s.x[sB.particle_a].w, s.x[sB.particle_b].w, sB.rest_length);
    const float4 rel = qNormalize(qMul(qConj(oA), oB));
    float4 rr = qNormalize(make_float4(jt.rest_relative_orientation[0], jt.rest_relative_orientation[1],
                                       jt.rest_relative_orientation[2], jt.rest_relative_orientation[3]));
    if (dot4(rel, rr) < 0.0f) rr = make_float4(-rr.x, -rr.y, -rr.z, -rr.w);
    const f3 Cv = xyz(rel) - xyz(rr);
    const float4 lambda = s.jointLambda[j];
    const float ba = mx(jt.bend_compliance, 0.0f) / mx(dt * dt, kEps);
    const float ta = mx(jt.twist_compliance, 0.0f) / mx(dt * dt, kEps);
    const f3 av{ta, ba, ba};
    m3 sys{{{av.x, 0.f, 0.f}, {0.f, av.y, 0.f}, {0.f, 0.f, av.z}}};
    const f3 va = xyz(oA), vb = xyz(oB);
    const float wa = oA.w, wb = oB.w;
    const f3 gAX{-wb, vb.z, -vb.y}, gAY{-vb.z, -wb, vb.x}, gAZ{vb.y, -vb.x, -wb}, gAW = vb;
    const f3 gBX{wa, -va.z, va.y}, gBY{va.z, wa, -va.x}, gBZ{-va.y, va.x, wa}, gBW = -va;
    addOuter(sys, imA, gAX, gAX);
    addOuter(sys, imA, gAY, gAY);
    addOuter(sys, imA, gAZ, gAZ);
    addOuter(sys, imA, gAW, gAW);
    addOuter(sys, imB, gBX, gBX);
    addOuter(sys, imB, gBY, gBY);
    addOuter(sys, imB, gBZ, gBZ);
    addOuter(sys, imB, gBW, gBW);
    const f3 rhs = -(Cv + av * xyz(lambda));
    const f3 dl = solve3(sys, rhs);
    if (dot(dl, dl) > 0.0f) {
        s.jointLambda[j] = mk4(xyz(lambda) + dl, 0.0f);
        tA = scale4(make_float4(dot(gAX, dl), dot(gAY, dl), dot(gAZ, dl), dot(gAW, dl)), imA * relax);
        tB = scale4(make_float4(dot(gBX, dl), dot(gBY, dl), dot(gBZ, dl), dot(gBW, dl)), imB * relax);
    }
    s.jointCorr[2 * size_t(j)] = tA;
    s.jointCorr[2 * size_t(j) + 1] = tB;
}

__global__ void __launch_bounds__(kThreads) k_solveJoints(Scene s, float dt, float relax)
{
    pdlEnter();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < s.J) solveJointAt(s, dt, relax, j);
}

// physics_strand_apply_joint_corrections.cs.hlsl
__device__ __forceinline__ void applyJointsAt(const Scene &s, uint32_t g)
{
    const uint2 r = s.segJointRanges[g];
    float4 total = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t k = 0; k < r.y; ++k) {
        const uint2 ref = s.segJointInc[r.x + k];
        total = add4(total, s.jointCorr[2 * size_t(ref.x) + (ref.y == 0u ? 0u : 1u)]);
    }
    s.segOrient[g] = qNormalize(add4(s.segOrient[g], total));
}

__global__ void __launch_bounds__(kThreads) k_applyJoints(Scene s)
{
    pdlEnter();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < s.S) applyJointsAt(s, g);
}

// physics_strand_solve_distance_constraints.cs.hlsl:10-59
__device__ __forceinline__ void solveDistanceAt(const Scene &s, float dt, float relax, uint32_t c)
{
    const cn_strand_distance dc = s.dists[c];
    float4 cA = make_float4(0.f, 0.f, 0.f, 0.f), cB = cA;
    const float4 a = s.x[dc.particle_a], b = s.x[dc.particle_b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    const f3 delta = xyz(b) - xyz(a);
    const float l2 = dot(delta, delta);
    if (wSum > kEps && l2 > kEps) {
        const float len = sqrtf(l2);
        const f3 grad = delta / len;
        const float alpha = mx(dc.distance_compliance, 0.0f) / mx(dt * dt, kEps);
        const float lambda = s.distLambda[c];
        const float Cv = len - dc.rest_length;
        const float den = wSum + alpha;
        if (den > kEps) {
            const float dl = -(Cv + alpha * lambda) / den;
            s.distLambda[c] = lambda + dl;
            cA = mk4(wA * dl * -grad * relax, 0.0f);
            cB = mk4(wB * dl * grad * relax, 0.0f);
        }
    }
    const uint2 d = reinterpret_cast<const uint2 *>(s.distDst)[c];
    putRecord(s.distCorr, d.x, cA);
    putRecord(s.distCorr, d.y, cB);
}

__global__ void __launch_bounds__(kThreads) k_solveDistances(Scene s, float dt, float relax)
{
    pdlEnter();
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < s.SD) solveDistanceAt(s, dt, relax, c);
}

__device__ __forceinline__ void atomicAdd3(float4 *p, f3 v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}

// ------------------------------------------------------------------------------------------
// Contacts
// ------------------------------------------------------------------------------------------
// physics_particle_generate_explicit_contacts.cs.hlsl (no suturing state, no rigid proxies)
__device__ __forceinline__ void particleContactGenerateAt(const Scene &s, uint32_t pi)
{
    ParticleContact out{};
    const uint2 pr = s.particlePairs[pi];
    const uint32_t a = pr.x, b = pr.y;
    out.material = mk4(combineContactMaterial(s.contactMaterials[s.matIdx[a]], s.contactMaterials[s.matIdx[b]]), 0.0f);
    if (!(s.kinds[a] == CN_PARTICLE_FLUID && s.kinds[b] == CN_PARTICLE_FLUID)) {
        const f3 pa = xyz(s.x[a]), pb = xyz(s.x[b]);
        const float cr = s.radii[a] + s.radii[b];
        const f3 delta = pb - pa;
        const float d2 = dot(delta, delta);
        if (d2 <= kEps) {
            out.a = a; out.b = b; out.active = 1u;
            out.normalPenetration = make_float4(0.f, 1.f, 0.f, cr);
        } else {
            const float dist = sqrtf(d2);
            const float pen = cr - dist;
            if (pen > 0.0f) {
                out.a = a; out.b = b; out.active = 1u;
                out.normalPenetration = mk4(delta / dist, pen);
            }
        }
    }
    s.particleContacts[pi] = out;
}


// The rigid side of a proxy particle in a particle-particle contact: its body (inverse mass only
// for a dynamic body), the contact point at the body's predicted pose and its lever arm.
struct ProxySide {
    uint32_t body;
    float4 q;
    f3 r, invI;
};

__device__ __forceinline__ void loadProxySide(const Scene &s, uint32_t p, ProxySide &ps, float &invMass, f3 &cur)
{
    const uint32_t b = s.ownerIdx[p];
    const float4 bp = s.predBodyPos[b];
    ps.body = b;
    ps.q = qNormalize(s.predBodyRot[b]);
    invMass = s.bodyType[b] == CN_BODY_DYNAMIC ? bp.w : 0.0f;
    ps.invI = invMass > kEps ? xyz(s.bodyInvInertia[b]) : f3{0.f, 0.f, 0.f};
    cur = xyz(bp) + qRotate(ps.q, xyz(s.proxyLocal[p]));
    ps.r = cur - xyz(bp);
}

__device__ __forceinline__ f3 proxyPreviousPoint(const Scene &s, uint32_t p, uint32_t b)
{
    return xyz(s.prevBodyPos[b]) + qRotate(qNormalize(s.prevBodyRot[b]), xyz(s.proxyLocal[p]));
}

// physics_particle_solve_explicit_contacts.cs.hlsl; float atomics as in the reference.  A rigid
// proxy's share goes to its body's translation / rotation sums (effective mass with the lever
// arm); every other particle's to its position correction.
__device__ __forceinline__ void particleContactSolveAt(const Scene &s, const Config &cfg, uint32_t pi)
{
    const ParticleContact c = s.particleContacts[pi];
    if (c.active == 0u) return;
    atomicAdd(&s.meta_->activeParticleContacts, 1u);
    const float4 A = s.x[c.a], Bp = s.x[c.b];
    float iA = A.w, iB = Bp.w;
    f3 curA = xyz(A), curB = xyz(Bp);
    const bool proxyA = c.a < s.nProxy, proxyB = c.b < s.nProxy;
    ProxySide psA{}, psB{};
    if (proxyA) loadProxySide(s, c.a, psA, iA, curA);
    if (proxyB) loadProxySide(s, c.b, psB, iB, curB);
    if (iA <= kEps && iB <= kEps) return;
    const float pen = mn(mx(c.normalPenetration.w - cfg.slop, 0.0f), cfg.softMaxCorrection);
    if (pen <= 0.0f) return;
    const f3 mat = xyz(c.material);
    const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
    const f3 prevA = proxyA ? proxyPreviousPoint(s, c.a, psA.body) : xyz(s.xprev[c.a]);
    const f3 prevB = proxyB ? proxyPreviousPoint(s, c.b, psB.body) : xyz(s.xprev[c.b]);
    const f3 relDisp = (curB - prevB) - (curA - prevA);
    const float nmA = proxyA ? contactEffectiveMass(iA, psA.invI, psA.q, psA.r, n) : iA;
    const float nmB = proxyB ? contactEffectiveMass(iB, psB.invI, psB.q, psB.r, n) : iB;
    const float denom = nmA + nmB;
    if (denom <= kEps) return;
    const float lambda = (pen / denom) * cfg.softContactRelaxation;
    f3 cA{0.f, 0.f, 0.f}, cB{0.f, 0.f, 0.f}, tA{0.f, 0.f, 0.f}, tB{0.f, 0.f, 0.f}, rA{0.f, 0.f, 0.f},
        rB{0.f, 0.f, 0.f};
    if (proxyA) {
        tA = -n * (iA * lambda);
        rA = -mulWorldInvInertia(psA.invI, psA.q, cross(psA.r, n)) * lambda;
    } else {
        cA = -n * (iA * lambda);
    }
    if (proxyB) {
        tB = n * (iB * lambda);
        rB = mulWorldInvInertia(psB.invI, psB.q, cross(psB.r, n)) * lambda;
    } else {
        cB = n * (iB * lambda);
    }
    const f3 fd = positionFrictionDelta(projectOntoTangent(relDisp, n), pen, mat.x, mat.z,
                                        cfg.positionFrictionMinDistance);
    const float fdist = length(fd);
    if (fdist > 0.0f) {
        const f3 t = fd / fdist;
        const float tmA = proxyA ? contactEffectiveMass(iA, psA.invI, psA.q, psA.r, t) : iA;
        const float tmB = proxyB ? contactEffectiveMass(iB, psB.invI, psB.q, psB.r, t) : iB;
        const float tden = tmA + tmB;
        if (tden > kEps) {
            const float tl = (fdist / tden) * cfg.softContactRelaxation;
            if (proxyA) {
                tA += t * (iA * tl);
                rA += mulWorldInvInertia(psA.invI, psA.q, cross(psA.r, t)) * tl;
            } else {
                cA += t * (iA * tl);
            }
            if (proxyB) {
                tB -= t * (iB * tl);
                rB -= mulWorldInvInertia(psB.invI, psB.q, cross(psB.r, t)) * tl;
            } else {
                cB -= t * (iB * tl);
            }
        }
    }
    if (!proxyA && iA > kEps) atomicAdd3(&s.posCorr[c.a], cA);
    if (!proxyB && iB > kEps) atomicAdd3(&s.posCorr[c.b], cB);
    if (proxyA && iA > kEps) {
        atomicAdd3(&s.bodyTransCorr[psA.body], tA);
        atomicAdd3(&s.bodyRotCorr[psA.body], rA);
    }
    if (proxyB && iB > kEps) {
        atomicAdd3(&s.bodyTransCorr[psB.body], tB);
        atomicAdd3(&s.bodyRotCorr[psB.body], rB);
    }
}

// physics_particle_generate_explicit_contacts + physics_particle_solve_explicit_contacts, one pass:
// a pair's solve reads only its own contact and the two positions, which no pair changes (the
// corrections are summed into posCorr), so generating and solving it in the same thread gives the
// two-pass results.  The active-contact count is published and cleared by the position-correction
// apply that follows every such pass.
__global__ void __launch_bounds__(kThreads) k_particleContacts(Scene s, Config cfg)
{
    pdlEnter();
    // a fixed grid strides over the pairs that exist (a device count), not the capacity
    const uint32_t count = s.meta_->particlePairCount;
    for (uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x; pi < count; pi += gridDim.x * blockDim.x) {
        particleContactGenerateAt(s, pi);
        particleContactSolveAt(s, cfg, pi);
    }
}

// Particle-rigid contact for candidate pair `pi`: physics_particle_rigid_generate_contacts.cs.hlsl:29-210
// Particle-side inputs of a particle's rigid contacts, fetched once before its pair loop (in one
// memory round trip with the first pair).
struct ContactParticle {
    f3 pos, prev;
    float radius;
    uint4 meta;
    float4 material;
    bool proxy;
};

__device__ __forceinline__ ContactParticle loadContactParticle(const Scene &s, uint32_t i, float4 x)
{
    ContactParticle p;
    p.pos = xyz(x);
    p.prev = xyz(s.xprev[i]);
    p.radius = s.radii[i];
    p.meta = s.meta[i];
    p.material = s.contactMaterials[s.matIdx[i]];
    p.proxy = s.ownerTypes[i] == CN_OWNER_RIGID_BODY;
    return p;
}

__device__ __forceinline__ RigidContact generateRigidContact(const Scene &s, uint32_t i, uint32_t b,
                                                             const ContactParticle &pt)
{
    RigidContact out{};
    if (pt.proxy) return out;
    const f3 sp = pt.pos;
    const float sr = pt.radius;
    const uint4 m = pt.meta;
    const f3 bpos = xyz(s.predBodyPos[b]);
    const float4 bq = qNormalize(s.predBodyRot[b]);
    const float4 bsc = s.bodyScale[b];
    const uint2 cr = s.bodyColRanges[b];
    float bestPen = 0.0f;
    uint32_t bestCol = 0;
    f3 bestN{0.f, 1.f, 0.f}, bestW{0.f, 0.f, 0.f};
    for (uint32_t k = 0; k < kColliderIterationCap; ++k) {
        if (k >= cr.y) break;
        const uint32_t c = s.bodyColIdx[cr.x + k];
        const cn_collider_broadphase bp = s.colBp[c];
        const cn_collider_geometry cg = s.colGeo[c]; // before the filter: same round trip as bp
        if (bp.enabled_flag == 0u || bp.environment_index != m.x) continue;
        if ((m.w & bp.collision_layer) == 0u || (bp.collision_mask & m.z) == 0u) continue;
        const f3 clp{cg.local_position[0], cg.local_position[1], cg.local_position[2]};
        const float4 clq = qNormalize(make_float4(cg.local_orientation[0], cg.local_orientation[1],
                                                  cg.local_orientation[2], cg.local_orientation[3]));
        const f3 cwp = bpos + qRotate(bq, clp);
        const float4 cwq = qNormalize(qMul(bq, clq));
        const f3 pl = qInvRotate(cwq, sp - cwp);
        f3 nl{0.f, 1.f, 0.f}, cw{0.f, 0.f, 0.f};
        float sd = 0.0f;
        const float4 sp4 = make_float4(cg.shape_params[0], cg.shape_params[1], cg.shape_params[2], cg.shape_params[3]);
        if (bp.shape_type == CN_COLLIDER_SPHERE) {
            const float r = sphereRadius(sp4, bsc);
            const float l = sqrtf(dot(pl, pl));
            nl = l > kEps ? (pl / l) : f3{0.f, 1.f, 0.f};
            sd = l - r;
            cw = cwp + qRotate(cwq, nl * r);
        } else if (bp.shape_type == CN_COLLIDER_BOX) {
            const f3 he = boxHalfExtents(sp4, bsc);
            const f3 cl = clamp3(pl, -he, he);
            const f3 d = pl - cl;
            const float dl = sqrtf(dot(d, d));
            if (dl > kEps) {
                nl = d / dl;
                sd = dl;
                cw = cwp + qRotate(cwq, cl);
            } else {
                nl = closestFaceNormalLocal(pl, he);
                const f3 ds = he - fabs3(pl);
                sd = -mn(ds.x, mn(ds.y, ds.z));
                f3 cs = pl;
                if (fabsf(nl.x) > 0.5f) cs.x = nl.x * he.x;
                else if (fabsf(nl.y) > 0.5f) cs.y = nl.y * he.y;
                else cs.z = nl.z * he.z;
                cw = cwp + qRotate(cwq, cs);
            }
        } else {
            f3 a, b2;
            float cap = 0.0f;
            capsuleSegment(cwp, cwq, sp4, bsc, a, b2, cap);
            const f3 seg = b2 - a;
            const float l2 = dot(seg, seg);
            float t = 0.0f;
            if (l2 > kEps) t = saturate(dot(sp - a, seg) / l2);
            const f3 cl = lerp3(a, b2, t);
            const f3 d = sp - cl;
            const float l = sqrtf(dot(d, d));
            const f3 wn = l > kEps ? (d / l) : f3{1.f, 0.f, 0.f};
            sd = l - cap;
            nl = qInvRotate(cwq, wn);
            cw = cl + wn * cap;
        }
        const float pen = sr - sd;
        if (pen <= 0.0f || pen <= bestPen) continue;
        bestPen = pen;
        bestCol = c;
        bestN = safeNormalize(qRotate(cwq, nl), f3{0.f, 1.f, 0.f});
        bestW = cw;
    }
    if (bestPen > 0.0f) {
        out.particle = i; out.body = b; out.collider = bestCol; out.active = 1u;
        out.normalPenetration = mk4(bestN, bestPen);
        out.rigidLocalPoint = mk4(qInvRotate(bq, bestW - bpos), 0.0f);
    }
    return out;
}

// physics_particle_rigid_solve_contacts.cs.hlsl:27-141 for one contact: the particle's correction
// and, for a dynamic body, the body's translation / rotation corrections.
struct ContactCorrection {
    f3 soft, rigidT, rigidR;
    bool rigid;
};

__device__ __forceinline__ ContactCorrection solveRigidContact(const Scene &s, const Config &cfg,
                                                               const RigidContact &c, float4 sp,
                                                               const ContactParticle &pt)
{
    ContactCorrection out{f3{0.f, 0.f, 0.f}, f3{0.f, 0.f, 0.f}, f3{0.f, 0.f, 0.f}, false};
    const uint32_t b = c.body;
    const float iS = sp.w;
    const f3 prevS = pt.prev;
    const float4 prevB = s.prevBodyPos[b], predB = s.predBodyPos[b];
    const float4 prevQ = qNormalize(s.prevBodyRot[b]), predQ = qNormalize(s.predBodyRot[b]);
    const float iR = s.bodyType[b] == CN_BODY_DYNAMIC ? predB.w : 0.0f;
    if (iS <= kEps && iR <= kEps) return out;
    const float pen = mn(mx(c.normalPenetration.w - cfg.slop, 0.0f), cfg.softMaxCorrection);
    if (pen <= 0.0f) return out;
    const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
    f3 inI = xyz(s.bodyInvInertia[b]);
    const f3 mat = combineContactMaterial(pt.material, s.colMat[c.collider]);
    if (iR <= kEps) inI = f3{0.f, 0.f, 0.f};
    const f3 prevCP = xyz(prevB) + qRotate(prevQ, xyz(c.rigidLocalPoint));
    const f3 cp = xyz(predB) + qRotate(predQ, xyz(c.rigidLocalPoint));
    const f3 rR = cp - xyz(predB);
    const float nmR = contactEffectiveMass(iR, inI, predQ, rR, n);
    const float denom = iS + nmR;
    if (denom <= kEps) return out;
    const float lambda = (pen / denom) * cfg.softContactRelaxation;
    f3 corr = n * (iS * lambda);
    f3 rt = -n * (iR * lambda);
    f3 rr = -mulWorldInvInertia(inI, predQ, cross(rR, n)) * lambda;
    const f3 relDisp = (cp - prevCP) - (xyz(sp) - prevS);
    const f3 fd = positionFrictionDelta(projectOntoTangent(relDisp, n), pen, mat.x, mat.z,
                                        cfg.positionFrictionMinDistance);
    const float fdist = length(fd);
    if (fdist > 0.0f) {
        const f3 t = fd / fdist;
        const float tmR = contactEffectiveMass(iR, inI, predQ, rR, t);
        const float tden = iS + tmR;
        if (tden > kEps) {
            const float tl = fdist / tden;
            corr += t * (tl * iS * cfg.softContactRelaxation);
            rt -= t * (tl * iR * cfg.softContactRelaxation);
            rr -= mulWorldInvInertia(inI, predQ, cross(rR, t)) * (tl * cfg.softContactRelaxation);
        }
    }
    if (iS > kEps) out.soft = corr;
    if (iR > kEps) {
        out.rigidT = rt;
        out.rigidR = rr;
        out.rigid = true;
    }
    return out;
}

// Generate + solve every candidate pair of particle i (pairs are particle-major), then either
// accumulate into posCorr (explicit contacts present) or apply directly
// (physics_particle_apply_position_corrections.cs.hlsl:8-30).
// Particle i's contacts from its position sp (its x, or the value the fused gather just computed).
__device__ __forceinline__ void rigidContactsFrom(const Scene &s, const Config &cfg, bool applyDirect, uint32_t i,
                                                  const float4 sp)
{
    const uint32_t cnt = s.candCount[i];
    const uint32_t off = s.candOffset[i]; // with the count: one round trip fewer
    f3 corr{0.f, 0.f, 0.f};
    bool any = false;
    // A particle without weight takes no correction, and with no dynamic body nothing receives
    // its contacts' shares: only the stored records (the last contact iteration) need them.
    const bool inert = sp.w <= kEps && !s.hasDynamic && !s.storeRigidContacts;
    if (cnt && !inert) {
        const uint32_t lim = s.meta_->rigidPairCount;
        const ContactParticle pt = loadContactParticle(s, i, sp);
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t pi = off + k;
            if (pi >= lim) break;
            const uint2 pr = s.rigidPairs[pi]; // pr.x == i: pairs are emitted particle-major
            const RigidContact c = generateRigidContact(s, i, pr.y, pt);
            if (s.storeRigidContacts) s.rigidContacts[pi] = c;
            if (!c.active) continue;
            const ContactCorrection d = solveRigidContact(s, cfg, c, sp, pt);
            // the particle's float-atomic order of the reference == pair order here
            if (sp.w > kEps) {
                corr = corr + d.soft;
                any = true;
            }
            if (d.rigid) { // many particles push one body: float atomics, as the reference
                atomicAdd3(&s.bodyTransCorr[pr.y], d.rigidT);
                atomicAdd3(&s.bodyRotCorr[pr.y], d.rigidR);
            }
        }
    }
    if (applyDirect) {
        // applyParticlePositionCorrections with an accumulator that only this pass wrote
        if (sp.w <= kEps) return;
        s.x[i] = mk4(xyz(sp) + corr, sp.w);
    } else if (any) {
        float4 pc = s.posCorr[i];
        pc = mk4(xyz(pc) + corr, pc.w);
        s.posCorr[i] = pc;
    }
}

__device__ __forceinline__ void rigidContactsAt(const Scene &s, const Config &cfg, bool applyDirect, uint32_t i)
{
    rigidContactsFrom(s, cfg, applyDirect, i, s.x[i]);
}

__global__ void __launch_bounds__(kThreads) k_rigidContacts(Scene s, Config cfg, bool applyDirect)
{
    pdlEnter();
    forEachElem(s.wP, s.N, [&](uint32_t i) { rigidContactsAt(s, cfg, applyDirect, i); });
}

// The tet family's gather and the particle-rigid contacts that follow it, in one pass, for
// iterations without particle-particle contacts: a particle's rigid contacts read only its own
// position, its candidate pairs and the colliders, so running them in the same thread right after
// its gather (over the same particles as the two per-phase kernels: the tet window, then every
// particle) gives their results bit for bit with one launch and one pass over x fewer.
__global__ void __launch_bounds__(kThreads) k_applyTetsRigidContacts(Scene s, Config cfg)
{
    pdlEnter();
    // the gathered position goes to the contacts in registers: x is read and written once
    forEachElem(s.wP, s.N, [&](uint32_t i) {
        float4 p = s.x[i];
        if (s.wP.tiles || (i >= s.tetWin.x && i < s.tetWin.y)) p = gatheredPosition(s.tetRanges, s.tetCorr, i, p);
        rigidContactsFrom(s, cfg, true, i, p);
    });
}

// physics_particle_apply_position_corrections.cs.hlsl:8-30
__device__ __forceinline__ void applyPositionCorrectionAt(const Scene &s, uint32_t i)
{
    const f3 c = xyz(s.posCorr[i]);
    s.posCorr[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 p = s.x[i];
    if (p.w <= kEps) return;
    s.x[i] = mk4(xyz(p) + c, p.w);
}

// The particle-particle pass of this iteration is complete: its active-contact count becomes the
// reported one and the counter starts again at zero for the next pass.
__device__ __forceinline__ void publishParticleContactCount(const Scene &s)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s.meta_->activeParticleContactsLast = s.meta_->activeParticleContacts;
        s.meta_->activeParticleContacts = 0u;
    }
}

__global__ void __launch_bounds__(kThreads) k_applyPositionCorrections(Scene s)
{
    pdlEnter();
    publishParticleContactCount(s);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.N) applyPositionCorrectionAt(s, i);
}


// ------------------------------------------------------------------------------------------
// Velocity update and velocity-level passes
// ------------------------------------------------------------------------------------------
// physics_particle_update_velocities.cs.hlsl:13-44 (the fluid accumulated delta lives at the
// particle's sorted slot)
__device__ __forceinline__ void updateVelocityAt(const Scene &s, float dt, const float4 *Dfinal, uint32_t i)
{
    const float4 p = s.x[i];
    const float4 prev = s.xprev[i];      // loaded with x (not after the mass test):
    const uint32_t mi = s.matIdx[i];     // one round trip fewer
    if (p.w <= kEps || dt <= kEps) {
        s.v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const f3 pp = xyz(prev);
    f3 pos = xyz(p);
    if (Dfinal && s.kinds[i] == CN_PARTICLE_FLUID) {
        pos += xyz(Dfinal[s.rank[i]]);
        s.x[i] = mk4(pos, p.w);
    }
    const float damping = mx(s.contactMaterials[mi].z, 0.0f);
    const float ds = mx(1.0f - damping * dt, 0.0f);
    s.v[i] = mk4(((pos - pp) / dt) * ds, 0.0f);
}

__global__ void __launch_bounds__(kThreads) k_updateVelocities(Scene s, float dt, const float4 *Dfinal)
{
    pdlEnter();
    forEachElem(s.wP, s.N, [&](uint32_t i) { updateVelocityAt(s, dt, Dfinal, i); });
}

// physics_fluid_project_boundary_velocities.cs.hlsl:24-117
__global__ void __launch_bounds__(kThreads) k_fluidBoundaryVelocities(Scene s, float dt, Config cfg)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N || s.kinds[i] != CN_PARTICLE_FLUID) return;
    const uint32_t slot = s.rank[i];
    if (!hasBoundary(s, slot)) return;
    const f3 pos = xyz(s.x[i]);
    const float pr = mx(s.radii[i], 0.0f);
    const f3 vel = xyz(s.v[i]);
    const float4 pm = s.contactMaterials[s.matIdx[i]];
    const float pd = mx(pm.z, 0.0f);
    float bestD = 3.402823466e+38f;
    f3 bestN{0.f, 1.f, 0.f}, bestMat{0.f, 0.f, 0.f};
    bool found = false;
    forEachBoundary(s, slot, [&](uint32_t k) {
        const uint32_t c = s.colQueryOrder[k];
        float sd = 0.0f;
        f3 n{0.f, 1.f, 0.f};
        if (!fluidBoundaryContactInfo(s, c, pos, sd, n)) return;
        const float cd = pr + 2.0f * cfg.slop;
        if (sd > cd) return;
        if (sd < bestD) {
            bestD = sd;
            bestN = n;
            bestMat = combineContactMaterial(pm, s.colMat[c]);
            found = true;
        }
    });
    if (!found) return;
    const float pen = mx(pr - bestD, 0.0f);
    const float cd = mx(pr + 2.0f * cfg.slop, 1.0e-5f);
    const float cw = saturate((cd - bestD) / cd);
    f3 rv = vel;
    const float nv = dot(rv, bestN);
    if (nv < 0.0f) rv -= bestN * nv;
    f3 tv = projectOntoTangent(rv, bestN);
    if (dt > kEps) {
        const f3 fd = positionFrictionDelta(tv * dt, mx(pen, cfg.slop), bestMat.x, bestMat.z,
                                            cfg.positionFrictionMinDistance);
        tv -= fd / dt;
    }
    const float tds = mx(1.0f - pd * cw * dt, 0.0f);
    tv = tv * tds;
    rv = bestN * mx(dot(rv, bestN), 0.0f) + tv;
    s.v[i] = mk4(rv, 0.0f);
}

// physics_particle_rigid_solve_contact_velocities.cs.hlsl + apply_contact_velocities.cs.hlsl for
// all `iterations` at once: with static/kinematic bodies each particle's velocity only depends
// on its own contacts, and the per-particle sum runs in contact order.
__device__ __forceinline__ void rigidContactVelocitiesAt(const Scene &s, uint32_t iterations, const Config &cfg, uint32_t i)
{
    const uint32_t cnt = s.candCount[i];
    const uint32_t off = s.candOffset[i]; // with the count: one round trip fewer
    if (cnt == 0u) return;
    const float iS = s.x[i].w;
    const float4 v0 = s.v[i];
    if (iS <= kEps) return; // corrections are only applied to particles with mass
    const uint32_t lim = s.meta_->rigidPairCount;
    const float rpt = cfg.restitutionPenetrationThreshold;
    f3 vel = xyz(v0);
    const float vw = v0.w;
    for (uint32_t it = 0; it < iterations; ++it) {
        f3 corr{0.f, 0.f, 0.f};
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t pi = off + k;
            if (pi >= lim) break;
            const RigidContact c = s.rigidContacts[pi];
            if (!c.active) continue;
            const uint32_t b = c.body;
            const float4 rp = s.predBodyPos[b];
            const float iR = s.bodyType[b] == CN_BODY_DYNAMIC ? rp.w : 0.0f;
            const float4 rq = qNormalize(s.predBodyRot[b]);
            const f3 rl = xyz(s.predBodyLin[b]), ra = xyz(s.predBodyAng[b]);
            const f3 inI = xyz(s.bodyInvInertia[b]);
            const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
            const f3 cp = xyz(rp) + qRotate(rq, xyz(c.rigidLocalPoint));
            const f3 rR = cp - xyz(rp);
            const f3 rcv = rl + cross(ra, rR);
            const f3 rel = vel - rcv;
            const float nv = dot(rel, n);
            if (nv >= 0.0f) continue;
            const float nd = iS + contactEffectiveMass(iR, inI, rq, rR, n);
            if (nd <= kEps) continue;
            const f3 mat = combineContactMaterial(s.contactMaterials[s.matIdx[i]], s.colMat[c.collider]);
            const bool er = (-nv > cfg.restitutionVelocityThreshold) && (c.normalPenetration.w <= rpt);
            const float rest = er ? saturate(mat.y) : 0.0f;
            const float dnv = er ? (-rest * nv) : 0.0f;
            const float imp = mx(0.0f, (dnv - nv) / nd);
            corr = corr + (n * imp) * iS;
        }
        vel = vel + corr;
    }
    s.v[i] = mk4(vel, vw);
}

__global__ void __launch_bounds__(kThreads) k_rigidContactVelocities(Scene s, uint32_t iterations, Config cfg)
{
    forEachElem(s.wP, s.N, [&](uint32_t i) { rigidContactVelocitiesAt(s, iterations, cfg, i); });
}

// ------------------------------------------------------------------------------------------
// Dynamic bodies
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ f3 clampLength(f3 v, float maxLen)
{
    const float l = length(v);
    if (l > maxLen && l > kEps) v = v * (maxLen / l);
    return v;
}

// physics_rigid_apply_corrections.cs.hlsl:13-54 (clears the sums for the next pass)
__global__ void k_applyRigidCorrections(Scene s, Config cfg)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.B) return;
    float4 p = s.predBodyPos[b];
    float4 q = qNormalize(s.predBodyRot[b]);
    f3 tc = xyz(s.bodyTransCorr[b]);
    f3 rc = xyz(s.bodyRotCorr[b]);
    if (s.bodyType[b] == CN_BODY_DYNAMIC && p.w != 0.0f) {
        tc = clampLength(tc, cfg.maxTranslationCorrection);
        rc = clampLength(rc, cfg.maxRotationCorrection);
        p = mk4(xyz(p) + tc, p.w);
        q = qNormalize(qMul(qFromRotationVector(rc), q));
    }
    s.predBodyPos[b] = p;
    s.predBodyRot[b] = q;
    s.bodyTransCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.bodyRotCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// physics_rigid_update_velocities.cs.hlsl:14-51
__global__ void k_updateRigidVelocities(Scene s, float dt)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.B) return;
    const float4 prevP = s.prevBodyPos[b];
    const float4 prevQ = qNormalize(s.prevBodyRot[b]);
    const float4 p = s.predBodyPos[b];
    float4 q = qNormalize(s.predBodyRot[b]);
    if (s.bodyType[b] == CN_BODY_STATIC) {
        s.predBodyRot[b] = qNormalize(q);
        s.predBodyLin[b] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.predBodyAng[b] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const f3 l = (xyz(p) - xyz(prevP)) / mx(dt, kEps);
    const f3 a = angularVelocityFromQuaternionDelta(prevQ, q, mx(dt, kEps));
    s.predBodyRot[b] = q;
    s.predBodyLin[b] = mk4(l, 0.0f);
    s.predBodyAng[b] = mk4(a, 0.0f);
}

// One iteration of physics_particle_rigid_solve_contact_velocities.cs.hlsl:30-123 with dynamic
// bodies: a particle's impulses from its contacts (pair order, its velocity of this iteration)
// are applied to it directly (physics_particle_apply_contact_velocities); the bodies' shares are
// summed with float atomics and applied by k_applyRigidContactVelocities.
__global__ void __launch_bounds__(kThreads) k_rigidContactVelocityStep(Scene s, Config cfg)
{
    forEachElem(s.wP, s.N, [&](uint32_t i) {
        const uint32_t cnt = s.candCount[i];
        const uint32_t off = s.candOffset[i];
        if (cnt == 0u) return;
        const float iS = s.x[i].w;
        const float4 v0 = s.v[i];
        const uint32_t lim = s.meta_->rigidPairCount;
        const f3 vel = xyz(v0);
        f3 corr{0.f, 0.f, 0.f};
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t pi = off + k;
            if (pi >= lim) break;
            const RigidContact c = s.rigidContacts[pi];
            if (!c.active) continue;
            const uint32_t b = c.body;
            const float4 rp = s.predBodyPos[b];
            const float iR = s.bodyType[b] == CN_BODY_DYNAMIC ? rp.w : 0.0f;
            if (iS <= kEps && iR <= kEps) continue;
            const float4 rq = qNormalize(s.predBodyRot[b]);
            const f3 rl = xyz(s.predBodyLin[b]), ra = xyz(s.predBodyAng[b]);
            const f3 inI = xyz(s.bodyInvInertia[b]);
            const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
            const f3 cp = xyz(rp) + qRotate(rq, xyz(c.rigidLocalPoint));
            const f3 rR = cp - xyz(rp);
            const f3 rel = vel - (rl + cross(ra, rR));
            const float nv = dot(rel, n);
            if (nv >= 0.0f) continue;
            const float nd = iS + contactEffectiveMass(iR, inI, rq, rR, n);
            if (nd <= kEps) continue;
            const f3 mat = combineContactMaterial(s.contactMaterials[s.matIdx[i]], s.colMat[c.collider]);
            const bool er = (-nv > cfg.restitutionVelocityThreshold) && (c.normalPenetration.w <= cfg.restitutionPenetrationThreshold);
            const float rest = er ? saturate(mat.y) : 0.0f;
            const float dnv = er ? (-rest * nv) : 0.0f;
            const f3 ti = n * mx(0.0f, (dnv - nv) / nd);
            if (iS > kEps) corr = corr + ti * iS;
            if (iR > kEps) {
                atomicAdd3(&s.bodyLinVelCorr[b], -ti * iR);
                atomicAdd3(&s.bodyAngVelCorr[b], mulWorldInvInertia(inI, rq, cross(rR, -ti)));
            }
        }
        if (iS > kEps) s.v[i] = mk4(vel + corr, v0.w);
    });
}

// physics_rigid_apply_contact_velocities.cs.hlsl:14-58
__global__ void k_applyRigidContactVelocities(Scene s, Config cfg)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.B) return;
    float4 lin = s.predBodyLin[b], ang = s.predBodyAng[b];
    if (s.bodyType[b] == CN_BODY_DYNAMIC) {
        const f3 lc = clampLength(xyz(s.bodyLinVelCorr[b]), cfg.maxLinearVelocityCorrection);
        const f3 ac = clampLength(xyz(s.bodyAngVelCorr[b]), cfg.maxAngularVelocityCorrection);
        lin = mk4(xyz(lin) + lc, lin.w);
        ang = mk4(xyz(ang) + ac, ang.w);
    }
    s.predBodyLin[b] = lin;
    s.predBodyAng[b] = ang;
    s.bodyLinVelCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.bodyAngVelCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// physics_particle_solve_contact_velocities.cs.hlsl with float atomics: a rigid proxy moves with
// its body's velocity at the proxy's lever arm, and its impulse share goes to the body's
// velocity sums.
__device__ __forceinline__ void particleContactVelocitiesAt(const Scene &s, const Config &cfg, uint32_t pi)
{
    const ParticleContact c = s.particleContacts[pi];
    if (c.active == 0u) return;
    float iA = s.x[c.a].w, iB = s.x[c.b].w;
    f3 vA = xyz(s.v[c.a]), vB = xyz(s.v[c.b]);
    const bool proxyA = c.a < s.nProxy, proxyB = c.b < s.nProxy;
    ProxySide psA{}, psB{};
    if (proxyA) {
        f3 cur;
        loadProxySide(s, c.a, psA, iA, cur);
        psA.r = qRotate(psA.q, xyz(s.proxyLocal[c.a]));
        vA = xyz(s.predBodyLin[psA.body]) + cross(xyz(s.predBodyAng[psA.body]), psA.r);
    }
    if (proxyB) {
        f3 cur;
        loadProxySide(s, c.b, psB, iB, cur);
        psB.r = qRotate(psB.q, xyz(s.proxyLocal[c.b]));
        vB = xyz(s.predBodyLin[psB.body]) + cross(xyz(s.predBodyAng[psB.body]), psB.r);
    }
    if (iA <= kEps && iB <= kEps) return;
    const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
    const float nv = dot(vB - vA, n);
    if (nv >= 0.0f) return;
    const float nmA = proxyA ? contactEffectiveMass(iA, psA.invI, psA.q, psA.r, n) : iA;
    const float nmB = proxyB ? contactEffectiveMass(iB, psB.invI, psB.q, psB.r, n) : iB;
    const float denom = nmA + nmB;
    if (denom <= kEps) return;
    const f3 mat = xyz(c.material);
    const bool er = (-nv > cfg.restitutionVelocityThreshold) && (c.normalPenetration.w <= cfg.restitutionPenetrationThreshold);
    const float rest = er ? saturate(mat.y) : 0.0f;
    const float dnv = er ? (-rest * nv) : 0.0f;
    const float imp = mx(0.0f, (dnv - nv) / denom);
    const f3 ti = n * imp;
    if (!proxyA && iA > kEps) atomicAdd3(&s.velCorr[c.a], -ti * iA);
    if (!proxyB && iB > kEps) atomicAdd3(&s.velCorr[c.b], ti * iB);
    if (proxyA && iA > kEps) {
        atomicAdd3(&s.bodyLinVelCorr[psA.body], -ti * iA);
        atomicAdd3(&s.bodyAngVelCorr[psA.body], mulWorldInvInertia(psA.invI, psA.q, cross(psA.r, -ti)));
    }
    if (proxyB && iB > kEps) {
        atomicAdd3(&s.bodyLinVelCorr[psB.body], ti * iB);
        atomicAdd3(&s.bodyAngVelCorr[psB.body], mulWorldInvInertia(psB.invI, psB.q, cross(psB.r, ti)));
    }
}

__global__ void __launch_bounds__(kThreads) k_particleContactVelocities(Scene s, Config cfg)
{
    // a fixed grid strides over the pairs that exist (a device count), not the capacity
    const uint32_t count = s.meta_->particlePairCount;
    for (uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x; pi < count; pi += gridDim.x * blockDim.x)
        particleContactVelocitiesAt(s, cfg, pi);
}

// physics_particle_apply_contact_velocities.cs.hlsl
__global__ void __launch_bounds__(kThreads) k_applyContactVelocities(Scene s)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    float4 v = s.v[i];
    const float im = s.x[i].w;
    const f3 c = xyz(s.velCorr[i]);
    if (im > kEps) v = mk4(xyz(v) + c, v.w);
    s.v[i] = v;
    s.velCorr[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Debug export: compacted (key, start, end, 0) runs in sorted order (reference table layout).
__global__ void k_runFlags(Scene s, uint32_t *flags)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N) return;
    flags[slot] = (slot == 0 || s.keysA[slot - 1] != s.keysA[slot]) ? 1u : 0u;
}
__global__ void k_runCompact(Scene s, const uint32_t *flags, const uint32_t *offsets, uint4 *out, uint32_t cap)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= s.N || flags[slot] == 0u) return;
    const uint32_t r = offsets[slot];
    if (r >= cap) return;
    out[r] = make_uint4(s.keysA[slot], slot, s.cellEnd[slot] & 0x7fffffffu, 0u);
}

// ------------------------------------------------------------------------------------------
// Surface render passes: render-vertex skinning, triangle and vertex normals, chunk and surface
// world AABBs.  They read only the positions the frame ends with, so they run once per frame
// (the reference dispatches them after every substep; earlier substeps' outputs are overwritten
// before anyone can read them).
// ------------------------------------------------------------------------------------------
// physics_surface_skin_render_vertices.cs.hlsl:14-36 and
// physics_surface_update_triangle_normals.cs.hlsl:8-24 (one thread covers a vertex and a triangle)
__global__ void __launch_bounds__(kThreads) k_surfaceSkinTriangles(Scene s)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.surfV) {
        const uint4 pi = s.surfBind[2 * size_t(i)];
        const uint4 wb = s.surfBind[2 * size_t(i) + 1];
        const float4 q0 = s.x[pi.x], q1 = s.x[pi.y], q2 = s.x[pi.z], q3 = s.x[pi.w];
        f3 acc{0.f, 0.f, 0.f};
        acc += __uint_as_float(wb.x) * xyz(q0);
        acc += __uint_as_float(wb.y) * xyz(q1);
        acc += __uint_as_float(wb.z) * xyz(q2);
        acc += __uint_as_float(wb.w) * xyz(q3);
        s.surfPos[i] = mk4(acc, 1.0f);
    }
    if (i < s.surfT) {
        const uint4 t = s.surfTri[i];
        const f3 p0 = xyz(s.x[t.x]), p1 = xyz(s.x[t.y]), p2 = xyz(s.x[t.z]);
        s.surfTriN[i] = mk4(cross(p2 - p0, p1 - p0), 0.0f);
    }
}

// physics_surface_update_render_normals.cs.hlsl:18-48: incident face normals summed in range
// order (fetched kGatherBatch at a time), normalised with 1 / sqrt (the shader's rsqrt is the
// hardware approximation; this is its correctly rounded value), fallback when degenerate.
__global__ void __launch_bounds__(kThreads) k_surfaceVertexNormals(Scene s)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.surfV) return;
    const uint4 r = s.surfRanges[i];
    f3 acc{0.f, 0.f, 0.f};
    for (uint32_t k = 0; k < r.y; k += kGatherBatch) {
        uint32_t tri[kGatherBatch];
#pragma unroll
        for (uint32_t j = 0; j < kGatherBatch; ++j) tri[j] = (k + j < r.y) ? s.surfIdx[r.x + k + j] : 0u;
        float4 n[kGatherBatch];
#pragma unroll
        for (uint32_t j = 0; j < kGatherBatch; ++j)
            if (k + j < r.y) n[j] = s.surfTriN[tri[j]];
#pragma unroll
        for (uint32_t j = 0; j < kGatherBatch; ++j)
            if (k + j < r.y) acc += xyz(n[j]);
    }
    f3 nrm = acc;
    const float lenSq = dot(nrm, nrm);
    if (lenSq <= 1.0e-12f) nrm = xyz(s.surfFallback[i]);
    else nrm = nrm * (1.0f / sqrtf(lenSq));
    s.surfNrm[i] = mk4(nrm, 0.0f);
}

__device__ __forceinline__ void warpMinMax(f3 &mn, f3 &mx3)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn.x = fminf(mn.x, __shfl_xor_sync(0xffffffffu, mn.x, o));
        mn.y = fminf(mn.y, __shfl_xor_sync(0xffffffffu, mn.y, o));
        mn.z = fminf(mn.z, __shfl_xor_sync(0xffffffffu, mn.z, o));
        mx3.x = fmaxf(mx3.x, __shfl_xor_sync(0xffffffffu, mx3.x, o));
        mx3.y = fmaxf(mx3.y, __shfl_xor_sync(0xffffffffu, mx3.y, o));
        mx3.z = fmaxf(mx3.z, __shfl_xor_sync(0xffffffffu, mx3.z, o));
    }
}

constexpr float kBoundsInit = 3.402823e+38f;

// physics_surface_update_bounds.cs.hlsl:12-65: one warp per 64-particle chunk (min / max are
// exact, so the reduction order does not matter)
__global__ void __launch_bounds__(kThreads) k_surfaceChunkBounds(Scene s)
{
    const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (c >= s.surfChunks) return; // the whole warp leaves together
    const uint4 ch = s.surfChunk[c];
    if (ch.z == 0u) {
        if (lane == 0u) {
            s.surfChunkAabb[2 * size_t(c)] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.surfChunkAabb[2 * size_t(c) + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        return;
    }
    f3 mn{kBoundsInit, kBoundsInit, kBoundsInit}, mxv{-kBoundsInit, -kBoundsInit, -kBoundsInit};
    for (uint32_t k = lane; k < ch.z; k += 32u) {
        const f3 p = xyz(s.x[ch.y + k]);
        mn = f3{fminf(mn.x, p.x), fminf(mn.y, p.y), fminf(mn.z, p.z)};
        mxv = f3{fmaxf(mxv.x, p.x), fmaxf(mxv.y, p.y), fmaxf(mxv.z, p.z)};
    }
    warpMinMax(mn, mxv);
    if (lane == 0u) {
        s.surfChunkAabb[2 * size_t(c)] = mk4(mn, 0.0f);
        s.surfChunkAabb[2 * size_t(c) + 1] = mk4(mxv, 0.0f);
    }
}

// physics_surface_finalize_bounds.cs.hlsl:12-66: one warp per surface over its chunks
__global__ void __launch_bounds__(kThreads) k_surfaceWorldBounds(Scene s)
{
    const uint32_t sf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (sf >= s.surfS) return;
    const uint2 r = s.surfChunkRange[sf];
    if (r.y == 0u) {
        if (lane == 0u) {
            s.surfWorldAabb[2 * size_t(sf)] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.surfWorldAabb[2 * size_t(sf) + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        return;
    }
    f3 mn{kBoundsInit, kBoundsInit, kBoundsInit}, mxv{-kBoundsInit, -kBoundsInit, -kBoundsInit};
    for (uint32_t k = lane; k < r.y; k += 32u) {
        const f3 a = xyz(s.surfChunkAabb[2 * size_t(r.x + k)]), b = xyz(s.surfChunkAabb[2 * size_t(r.x + k) + 1]);
        mn = f3{fminf(mn.x, a.x), fminf(mn.y, a.y), fminf(mn.z, a.z)};
        mxv = f3{fmaxf(mxv.x, b.x), fmaxf(mxv.y, b.y), fmaxf(mxv.z, b.z)};
    }
    warpMinMax(mn, mxv);
    if (lane == 0u) {
        s.surfWorldAabb[2 * size_t(sf)] = mk4(mn, 0.0f);
        s.surfWorldAabb[2 * size_t(sf) + 1] = mk4(mxv, 0.0f);
    }
}

} // namespace

// ------------------------------------------------------------------------------ launchers
void launchRigidPredict(const Scene &s, float dt, float gx, float gy, float gz, cudaStream_t st)
{
    if (s.B == 0 && s.C == 0) return;
    if (!s.wB.tiles && s.B + s.C > 4u * kThreads) {
        if (s.B) k_rigidPredictBodies<<<blocksFor(s.B), kThreads, 0, st>>>(s, dt, gx, gy, gz);
        if (s.C) k_colliderBoundsFrames<<<blocksFor(s.C), kThreads, 0, st>>>(s);
        return;
    }
    k_rigidPredict<<<1, kThreads, 0, st>>>(s, dt, gx, gy, gz);
}

void launchApplyBodyTargets(const Scene &s, const BodyTarget *list, const uint32_t *count, uint32_t capacity,
                            cudaStream_t st)
{
    if (capacity == 0) return;
    k_applyBodyTargets<<<blocksFor(capacity) < 64u ? blocksFor(capacity) : 64u, kThreads, 0, st>>>(s, list, count);
}

void launchCopyPredictedRigid(const Scene &s, cudaStream_t st)
{
    if (s.B == 0) return;
    k_copyPredictedRigid<<<1, kThreads, 0, st>>>(s);
}

void launchPredictAndKeys(const Scene &s, float dt, const Config &c, cudaStream_t st)
{
    if (s.N == 0) return;
    k_predictKeys<<<gridFor(s.wP, s.N), kThreads, 0, st>>>(s, dt, c.gravity[0], c.gravity[1], c.gravity[2],
                                                       s.entries != nullptr);
}

void launchCellSetup(const Scene &s, uint32_t *scanTmp, void *sortScratch, cudaStream_t st)
{
    if (s.N == 0) return;
    cudaMemsetAsync(s.tableKeys, 0xff, size_t(s.tableMask + 1) * sizeof(uint32_t), st);
    k_cellSetup<<<blocksFor(s.N), kThreads, 0, st>>>(s);
    if (s.runFlag) {
        exclusiveScan(s.runFlag, s.runIdx, s.N, s.runTotal, scanTmp + 1, st);
        cudaMemsetAsync(s.runKey, 0xff, size_t(s.N) * sizeof(uint32_t), st);
        k_runKeys<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        radixSortPairs(s.runKey, s.runVal, s.runKeyB, s.runValB, s.N, sortScratch, &s.meta_->waitTimeouts, st,
                       s.runTotal);
        k_runLengths<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        exclusiveScan(s.runLenSorted, s.runCompStart, s.N, scanTmp, scanTmp + 1, st);
        k_runPlace<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        k_computeOrderSetup<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        if (s.bList) { // per-slot fluid boundary candidate lists (more colliders than the mask holds)
            exclusiveScan(s.bCount, s.bOffset, s.N, scanTmp, scanTmp + 1, st);
            k_fluidBoundaryEmit<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        }
        // the runs number at most N (about N / 8 in a settled fluid): a fixed grid strides over them
        const unsigned grid = unsigned(std::min<size_t>(blocksFor(size_t(s.N) * 27u), 148u * 16u));
        k_runNeighbors<<<grid, kThreads, 0, st>>>(s);
    }
}

void launchRigidCandidates(const Scene &s, uint32_t *scanTmp, size_t, cudaStream_t st)
{
    if (s.N == 0) return;
    if (s.wP.tiles) cudaMemsetAsync(s.candCount, 0, sizeof(uint32_t) * s.N, st); // scenes not stepped: none
    k_rigidCandidates<false><<<gridFor(s.wP, s.N), kThreads, 0, st>>>(s, nullptr);
    uint32_t *total = scanTmp;
    exclusiveScan(s.candCount, s.candOffset, s.N, total, scanTmp + 1, st);
    k_rigidCandidates<true><<<gridFor(s.wP, s.N), kThreads, 0, st>>>(s, total);
}

void launchParticleCandidates(const Scene &s, uint32_t *scanTmp, size_t, cudaStream_t st)
{
    if (s.N == 0) return;
    k_particleCandidates<false><<<blocksFor(s.N), kThreads, 0, st>>>(s, nullptr);
    uint32_t *total = scanTmp;
    exclusiveScan(s.ppCount, s.ppOffset, s.N, total, scanTmp + 1, st);
    k_particleCandidates<true><<<blocksFor(s.N), kThreads, 0, st>>>(s, total);
}

// The first iteration of a substep as a superset-only cell walk plus the filter of the later
// iterations (true), or one walk that also builds the list and the density (false).
constexpr bool kSplitSupersetBuild = true;

// Positions of iteration k: buffer A (s.P) for even k, B (s.Pb) for odd k when double-buffered.
inline Scene withPositions(const Scene &s, uint32_t iter)
{
    Scene c = s;
    if (s.Pb && (iter & 1u)) c.P = s.Pb;
    return c;
}

void launchFluidGather(const Scene &s, uint32_t iter, cudaStream_t st)
{
    if (s.N == 0) return;
    const float4 *Dcur = (iter & 1u) ? s.Db : s.Da;
    float4 *second = iter == 0 ? (s.Pb ? s.Pb : s.P0) : nullptr;
    launchPdl(k_fluidGather, blocksFor(s.N), kThreads, st, withPositions(s, iter), s.Xs, Dcur, iter, second,
                                                       iter > 0 ? s.P0 : nullptr);
}

bool fluidGatherEachIteration(const Scene &s) { return s.Pb == nullptr; }

bool fluidListsInterleaved() { return kInterleavedLists; }

void launchFluidNeighborsDensity(const Scene &s, const Config &c, uint32_t iter, bool walkCells, cudaStream_t st)
{
    if (s.N == 0) return;
    const Scene sp = withPositions(s, iter);
    float4 *Dk = (iter & 1u) ? s.Db : s.Da;
    const unsigned g = fluidBlocksFor(s.N);
    if (s.sup == nullptr || walkCells) {
        if (s.fluidExtras) launchPdl(k_fluidNeighborsDensity<0u, true>, g, kFluidThreads, st, sp, c, true, iter, Dk);
        else launchPdl(k_fluidNeighborsDensity<0u, false>, g, kFluidThreads, st, sp, c, true, iter, Dk);
    } else if (iter == 0 && !kSplitSupersetBuild) {
        if (s.fluidExtras) launchPdl(k_fluidNeighborsDensity<1u, true>, g, kFluidThreads, st, sp, c, true, iter, Dk);
        else launchPdl(k_fluidNeighborsDensity<1u, false>, g, kFluidThreads, st, sp, c, true, iter, Dk);
    } else {
        if (iter == 0) { // the superset, then the filter below
            if (s.fluidExtras) launchPdl(k_fluidNeighborsDensity<3u, true>, g, kFluidThreads, st, sp, c, true, iter, Dk);
            else launchPdl(k_fluidNeighborsDensity<3u, false>, g, kFluidThreads, st, sp, c, true, iter, Dk);
        }
        if (s.fluidExtras) launchPdl(k_fluidNeighborsDensity<2u, true>, g, kFluidThreads, st, sp, c, true, iter, Dk);
        else launchPdl(k_fluidNeighborsDensity<2u, false>, g, kFluidThreads, st, sp, c, true, iter, Dk);
    }
}

void launchFluidDeltaApplyClamp(const Scene &s, uint32_t iter, float dt, const Config &c, bool writeDebug,
                                cudaStream_t st)
{
    if (s.N == 0) return;
    const float4 *Dcur = (iter & 1u) ? s.Db : s.Da;
    float4 *Dnext = (iter & 1u) ? s.Da : s.Db;
    float4 *Pnext = s.Pb ? ((iter & 1u) ? s.P : s.Pb) : nullptr;
    if (s.fluidExtras)
        launchPdl(k_fluidDeltaApplyClamp<true>, fluidBlocksFor(s.N), kFluidThreads, st, withPositions(s, iter), c, s.Xs, Dcur, Dnext,
                                                                      iter, dt, writeDebug, Pnext);
    else
        launchPdl(k_fluidDeltaApplyClamp<false>, fluidBlocksFor(s.N), kFluidThreads, st, withPositions(s, iter), c, s.Xs, Dcur, Dnext,
                                                                       iter, dt, writeDebug, Pnext);
}

void launchFluidIteration(const Scene &s, uint32_t iter, float dt, const Config &c, bool writeDebug,
                          cudaStream_t st)
{
    if (iter == 0 || fluidGatherEachIteration(s)) launchFluidGather(s, iter, st);
    launchFluidNeighborsDensity(s, c, iter, false, st);
    launchFluidDeltaApplyClamp(s, iter, dt, c, writeDebug, st);
}

void launchFluidVorticity(const Scene &s, float dt, cudaStream_t st)
{
    if (s.N == 0 || !s.fluidVort) return;
    k_fluidVorticity<<<blocksFor(s.N), kThreads, 0, st>>>(s);
    k_fluidVorticityApply<<<blocksFor(s.N), kThreads, 0, st>>>(s, dt);
}

void launchFluidNeighborsOnly(const Scene &s, cudaStream_t st)
{
    if (s.N == 0) return;
    // Positions after the velocity update; the accumulated delta was folded into x.
    launchPdl(k_fluidGather, blocksFor(s.N), kThreads, st, s, s.Xs, s.Da, 0u, nullptr, nullptr);
    Config dummy{};
    launchPdl(k_fluidNeighborsDensity<0u, false>, fluidBlocksFor(s.N), kFluidThreads, st, s, dummy, false, 0u, nullptr);
}

// ------------------------------------------------------------------------------------------
// Graph-coloured XPBD schedules
// ------------------------------------------------------------------------------------------
// A colour's constraints share no particle (no segment, for joints).  Each constraint is solved
// by the gather schedule's own per-constraint function, which writes its correction records and
// lambda; the same thread then moves its records into the particles (Gauss-Seidel: applied
// before the next colour is solved) or into the per-particle sum (colour Jacobi: every
// correction of the family from the positions at the family's start, summed in colour order).
__device__ __forceinline__ void moveRecord(const Scene &s, bool gaussSeidel, uint32_t p, float4 r)
{
    if (p >= s.N) return;
    if (gaussSeidel) {
        const float4 q = s.x[p];
        if (q.w > kEps) s.x[p] = mk4(xyz(q) + xyz(r), q.w);
    } else {
        const float4 a = s.softAcc[p];
        s.softAcc[p] = mk4(xyz(a) + xyz(r), 0.0f);
    }
}

__device__ __forceinline__ void moveOrientation(const Scene &s, bool gaussSeidel, uint32_t g, float4 r)
{
    if (g >= s.S) return;
    if (gaussSeidel) s.segOrient[g] = qNormalize(add4(s.segOrient[g], r));
    else s.orientAcc[g] = add4(s.orientAcc[g], r);
}

template <uint32_t kFam>
__device__ __forceinline__ void colourConstraint(const Scene &s, float dt, float relax, bool gaussSeidel, uint32_t c)
{
    if constexpr (kFam == kFamEdges) {
        solveEdge(s, dt, relax, c);
        const cn_soft_edge ed = s.edges[c];
        const uint2 d = reinterpret_cast<const uint2 *>(s.edgeDst)[c];
        moveRecord(s, gaussSeidel, ed.particle_a, recordAt(s.edgeCorr, d.x));
        moveRecord(s, gaussSeidel, ed.particle_b, recordAt(s.edgeCorr, d.y));
    } else if constexpr (kFam == kFamSegments) {
        // a segment's orientation is read by its own constraint alone: applied in place
        solveSegmentAt(s, dt, relax, c);
        const cn_strand_segment sg = s.segs[c];
        moveRecord(s, gaussSeidel, sg.particle_a, s.segCorr[3 * size_t(c)]);
        moveRecord(s, gaussSeidel, sg.particle_b, s.segCorr[3 * size_t(c) + 1]);
        s.segOrient[c] = qNormalize(add4(s.segOrient[c], s.segCorr[3 * size_t(c) + 2]));
    } else if constexpr (kFam == kFamBends) {
        const uint4 d = reinterpret_cast<const uint4 *>(s.bendDst)[c];
        if (c < s.Bn) {
            solveBendAt(s, dt, relax, c);
            const cn_soft_bend b = s.bends[c];
            moveRecord(s, gaussSeidel, b.particle0, recordAt(s.bendCorr, d.x));
            moveRecord(s, gaussSeidel, b.particle1, recordAt(s.bendCorr, d.y));
            moveRecord(s, gaussSeidel, b.particle2, recordAt(s.bendCorr, d.z));
        } else {
            solveDihedralAt(s, dt, relax, c - s.Bn);
            const cn_cloth_dihedral h = s.dihedrals[c - s.Bn];
            moveRecord(s, gaussSeidel, h.edge_particle0, recordAt(s.bendCorr, d.x));
            moveRecord(s, gaussSeidel, h.edge_particle1, recordAt(s.bendCorr, d.y));
            moveRecord(s, gaussSeidel, h.opposite_particle0, recordAt(s.bendCorr, d.z));
            moveRecord(s, gaussSeidel, h.opposite_particle1, recordAt(s.bendCorr, d.w));
        }
    } else if constexpr (kFam == kFamJoints) {
        solveJointAt(s, dt, relax, c);
        const cn_strand_joint jt = s.joints[c];
        moveOrientation(s, gaussSeidel, jt.segment_a, s.jointCorr[2 * size_t(c)]);
        moveOrientation(s, gaussSeidel, jt.segment_b, s.jointCorr[2 * size_t(c) + 1]);
    } else if constexpr (kFam == kFamDistances) {
        solveDistanceAt(s, dt, relax, c);
        const cn_strand_distance dc = s.dists[c];
        const uint2 d = reinterpret_cast<const uint2 *>(s.distDst)[c];
        moveRecord(s, gaussSeidel, dc.particle_a, recordAt(s.distCorr, d.x));
        moveRecord(s, gaussSeidel, dc.particle_b, recordAt(s.distCorr, d.y));
    } else {
        solveTet(s, dt, relax, c);
        const cn_soft_tet t = s.tets[c];
        const uint4 d = reinterpret_cast<const uint4 *>(s.tetDst)[c];
        moveRecord(s, gaussSeidel, t.particle_indices[0], recordAt(s.tetCorr, d.x));
        moveRecord(s, gaussSeidel, t.particle_indices[1], recordAt(s.tetCorr, d.y));
        moveRecord(s, gaussSeidel, t.particle_indices[2], recordAt(s.tetCorr, d.z));
        moveRecord(s, gaussSeidel, t.particle_indices[3], recordAt(s.tetCorr, d.w));
    }
}

// A coloured batch's constraint at colour position q (its edges and tets stored in colour order):
// the same per-constraint solve, its lambda at q, the corrections moved from registers; a tet that
// keeps its previous corrections takes them from its colour-ordered record.  Same values, same
// order of the moves as colourConstraint.
template <uint32_t kFam>
__device__ __forceinline__ void colourConstraintOrdered(const Scene &s, float dt, float relax, bool gaussSeidel, uint32_t q)
{
    float newLambda;
    if constexpr (kFam == kFamEdges) {
        const PackedEdge ed = s.edgesC[q];
        float4 cA, cB;
        if (edgeSolve(s, dt, relax, ed, s.edgeLambda[q], newLambda, cA, cB)) s.edgeLambda[q] = newLambda;
        moveRecord(s, gaussSeidel, ed.a, cA);
        moveRecord(s, gaussSeidel, ed.b & 0x7fffffffu, cB);
    } else {
        const cn_soft_tet t = s.tetsC[q];
        float4 c[4];
        float4 *rec = s.tetRecC + 4 * size_t(q);
        if (tetSolve(s, dt, relax, t, s.tetLambda[q], newLambda, c)) {
            s.tetLambda[q] = newLambda;
#pragma unroll
            for (int k = 0; k < 4; ++k) rec[k] = c[k];
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) c[k] = rec[k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) moveRecord(s, gaussSeidel, t.particle_indices[k], c[k]);
    }
}

// Colour position q of family kFam: the colour-ordered edges and tets where the scene holds them,
// else the constraint the colour order names.
template <uint32_t kFam>
__device__ __forceinline__ void colourAt(const Scene &s, float dt, float relax, bool gaussSeidel, uint32_t q)
{
    if constexpr (kFam == kFamEdges) {
        if (s.edgesC) {
            colourConstraintOrdered<kFamEdges>(s, dt, relax, gaussSeidel, q);
            return;
        }
    } else if constexpr (kFam == kFamTets) {
        if (s.tetsC) {
            colourConstraintOrdered<kFamTets>(s, dt, relax, gaussSeidel, q);
            return;
        }
    }
    colourConstraint<kFam>(s, dt, relax, gaussSeidel, s.colOrder[kFam][q]);
}

// End of a colour-Jacobi family: x += the family's sum (particles with invMass > kEps), sum
// cleared; for joints the orientation sum, then the normalisation every segment gets.
__device__ __forceinline__ void colourJacobiApplyAt(const Scene &s, uint32_t i)
{
    const float4 a = s.softAcc[i];
    s.softAcc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 p = s.x[i];
    if (p.w > kEps) s.x[i] = mk4(xyz(p) + xyz(a), p.w);
}

__device__ __forceinline__ void colourJacobiOrientAt(const Scene &s, uint32_t g)
{
    const float4 a = s.orientAcc[g];
    s.orientAcc[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.segOrient[g] = qNormalize(add4(s.segOrient[g], a));
}

template <uint32_t kFam, bool kGaussSeidel>
__global__ void __launch_bounds__(kThreads) k_colourSolve(Scene s, float dt, float relax, uint32_t begin, uint32_t end)
{
    pdlEnter();
    const uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (k < end) colourAt<kFam>(s, dt, relax, kGaussSeidel, k);
}

__global__ void __launch_bounds__(kThreads) k_colourJacobiApply(Scene s, uint2 win)
{
    pdlEnter();
    const uint32_t i = win.x + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < win.y) colourJacobiApplyAt(s, i);
}

__global__ void __launch_bounds__(kThreads) k_colourJacobiOrient(Scene s)
{
    pdlEnter();
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < s.S) colourJacobiOrientAt(s, g);
}

__host__ __device__ __forceinline__ uint32_t familySize(const Scene &s, uint32_t fam)
{
    return fam == kFamEdges ? s.E
         : fam == kFamSegments ? s.S
         : fam == kFamBends ? s.Bn + s.D
         : fam == kFamJoints ? s.J
         : fam == kFamDistances ? s.SD
         : s.T;
}

// The particles a family's colour-Jacobi sum can touch (strand distances share the strand
// segments' particles).
__host__ __device__ __forceinline__ uint2 familyWindow(const Scene &s, uint32_t fam)
{
    return fam == kFamEdges ? s.edgeWin
         : fam == kFamBends ? s.bendWin
         : fam == kFamTets ? s.tetWin
         : s.segWin;
}

template <uint32_t kFam>
void launchColourFamily(const Scene &s, float dt, float relax, const XpbdPlan &plan, cudaStream_t st)
{
    if (familySize(s, kFam) == 0) return;
    const bool gs = plan.schedule == CN_XPBD_COLOUR_GAUSS_SEIDEL;
    const uint32_t *starts = plan.hostStarts[kFam];
    for (uint32_t k = 0; k < plan.colours[kFam]; ++k) {
        const uint32_t b = starts[k], e = starts[k + 1];
        if (e <= b) continue;
        if (gs) launchPdl(k_colourSolve<kFam, true>, softBlocksFor(e - b), softThreads(s), st, s, dt, relax, b, e);
        else launchPdl(k_colourSolve<kFam, false>, softBlocksFor(e - b), softThreads(s), st, s, dt, relax, b, e);
    }
    if (gs) return;
    if (kFam == kFamJoints) {
        launchPdl(k_colourJacobiOrient, softBlocksFor(s.S), softThreads(s), st, s);
    } else {
        const uint2 win = familyWindow(s, kFam);
        if (win.y > win.x) launchPdl(k_colourJacobiApply, softBlocksFor(win.y - win.x), softThreads(s), st, s, win);
    }
}

// ------------------------------------------------------------------------------------------
// Fused iterations: one thread-block cluster, every iteration of the substep
// ------------------------------------------------------------------------------------------
// The phases of the per-phase kernels (family solve, family apply, particle-rigid contacts), each
// a loop of the cluster's threads over its elements, separated by cluster barriers: the
// barrier's release / acquire at cluster scope orders every global write of a phase before
// every read of the next.  Each element is computed by the same device function as in the
// per-phase kernels, so the results are the same bit for bit.  Every thread passes every barrier
// (the loops' trip counts are uniform), and nothing waits on anything but the barriers.
constexpr uint32_t kFusedThreads = 512u;
constexpr uint32_t kFusedMaxCtas = 16u;

struct FusedPlan {
    uint32_t iterations, softIterations, contactIterations, rigid;
    uint32_t colours[kFamilies];
    const uint32_t *starts[kFamilies];
};

template <uint32_t kFam, uint32_t kSchedule>
__device__ __forceinline__ void fusedFamily(const Scene &s, float dt, float relax, const FusedPlan &plan,
                                            uint32_t tid, uint32_t nth)
{
    namespace cg = cooperative_groups;
    const uint32_t n = familySize(s, kFam);
    if (n == 0u) return;
    if constexpr (kSchedule == CN_XPBD_GATHER) {
        for (uint32_t c = tid; c < n; c += nth) {
            if constexpr (kFam == kFamEdges) solveEdge(s, dt, relax, c);
            else if constexpr (kFam == kFamSegments) solveSegmentAt(s, dt, relax, c);
            else if constexpr (kFam == kFamBends) {
                if (c < s.Bn) solveBendAt(s, dt, relax, c);
                else solveDihedralAt(s, dt, relax, c - s.Bn);
            } else if constexpr (kFam == kFamJoints) solveJointAt(s, dt, relax, c);
            else if constexpr (kFam == kFamDistances) solveDistanceAt(s, dt, relax, c);
            else solveTet(s, dt, relax, c);
        }
        cg::this_cluster().sync();
        if constexpr (kFam == kFamEdges) {
            for (uint32_t i = s.edgeWin.x + tid; i < s.edgeWin.y; i += nth)
                applyGatherAt(s, s.edgeRanges, s.edgeCorr, i);
        } else if constexpr (kFam == kFamSegments) {
            const uint32_t m = segmentApplyThreads(s);
            for (uint32_t i = tid; i < m; i += nth) applySegmentsAt(s, i);
        } else if constexpr (kFam == kFamBends) {
            for (uint32_t i = s.bendWin.x + tid; i < s.bendWin.y; i += nth)
                applyGatherAt(s, s.bendRanges, s.bendCorr, i);
        } else if constexpr (kFam == kFamJoints) {
            for (uint32_t g = tid; g < s.S; g += nth) applyJointsAt(s, g);
        } else if constexpr (kFam == kFamDistances) {
            for (uint32_t i = s.segWin.x + tid; i < s.segWin.y; i += nth)
                applyGatherAt(s, s.segRanges, s.distCorr, i);
        } else {
            for (uint32_t i = s.tetWin.x + tid; i < s.tetWin.y; i += nth)
                applyGatherAt(s, s.tetRanges, s.tetCorr, i);
        }
        cg::this_cluster().sync();
    } else {
        constexpr bool gs = kSchedule == CN_XPBD_COLOUR_GAUSS_SEIDEL;
        const uint32_t *starts = plan.starts[kFam];
        for (uint32_t k = 0; k < plan.colours[kFam]; ++k) {
            const uint32_t b = starts[k], e = starts[k + 1];
            for (uint32_t j = b + tid; j < e; j += nth) colourAt<kFam>(s, dt, relax, gs, j);
            cg::this_cluster().sync();
        }
        if constexpr (!gs) {
            if constexpr (kFam == kFamJoints) {
                for (uint32_t g = tid; g < s.S; g += nth) colourJacobiOrientAt(s, g);
            } else {
                const uint2 win = familyWindow(s, kFam);
                for (uint32_t i = win.x + tid; i < win.y; i += nth) colourJacobiApplyAt(s, i);
            }
            cg::this_cluster().sync();
        }
    }
}

template <uint32_t kSchedule>
__global__ void __launch_bounds__(kFusedThreads, 1) k_fusedIterations(Scene s, Config cfg, float dt, FusedPlan plan)
{
    namespace cg = cooperative_groups;
    const cg::cluster_group cl = cg::this_cluster();
    const uint32_t tid = cl.block_rank() * blockDim.x + threadIdx.x;
    const uint32_t nth = cl.num_blocks() * blockDim.x;
    const float relax = cfg.softInternalRelaxation;
    for (uint32_t it = 0; it < plan.iterations; ++it) {
        if (it < plan.softIterations) {
            fusedFamily<kFamEdges, kSchedule>(s, dt, relax, plan, tid, nth);
            fusedFamily<kFamSegments, kSchedule>(s, dt, relax, plan, tid, nth);
            fusedFamily<kFamBends, kSchedule>(s, dt, relax, plan, tid, nth);
            fusedFamily<kFamJoints, kSchedule>(s, dt, relax, plan, tid, nth);
            fusedFamily<kFamDistances, kSchedule>(s, dt, relax, plan, tid, nth);
            fusedFamily<kFamTets, kSchedule>(s, dt, relax, plan, tid, nth);
        }
        if (plan.rigid != 0u && it < plan.contactIterations) {
            for (uint32_t i = tid; i < s.N; i += nth) rigidContactsAt(s, cfg, true, i);
            cl.sync();
        }
    }
}

// A batch tick's iterations as one persistent kernel: each thread-block cluster takes the next
// stepped scene from a device counter and runs every iteration of the substep on it (edge and
// tet families in the gather schedule, then the particle-rigid contacts), its phases separated
// by cluster barriers, so one scene's records and positions stay on chip across the iterations
// instead of the whole pool streaming through HBM once per phase.  Per element the same device
// functions as the per-phase batch kernels: bit-identical results.  The scene index is taken by
// one thread and handed to the cluster through its shared memory between two barriers, so the
// loop's trip count is uniform over the cluster.
constexpr uint32_t kBatchFusedThreads = 256u;

__global__ void __launch_bounds__(kBatchFusedThreads, 2) k_batchFusedIterations(Scene s, Config cfg, float dt,
                                                                           BatchFusedPlan plan)
{
    namespace cg = cooperative_groups;
    const cg::cluster_group cl = cg::this_cluster();
    __shared__ uint32_t taken;
    const uint32_t tid = cl.block_rank() * blockDim.x + threadIdx.x;
    const uint32_t nth = cl.num_blocks() * blockDim.x;
    const uint32_t count = *plan.sceneCount;
    const float relax = cfg.softInternalRelaxation;
    for (;;) {
        if (cl.block_rank() == 0u && threadIdx.x == 0u) taken = atomicAdd(plan.next, 1u);
        cl.sync();
        const uint32_t j = *cl.map_shared_rank(&taken, 0);
        cl.sync(); // every thread has its copy before the leader takes the next one
        if (j >= count) break;
        const uint2 pr = plan.scenes[kSceneListStride * j], er = plan.scenes[kSceneListStride * j + 1u],
                    tr = plan.scenes[kSceneListStride * j + 2u];
        for (uint32_t it = 0; it < plan.iterations; ++it) {
            if ((s.E || s.T) && it < plan.softIterations) {
                if (s.E) {
                    for (uint32_t e = er.x + tid; e < er.y; e += nth) solveEdge(s, dt, relax, e);
                    cl.sync();
                    for (uint32_t i = pr.x + tid; i < pr.y; i += nth) applyGatherAt(s, s.edgeRanges, s.edgeCorr, i);
                    cl.sync();
                }
                if (s.T) {
                    for (uint32_t t = tr.x + tid; t < tr.y; t += nth) solveTet(s, dt, relax, t);
                    cl.sync();
                    for (uint32_t i = pr.x + tid; i < pr.y; i += nth) applyGatherAt(s, s.tetRanges, s.tetCorr, i);
                    cl.sync();
                }
            }
            if (it < plan.contactIterations) {
                for (uint32_t i = pr.x + tid; i < pr.y; i += nth) rigidContactsAt(s, cfg, true, i);
                cl.sync();
            }
        }
    }
}

template <uint32_t kSchedule> cudaError_t fusedLaunch(const Scene &s, const Config &c, float dt, const FusedPlan &plan,
                                                     const FusedShape &shape, cudaStream_t st)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(shape.ctas, 1, 1);
    cfg.blockDim = dim3(shape.threads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = shape.ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_fusedIterations<kSchedule>, s, c, dt, plan);
}

// Grid of an apply pass: the batch's work list, else the family's particle window.
inline unsigned applyGrid(const Scene &s, uint2 win)
{
    return s.wP.tiles ? gridFor(s.wP, s.N) : blocksFor(win.y > win.x ? win.y - win.x : 0u);
}


bool launchSoftIteration(const Scene &s, float dt, const Config &c, const XpbdPlan &plan, cudaStream_t st,
                         bool rigidContacts)
{
    if (plan.schedule == CN_XPBD_GATHER) return launchSoftIteration(s, dt, c, st, rigidContacts);
    const float relax = c.softInternalRelaxation;
    launchColourFamily<kFamEdges>(s, dt, relax, plan, st);
    launchColourFamily<kFamSegments>(s, dt, relax, plan, st);
    launchColourFamily<kFamBends>(s, dt, relax, plan, st);
    launchColourFamily<kFamJoints>(s, dt, relax, plan, st);
    launchColourFamily<kFamDistances>(s, dt, relax, plan, st);
    launchColourFamily<kFamTets>(s, dt, relax, plan, st);
    return false;
}

FusedShape fusedIterationsShape()
{
    // one CTA per SM, as many SMs as one cluster may span (16 where the device allows the
    // non-portable size, else the portable 8)
    FusedShape out;
    const void *fns[3] = {reinterpret_cast<const void *>(&k_fusedIterations<CN_XPBD_GATHER>),
                          reinterpret_cast<const void *>(&k_fusedIterations<CN_XPBD_COLOUR_JACOBI>),
                          reinterpret_cast<const void *>(&k_fusedIterations<CN_XPBD_COLOUR_GAUSS_SEIDEL>)};
    for (const void *f : fns)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return out;
        }
    for (uint32_t ctas : {kFusedMaxCtas, 8u}) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(ctas, 1, 1);
        cfg.blockDim = dim3(kFusedThreads, 1, 1);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        bool ok = true;
        for (const void *f : fns) {
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, f, &cfg) != cudaSuccess || clusters < 1) {
                cudaGetLastError();
                ok = false;
                break;
            }
        }
        if (ok) {
            out.ctas = ctas;
            out.threads = kFusedThreads;
            return out;
        }
    }
    return out;
}

void launchFusedIterations(const Scene &s, const Config &c, float dt, const XpbdPlan &plan, uint32_t iterations,
                           uint32_t softIterations, uint32_t contactIterations, bool rigid, const FusedShape &shape,
                           cudaStream_t st)
{
    FusedPlan fp{};
    fp.iterations = iterations;
    fp.softIterations = softIterations;
    fp.contactIterations = contactIterations;
    fp.rigid = rigid ? 1u : 0u;
    for (uint32_t f = 0; f < kFamilies; ++f) {
        fp.colours[f] = plan.schedule == CN_XPBD_GATHER ? 0u : plan.colours[f];
        fp.starts[f] = plan.devStarts[f];
    }
    if (plan.schedule == CN_XPBD_COLOUR_JACOBI) fusedLaunch<CN_XPBD_COLOUR_JACOBI>(s, c, dt, fp, shape, st);
    else if (plan.schedule == CN_XPBD_COLOUR_GAUSS_SEIDEL) fusedLaunch<CN_XPBD_COLOUR_GAUSS_SEIDEL>(s, c, dt, fp, shape, st);
    else fusedLaunch<CN_XPBD_GATHER>(s, c, dt, fp, shape, st);
}

// Scatters an admitted scene's upload image into its pool ranges, rebasing every index field:
// particle indices by p0, incidence positions by ei0 / ti0, bodies by b0, colliders by c0, body
// collider lists by ci0, materials by m0 (the host rebasing of cn_batch_add_scene, on the device).
__global__ void __launch_bounds__(kThreads) k_admitScene(Scene s, AdmitImage a)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    auto seg = [&](uint32_t k) { return a.img + a.off[k]; };
    auto f4 = [&](uint32_t k) { return reinterpret_cast<const float4 *>(seg(k)); };
    auto u32 = [&](uint32_t k) { return reinterpret_cast<const uint32_t *>(seg(k)); };
    auto u2 = [&](uint32_t k) { return reinterpret_cast<const uint2 *>(seg(k)); };
    if (i < a.N) {
        const uint32_t p = a.p0 + i;
        const float4 x = f4(kAdmX)[i];
        s.x[p] = x;
        s.v[p] = f4(kAdmV)[i];
        s.xprev[p] = make_float4(x.x, x.y, x.z, 0.0f);
        const_cast<float *>(s.radii)[p] = reinterpret_cast<const float *>(seg(kAdmRadii))[i];
        const_cast<uint32_t *>(s.kinds)[p] = u32(kAdmKinds)[i];
        const_cast<uint4 *>(s.meta)[p] = reinterpret_cast<const uint4 *>(seg(kAdmMeta))[i];
        const_cast<uint32_t *>(s.matIdx)[p] = u32(kAdmMatIdx)[i] + a.m0;
        const_cast<uint32_t *>(s.fluidMatIdx)[p] = 0u;
        const uint32_t ot = u32(kAdmOwnerTypes)[i];
        const_cast<uint32_t *>(s.ownerTypes)[p] = ot;
        const_cast<uint32_t *>(s.ownerIdx)[p] = u32(kAdmOwnerIdx)[i] + (ot == CN_OWNER_RIGID_BODY ? a.b0 : 0u);
        const uint2 er = u2(kAdmEdgeRanges)[i], tr = u2(kAdmTetRanges)[i];
        const_cast<uint2 *>(s.edgeRanges)[p] = make_uint2(er.x + a.ei0, er.y);
        const_cast<uint2 *>(s.tetRanges)[p] = make_uint2(tr.x + a.ti0, tr.y);
        const_cast<uint2 *>(s.pColRange)[p] = make_uint2(a.c0, a.c0 + a.queryCount);
    }
    // a scene starts with zero correction records, as a solver's freshly cleared arena
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    auto edgeAt = [&](uint32_t k) {
        cn_soft_edge e = reinterpret_cast<const cn_soft_edge *>(seg(kAdmEdges))[k];
        e.particle_a += a.p0;
        e.particle_b += a.p0;
        return e;
    };
    auto tetAt = [&](uint32_t k) {
        cn_soft_tet t = reinterpret_cast<const cn_soft_tet *>(seg(kAdmTets))[k];
        for (int j = 0; j < 4; ++j) t.particle_indices[j] += a.p0;
        return t;
    };
    if (i < a.E) {
        const_cast<PackedEdge *>(s.edgesP)[a.e0 + i] = packEdge(edgeAt(i));
        const uint2 d = u2(kAdmEdgeDst)[i];
        reinterpret_cast<uint2 *>(const_cast<uint32_t *>(s.edgeDst))[a.e0 + i] =
            make_uint2(d.x == kNoSlot ? kNoSlot : d.x + a.ei0, d.y == kNoSlot ? kNoSlot : d.y + a.ei0);
        s.edgeCorr[a.ei0 + 2u * i] = zero4;
        s.edgeCorr[a.ei0 + 2u * i + 1u] = zero4;
    }
    if (i < a.T) {
        const_cast<cn_soft_tet *>(s.tets)[a.t0 + i] = tetAt(i);
        const uint4 d = reinterpret_cast<const uint4 *>(seg(kAdmTetDst))[i];
        auto rb = [&](uint32_t v) { return v == kNoSlot ? kNoSlot : v + a.ti0; };
        reinterpret_cast<uint4 *>(const_cast<uint32_t *>(s.tetDst))[a.t0 + i] = make_uint4(rb(d.x), rb(d.y), rb(d.z), rb(d.w));
        for (uint32_t k = 0; k < 4u; ++k) s.tetCorr[a.ti0 + 4u * i + k] = zero4;
    }
    if (i < a.M) const_cast<float4 *>(s.contactMaterials)[a.m0 + i] = f4(kAdmMaterials)[i];
    if (i < a.B) {
        const uint32_t b = a.b0 + i;
        s.bodyPos[b] = f4(kAdmBodyPos)[i];
        s.bodyRot[b] = f4(kAdmBodyRot)[i];
        s.bodyLin[b] = f4(kAdmBodyLin)[i];
        s.bodyAng[b] = f4(kAdmBodyAng)[i];
        const_cast<float4 *>(s.bodyScale)[b] = f4(kAdmBodyScale)[i];
        const_cast<float4 *>(s.bodyInvInertia)[b] = f4(kAdmBodyInvI)[i];
        const_cast<uint32_t *>(s.bodyType)[b] = u32(kAdmBodyType)[i];
        s.bodyKinPos[b] = f4(kAdmKinPos)[i];
        s.bodyKinRot[b] = f4(kAdmKinRot)[i];
        s.bodyKinFlags[b] = u32(kAdmKinFlags)[i];
        const uint2 r = u2(kAdmBodyColRanges)[i];
        const_cast<uint2 *>(s.bodyColRanges)[b] = make_uint2(r.x + a.ci0, r.y);
    }
    if (i < a.CI) const_cast<uint32_t *>(s.bodyColIdx)[a.ci0 + i] = u32(kAdmBodyColIdx)[i] + a.c0;
    if (i < a.C) {
        const uint32_t c = a.c0 + i;
        const_cast<cn_collider_geometry *>(s.colGeo)[c] = reinterpret_cast<const cn_collider_geometry *>(seg(kAdmColGeo))[i];
        cn_collider_broadphase bp = reinterpret_cast<const cn_collider_broadphase *>(seg(kAdmColBp))[i];
        bp.owner_body += a.b0;
        const_cast<cn_collider_broadphase *>(s.colBp)[c] = bp;
        const_cast<float4 *>(s.colMat)[c] = f4(kAdmColMat)[i];
    }
    if (i < a.queryCount) const_cast<uint32_t *>(s.colQueryOrder)[a.c0 + i] = u32(kAdmQueryOrder)[i] + a.c0;
    if (a.colWords) { // the colour-ordered copies, colour tables and records
        if (i < a.E) const_cast<PackedEdge *>(s.edgesC)[a.e0 + i] = packEdge(edgeAt(u32(kAdmEdgeColOrder)[i]));
        if (i < a.T) {
            const_cast<cn_soft_tet *>(s.tetsC)[a.t0 + i] = tetAt(u32(kAdmTetColOrder)[i]);
            for (uint32_t k = 0; k < 4u; ++k) s.tetRecC[4u * (size_t(a.t0) + i) + k] = zero4;
        }
        if (i < a.colWords) s.batchColStarts[a.k0 + i] = u32(kAdmColStarts)[i];
    }
}

void launchAdmitScene(const Scene &s, const AdmitImage &a, cudaStream_t st)
{
    const uint32_t n = std::max({a.N, a.E, a.T, a.B, a.C, a.CI, a.M, a.queryCount, a.colWords, 1u});
    k_admitScene<<<blocksFor(n), kThreads, 0, st>>>(s, a);
}

// The blocks of a batch colour pass: `chunks` blocks per stepped scene (the grid split evenly),
// block w taking scene w / chunks and every chunks-th stride of its range.
template <class F>
__device__ __forceinline__ void forSceneChunks(const uint32_t *sceneCount, F &&f)
{
    const uint32_t n = *sceneCount;
    if (n == 0u) return;
    const uint32_t chunks = max(gridDim.x / n, 1u);
    for (uint32_t w = blockIdx.x; w < n * chunks; w += gridDim.x) f(w / chunks, w % chunks, chunks);
}

// Colour k of one family over a batch tick's stepped scenes: each scene's colour-k range of its
// colour-ordered constraints (contiguous), scenes with fewer colours skipped.
template <uint32_t kFam, bool kGaussSeidel>
__global__ void __launch_bounds__(kThreads) k_colourSolveBatch(Scene s, float dt, float relax, uint32_t k,
                                                               const uint2 *scenes, const uint32_t *sceneCount)
{
    pdlEnter();
    forSceneChunks(sceneCount, [&](uint32_t j, uint32_t part, uint32_t chunks) {
        const uint2 range = scenes[kSceneListStride * j + (kFam == kFamEdges ? 1u : 2u)];
        const uint2 bases = scenes[kSceneListStride * j + 3u];
        const uint32_t *words = s.batchColStarts + (kFam == kFamEdges ? bases.x : bases.y);
        if (k >= words[0]) return;
        const uint32_t *starts = words + kColWordsHeader;
        const uint32_t b = range.x + starts[k], e = range.x + starts[k + 1u];
        for (uint32_t q = b + part * blockDim.x + threadIdx.x; q < e; q += chunks * blockDim.x)
            colourConstraintOrdered<kFam>(s, dt, relax, kGaussSeidel, q);
    });
}

// End of a batch colour-Jacobi family: each stepped scene's sums added over the family's window.
template <uint32_t kFam>
__global__ void __launch_bounds__(kThreads) k_colourJacobiApplyBatch(Scene s, const uint2 *scenes,
                                                                     const uint32_t *sceneCount)
{
    pdlEnter();
    forSceneChunks(sceneCount, [&](uint32_t j, uint32_t part, uint32_t chunks) {
        const uint32_t p0 = scenes[kSceneListStride * j].x;
        const uint2 bases = scenes[kSceneListStride * j + 3u];
        const uint32_t *words = s.batchColStarts + (kFam == kFamEdges ? bases.x : bases.y);
        if (words[0] == 0u) return;
        const uint32_t b = p0 + words[1], e = p0 + words[2];
        for (uint32_t i = b + part * blockDim.x + threadIdx.x; i < e; i += chunks * blockDim.x)
            colourJacobiApplyAt(s, i);
    });
}

template <uint32_t kFam>
void launchBatchColourFamily(const Scene &s, float dt, float relax, bool gs, uint32_t colours, const uint2 *scenes,
                             const uint32_t *sceneCount, uint32_t grid, cudaStream_t st)
{
    if ((kFam == kFamEdges ? s.E : s.T) == 0u) return;
    for (uint32_t k = 0; k < colours; ++k) {
        if (gs) launchPdl(k_colourSolveBatch<kFam, true>, grid, kThreads, st, s, dt, relax, k, scenes, sceneCount);
        else launchPdl(k_colourSolveBatch<kFam, false>, grid, kThreads, st, s, dt, relax, k, scenes, sceneCount);
    }
    if (!gs) launchPdl(k_colourJacobiApplyBatch<kFam>, grid, kThreads, st, s, scenes, sceneCount);
}

void launchBatchColourIteration(const Scene &s, float dt, const Config &c, uint32_t schedule, const uint32_t maxColours[2],
                                const uint2 *scenes, const uint32_t *sceneCount, uint32_t grid, cudaStream_t st)
{
    const bool gs = schedule == CN_XPBD_COLOUR_GAUSS_SEIDEL;
    const float relax = c.softInternalRelaxation;
    launchBatchColourFamily<kFamEdges>(s, dt, relax, gs, maxColours[0], scenes, sceneCount, grid, st);
    launchBatchColourFamily<kFamTets>(s, dt, relax, gs, maxColours[1], scenes, sceneCount, grid, st);
}

uint32_t batchFusedClusters(uint32_t ctas)
{
    if (ctas == 0u || ctas > 8u) return 0u;
    if (cudaFuncSetAttribute(reinterpret_cast<const void *>(&k_batchFusedIterations),
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0u;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(ctas, 1, 1);
    cfg.blockDim = dim3(kBatchFusedThreads, 1, 1);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, reinterpret_cast<const void *>(&k_batchFusedIterations), &cfg) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0u;
    }
    return clusters > 0 ? uint32_t(clusters) : 0u;
}

void launchBatchFusedIterations(const Scene &s, const Config &c, float dt, const BatchFusedPlan &plan, uint32_t ctas,
                                uint32_t clusters, cudaStream_t st)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(ctas * clusters, 1, 1);
    cfg.blockDim = dim3(kBatchFusedThreads, 1, 1);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_batchFusedIterations, s, c, dt, plan);
}

bool launchSoftIteration(const Scene &s, float dt, const Config &c, cudaStream_t st, bool rigidContacts)
{
    return launchSoftFamilies(s, dt, c, st, kAllFamilies, rigidContacts);
}

bool launchSoftFamilies(const Scene &s, float dt, const Config &c, cudaStream_t st, uint32_t families,
                        bool rigidContacts)
{
    const float relax = c.softInternalRelaxation;
    auto on = [&](uint32_t f) { return ((families >> f) & 1u) != 0u; };
    if (s.E && on(kFamEdges)) {
        launchPdl(k_solveEdges, softGridFor(s.wE, s.E), softThreads(s), st, s, dt, relax);
        launchPdl(k_applyGather, softApplyGrid(s, s.edgeWin), softThreads(s), st, s, s.edgeRanges, s.edgeCorr, s.edgeWin);
    }
    if (s.S && on(kFamSegments)) {
        launchPdl(k_solveSegments, softBlocksFor(s.S), softThreads(s), st, s, dt, relax);
        launchPdl(k_applySegments, softBlocksFor(segmentApplyThreads(s)), softThreads(s), st, s);
    }
    if ((s.Bn || s.D) && on(kFamBends)) {
        if (s.Bn) launchPdl(k_solveBends, softBlocksFor(s.Bn), softThreads(s), st, s, dt, relax);
        if (s.D) launchPdl(k_solveDihedrals, softBlocksFor(s.D), softThreads(s), st, s, dt, relax);
        launchPdl(k_applyGather, softApplyGrid(s, s.bendWin), softThreads(s), st, s, s.bendRanges, s.bendCorr, s.bendWin);
    }
    if (s.J && on(kFamJoints)) {
        launchPdl(k_solveJoints, softBlocksFor(s.J), softThreads(s), st, s, dt, relax);
        launchPdl(k_applyJoints, softBlocksFor(s.S), softThreads(s), st, s);
    }
    if (s.SD && on(kFamDistances)) {
        launchPdl(k_solveDistances, softBlocksFor(s.SD), softThreads(s), st, s, dt, relax);
        launchPdl(k_applyGather, softApplyGrid(s, s.segWin), softThreads(s), st, s, s.segRanges, s.distCorr, s.segWin);
    }
    if (s.T && on(kFamTets)) {
        launchPdl(k_solveTets, softGridFor(s.wT, s.T), softThreads(s), st, s, dt, relax);
        if (rigidContacts && s.N) {
            launchPdl(k_applyTetsRigidContacts, softGridFor(s.wP, s.N), softThreads(s), st, s, c);
            return true;
        }
        launchPdl(k_applyGather, softApplyGrid(s, s.tetWin), softThreads(s), st, s, s.tetRanges, s.tetCorr, s.tetWin);
    }
    return false;
}

void launchContacts(const Scene &s, const Config &c, bool particleContacts, bool rigidContacts,
                    cudaStream_t st)
{
    if (particleContacts) {
        const uint32_t cap = s.particlePairCapacity;
        launchPdl(k_particleContacts, pairGrid(cap), kThreads, st, s, c);
    }
    if (rigidContacts) launchPdl(k_rigidContacts, softGridFor(s.wP, s.N), softThreads(s), st, s, c, !particleContacts);
    if (particleContacts) launchPdl(k_applyPositionCorrections, blocksFor(s.N), kThreads, st, s);
}

void launchUpdateVelocities(const Scene &s, float dt, const float4 *fluidDelta, cudaStream_t st)
{
    if (s.N == 0) return;
    launchPdl(k_updateVelocities, gridFor(s.wP, s.N), kThreads, st, s, dt, fluidDelta);
}

void launchFluidBoundaryVelocities(const Scene &s, float dt, const Config &c, cudaStream_t st)
{
    if (s.N == 0 || s.colQueryCount == 0) return;
    k_fluidBoundaryVelocities<<<blocksFor(s.N), kThreads, 0, st>>>(s, dt, c);
}

void launchRigidContactVelocities(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st)
{
    if (s.N == 0 || iterations == 0) return;
    k_rigidContactVelocities<<<gridFor(s.wP, s.N), kThreads, 0, st>>>(s, iterations, c);
}

void launchApplyRigidCorrections(const Scene &s, const Config &c, cudaStream_t st)
{
    if (s.B == 0) return;
    k_applyRigidCorrections<<<blocksFor(s.B), kThreads, 0, st>>>(s, c);
}

void launchUpdateRigidVelocities(const Scene &s, float dt, cudaStream_t st)
{
    if (s.B == 0) return;
    k_updateRigidVelocities<<<blocksFor(s.B), kThreads, 0, st>>>(s, dt);
}

void launchRigidContactVelocitiesDynamic(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st)
{
    for (uint32_t it = 0; it < iterations; ++it) {
        if (s.N) k_rigidContactVelocityStep<<<gridFor(s.wP, s.N), kThreads, 0, st>>>(s, c);
        if (s.B) k_applyRigidContactVelocities<<<blocksFor(s.B), kThreads, 0, st>>>(s, c);
    }
}

void launchParticleContactVelocities(const Scene &s, uint32_t iterations, const Config &c, cudaStream_t st)
{
    for (uint32_t it = 0; it < iterations; ++it) {
        k_particleContactVelocities<<<pairGrid(s.particlePairCapacity), kThreads, 0, st>>>(s, c);
        k_applyContactVelocities<<<blocksFor(s.N), kThreads, 0, st>>>(s);
        // the bodies' sums (only proxies of dynamic bodies add to them)
        if (s.hasDynamic && s.nProxy) k_applyRigidContactVelocities<<<blocksFor(s.B), kThreads, 0, st>>>(s, c);
    }
}

// physics_particle_sync_rigid_proxy_particles.cs.hlsl after the bodies' corrections
__global__ void __launch_bounds__(kThreads) k_syncRigidProxies(Scene s)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nProxy) return;
    s.x[i] = mk4(proxyWorldPosition(s, i), s.x[i].w);
}

void launchSyncRigidProxies(const Scene &s, cudaStream_t st)
{
    if (s.nProxy) k_syncRigidProxies<<<blocksFor(s.nProxy), kThreads, 0, st>>>(s);
}

void launchSurfaceRender(const Scene &s, cudaStream_t st)
{
    const uint32_t vt = s.surfV > s.surfT ? s.surfV : s.surfT;
    if (vt) k_surfaceSkinTriangles<<<blocksFor(vt), kThreads, 0, st>>>(s);
    if (s.surfV) k_surfaceVertexNormals<<<blocksFor(s.surfV), kThreads, 0, st>>>(s);
    if (s.surfS) {
        if (s.surfChunks) k_surfaceChunkBounds<<<blocksFor(size_t(s.surfChunks) * 32u), kThreads, 0, st>>>(s);
        k_surfaceWorldBounds<<<blocksFor(size_t(s.surfS) * 32u), kThreads, 0, st>>>(s);
    }
}

void launchExportCellRanges(const Scene &s, uint4 *out, uint32_t capacity, uint32_t *scanTmp,
                            size_t, cudaStream_t st)
{
    if (s.N == 0) return;
    uint32_t *flags = scanTmp;
    uint32_t *offsets = scanTmp + s.N;
    uint32_t *total = scanTmp + 2 * size_t(s.N);
    k_runFlags<<<blocksFor(s.N), kThreads, 0, st>>>(s, flags);
    exclusiveScan(flags, offsets, s.N, total, total + 1, st);
    k_runCompact<<<blocksFor(s.N), kThreads, 0, st>>>(s, flags, offsets, out, capacity);
}

} // namespace cn
