// cn_rigid.cu -- rigid-rigid contacts of scenes with dynamic bodies (sm_100a).
//
// Per substep: an LBVH (Karras 2012: Morton codes of the AABB centres, the onesweep key sort,
// one thread per internal node to find its range and split, bottom-up refit where the second
// child to arrive builds the parent box) over the colliders' world AABBs; every moving collider
// walks it for its candidate pairs (count, scan, emit: a deterministic order); one thread per
// pair runs the narrow phase.  The contacts are then grouped by body pair (stable key sort)
// for the velocity solve, and depenetrated every position iteration.  Reference shaders:
// physics/rigid/broad_phase/, narrow_phase/physics_rigid_generate_contacts.cs.hlsl,
// solver/physics_rigid_depenetrate_contacts, init_contact_velocities, solve_contact_velocities.
#include <cstdint>
#include <cuda_runtime.h>

#include "cn_device.h"
#include "cn_math.cuh"

namespace cn {
namespace {

constexpr int kRigidThreads = 128;
constexpr uint32_t kBvhStack = 128; // the reference's traversal stack; deeper nodes are dropped

inline unsigned blocksOf(size_t n) { return n == 0 ? 1u : unsigned((n + kRigidThreads - 1) / kRigidThreads); }

__device__ __forceinline__ bool broadPhaseCollide(const cn_collider_broadphase &a, const cn_collider_broadphase &b)
{
    // ShouldBroadPhaseCollide (physics_shape_common.hlsli:12-21)
    if (a.environment_index != b.environment_index) return false;
    return (a.collision_mask & b.collision_layer) != 0u && (b.collision_mask & a.collision_layer) != 0u;
}

// ------------------------------------------------------------------------------------- LBVH
// Scene bounds of the AABB centres (physics_rigid_reduce_extent_*): one block.
constexpr int kBoundsThreads = 1024; // one block: every collider's centre in a few strides
__global__ void __launch_bounds__(kBoundsThreads) k_bvhBounds(Scene s)
{
    __shared__ float lo[3][kBoundsThreads], hi[3][kBoundsThreads];
    f3 mn{3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f}, mxv{-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (uint32_t k = threadIdx.x; k < s.colQueryCount; k += blockDim.x) {
        const uint32_t c = s.colQueryOrder[k];
        const f3 ctr = (xyz(s.colAabbMin[c]) + xyz(s.colAabbMax[c])) * 0.5f;
        mn = min3(mn, ctr);
        mxv = max3(mxv, ctr);
    }
    lo[0][threadIdx.x] = mn.x; lo[1][threadIdx.x] = mn.y; lo[2][threadIdx.x] = mn.z;
    hi[0][threadIdx.x] = mxv.x; hi[1][threadIdx.x] = mxv.y; hi[2][threadIdx.x] = mxv.z;
    __syncthreads();
    for (uint32_t st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int a = 0; a < 3; ++a) {
                lo[a][threadIdx.x] = fminf(lo[a][threadIdx.x], lo[a][threadIdx.x + st]);
                hi[a][threadIdx.x] = fmaxf(hi[a][threadIdx.x], hi[a][threadIdx.x + st]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        s.bvhBounds[0] = make_float4(lo[0][0], lo[1][0], lo[2][0], 0.f);
        s.bvhBounds[1] = make_float4(hi[0][0], hi[1][0], hi[2][0], 0.f);
    }
}

__device__ __forceinline__ uint32_t expandBits10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// physics_rigid_morton_codes.cs.hlsl: 30-bit code of the normalised AABB centre
__global__ void k_bvhMorton(Scene s)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= s.colQueryCount) return;
    const uint32_t c = s.colQueryOrder[k];
    const f3 lo = xyz(s.bvhBounds[0]), hi = xyz(s.bvhBounds[1]);
    const f3 ctr = (xyz(s.colAabbMin[c]) + xyz(s.colAabbMax[c])) * 0.5f;
    const f3 ext = hi - lo;
    auto q = [](float v, float l, float e) {
        const float t = e > 0.0f ? (v - l) / e : 0.0f;
        return uint32_t(fminf(fmaxf(t * 1024.0f, 0.0f), 1023.0f));
    };
    s.bvhKeyA[k] = expandBits10(q(ctr.x, lo.x, ext.x)) | (expandBits10(q(ctr.y, lo.y, ext.y)) << 1) |
                   (expandBits10(q(ctr.z, lo.z, ext.z)) << 2);
}

// Common-prefix length of sorted codes i and j, the index breaking ties (Karras 2012, section 4).
__device__ __forceinline__ int prefixDelta(const uint32_t *k, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __clz(uint32_t(i) ^ uint32_t(j));
    return __clz(a ^ b);
}

// Internal node i covers a range of sorted leaves found by its prefix; its split is where the
// prefix grows.  Internal nodes are 0 .. n-2, leaf i is node n-1+i.
__global__ void k_bvhBuild(Scene s)
{
    const int n = int(s.colQueryCount);
    const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n - 1) return;
    const uint32_t *k = s.bvhKeyA;
    const int d = (prefixDelta(k, n, i, i + 1) - prefixDelta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = prefixDelta(k, n, i, i - d);
    int lmax = 2;
    while (prefixDelta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (prefixDelta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = prefixDelta(k, n, i, j);
    int sp = 0;
    for (int div = 2;; div *= 2) {
        const int t = (l + div - 1) / div;
        if (prefixDelta(k, n, i, i + (sp + t) * d) > dnode) sp += t;
        if (t <= 1) break;
    }
    const int gamma = i + sp * d + (d < 0 ? d : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const uint32_t left = lo == gamma ? uint32_t(n - 1 + gamma) : uint32_t(gamma);
    const uint32_t right = hi == gamma + 1 ? uint32_t(n - 1 + gamma + 1) : uint32_t(gamma + 1);
    s.bvhChildren[i] = make_uint2(left, right);
    s.bvhParent[left] = uint32_t(i);
    s.bvhParent[right] = uint32_t(i);
}

// Leaf boxes, then up the tree: the second child to reach a parent writes the parent's box.
__global__ void k_bvhRefit(Scene s)
{
    const uint32_t n = s.colQueryCount;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = s.colQueryOrder[s.bvhValA[i]];
    uint32_t node = n - 1 + i;
    s.bvhMin[node] = s.colAabbMin[c];
    s.bvhMax[node] = s.colAabbMax[c];
    while (node != 0u) {
        const uint32_t p = s.bvhParent[node];
        __threadfence();
        if (atomicAdd(&s.bvhVisits[p], 1u) == 0u) return; // the sibling finishes this parent
        __threadfence();
        const uint2 ch = s.bvhChildren[p];
        const float4 a0 = __ldcg(&s.bvhMin[ch.x]), a1 = __ldcg(&s.bvhMax[ch.x]);
        const float4 b0 = __ldcg(&s.bvhMin[ch.y]), b1 = __ldcg(&s.bvhMax[ch.y]);
        s.bvhMin[p] = mk4(min3(xyz(a0), xyz(b0)), 0.f);
        s.bvhMax[p] = mk4(max3(xyz(a1), xyz(b1)), 0.f);
        float4 *w = s.bvhWide + size_t(p) * 4u; // the walk's record: child boxes and indices
        w[0] = mk4(xyz(a0), __uint_as_float(ch.x));
        w[1] = mk4(xyz(a1), 0.f);
        w[2] = mk4(xyz(b0), __uint_as_float(ch.y));
        w[3] = mk4(xyz(b1), 0.f);
        node = p;
    }
}

// physics_rigid_count_pairs / emit_pairs.cs.hlsl: moving collider k of the query order walks
// the tree; a moving partner counts once (higher collider index), a static one always.  The count
// pass also stages the first kPairStage canonical pairs of its walk (rrStage, kPairStage per
// moving collider), so the emit pass copies them to their scanned offsets and walks again only
// for a collider with more partners: one walk per collider, the same pairs in the same order.
constexpr uint32_t kPairStage = 64u;

template <class F>
__device__ __forceinline__ void walkPairs(const Scene &s, uint32_t cA, F &&emit)
{
    const cn_collider_broadphase a = s.colBp[cA];
    const f3 qmin = xyz(s.colAabbMin[cA]), qmax = xyz(s.colAabbMax[cA]);
    // a full stack skips the subtree, as the reference's 128-entry traversal stack does
    bvhQuery<kBvhStack>(s, qmin, qmax, [&](uint32_t leaf) -> bool {
        const uint32_t cB = s.colQueryOrder[s.bvhValA[leaf]];
        if (cB == cA) return true;
        const cn_collider_broadphase b = s.colBp[cB];
        if (b.owner_body == a.owner_body) return true;
        const bool bMoving = s.bodyType[b.owner_body] != CN_BODY_STATIC;
        if (bMoving && cB < cA) return true;
        if (!broadPhaseCollide(a, b)) return true;
        // CanonicalizeRigidPair (physics_rigid_types.hlsli:282-305): lower shape type first
        return emit(a.shape_type > b.shape_type ? make_uint2(cB, cA) : make_uint2(cA, cB));
    });
}

__global__ void k_rigidPairsCount(Scene s)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= s.activeMovingCount) return;
    uint32_t count = 0;
    uint2 *stage = s.rrStage + size_t(k) * kPairStage;
    if (s.colQueryCount >= 2u)
        walkPairs(s, s.colQueryOrder[k], [&](uint2 pr) -> bool {
            if (count < kPairStage) stage[count] = pr;
            ++count;
            return true;
        });
    s.rrCount[k] = count;
}

__global__ void k_rigidPairsEmit(Scene s, const uint32_t *total)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        s.meta_->requiredRigidRigidPairs = *total;
        s.meta_->rigidRigidPairCount = min(*total, s.rrCapacity);
        s.meta_->rigidContactSlots = kRigidPairContacts * min(*total, s.rrCapacity);
    }
    if (k >= s.activeMovingCount) return;
    const uint32_t count = s.rrCount[k];
    uint32_t write = s.rrOffset[k];
    if (count <= kPairStage) {
        const uint2 *stage = s.rrStage + size_t(k) * kPairStage;
        for (uint32_t j = 0; j < count && write < s.rrCapacity; ++j) s.rrPairs[write++] = stage[j];
        return;
    }
    walkPairs(s, s.colQueryOrder[k], [&](uint2 pr) -> bool {
        if (write >= s.rrCapacity) return false;
        s.rrPairs[write++] = pr;
        return true;
    });
}

// ------------------------------------------------------------------------------ narrow phase
// physics_rigid_contact_primitives.hlsli
__device__ __forceinline__ float penetrationFromPoints(f3 a, f3 b, f3 n) { return mx(0.0f, -dot(b - a, n)); }

__device__ bool sphereSphere(f3 cA, float rA, f3 cB, float rB, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0.f, 0.f, 0.f};
    pen = 0.0f;
    const f3 d = cB - cA;
    const float d2 = dot(d, d);
    const float r = rA + rB;
    if (d2 > r * r) return false;
    const float dist = sqrtf(mx(d2, 0.0f));
    n = dist > kEps ? d / dist : f3{0.f, 1.f, 0.f};
    pA = cA + n * rA;
    pB = cB - n * rB;
    pen = penetrationFromPoints(pA, pB, n);
    return pen > 0.0f;
}

__device__ bool sphereBox(f3 sc, float sr, f3 bc, float4 bq, f3 h, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0.f, 0.f, 0.f};
    pen = 0.0f;
    const f3 ls = qInvRotate(bq, sc - bc);
    const f3 cl = clamp3(ls, -h, h);
    const bool inside = ls.x >= -h.x && ls.y >= -h.y && ls.z >= -h.z && ls.x <= h.x && ls.y <= h.y && ls.z <= h.z;
    if (!inside) {
        const f3 bp = bc + qRotate(bq, cl);
        const f3 d = bp - sc;
        const float d2 = dot(d, d);
        if (d2 > sr * sr) return false;
        const float dist = sqrtf(mx(d2, 0.0f));
        n = dist > kEps ? d / dist : f3{0.f, 1.f, 0.f};
        pA = sc + n * sr;
        pB = bp;
        pen = penetrationFromPoints(pA, pB, n);
        return pen > 0.0f;
    }
    const f3 lfn = closestFaceNormalLocal(ls, h);
    const f3 fnw = qRotate(bq, lfn);
    const float depth = mn(h.x - fabsf(ls.x), mn(h.y - fabsf(ls.y), h.z - fabsf(ls.z)));
    n = -fnw;
    pB = bc + qRotate(bq, ls + lfn * depth);
    pA = sc + n * sr;
    pen = depth + sr;
    return pen > 0.0f;
}

__device__ bool sphereCapsule(f3 sc, float sr, f3 a, f3 b, float cr, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    const f3 seg = b - a;
    const float l2 = dot(seg, seg);
    float t = 0.0f;
    if (l2 > kEps) t = saturate(dot(sc - a, seg) / l2);
    return sphereSphere(sc, sr, a + seg * t, cr, n, pA, pB, pen);
}

__device__ __forceinline__ float boxProjectionRadius(f3 axis, const f3 *ax, f3 h)
{
    return h.x * fabsf(dot(axis, ax[0])) + h.y * fabsf(dot(axis, ax[1])) + h.z * fabsf(dot(axis, ax[2]));
}

__device__ __forceinline__ float comp(f3 v, uint32_t i) { return i == 0u ? v.x : (i == 1u ? v.y : v.z); }

// TestObbAxis: false on a separating axis; the smallest overlap wins (rsqrt as 1 / sqrt)
__device__ bool testObbAxis(f3 axis, f3 cd, const f3 *axA, f3 hA, const f3 *axB, f3 hB, uint32_t type, uint32_t ia,
                            uint32_t ib, float &minPen, f3 &best, uint32_t &bType, uint32_t &bA, uint32_t &bB)
{
    const float l2 = dot(axis, axis);
    if (l2 <= kEps) return true;
    const f3 n = axis * (1.0f / sqrtf(l2));
    const float dist = fabsf(dot(cd, n));
    const float overlap = boxProjectionRadius(n, axA, hA) + boxProjectionRadius(n, axB, hB) - dist;
    if (overlap < 0.0f) return false;
    if (overlap < minPen) {
        minPen = overlap;
        best = dot(cd, n) >= 0.0f ? n : -n;
        bType = type;
        bA = ia;
        bB = ib;
    }
    return true;
}

__device__ void boxSupportEdge(uint32_t axis, f3 c, const f3 *ax, f3 h, f3 dir, f3 &e0, f3 &e1)
{
    const uint32_t oa = (axis + 1u) % 3u, ob = (axis + 2u) % 3u;
    const float sa = dot(ax[oa], dir) >= 0.0f ? 1.0f : -1.0f;
    const float sb = dot(ax[ob], dir) >= 0.0f ? 1.0f : -1.0f;
    const f3 ec = c + ax[oa] * (comp(h, oa) * sa) + ax[ob] * (comp(h, ob) * sb);
    const f3 eh = ax[axis] * comp(h, axis);
    e0 = ec - eh;
    e1 = ec + eh;
}

__device__ void closestSegmentSegment(f3 a0, f3 a1, f3 b0, f3 b1, f3 &oa, f3 &ob)
{
    oa = a0;
    ob = b0;
    const f3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float sv = 0.0f, t = 0.0f;
    if (a <= kEps && e <= kEps) return;
    if (a <= kEps) {
        t = saturate(f / e);
    } else {
        const float c = dot(d1, r);
        if (e <= kEps) {
            sv = saturate(-c / a);
        } else {
            const float b = dot(d1, d2);
            const float den = a * e - b * b;
            if (den != 0.0f) sv = saturate((b * f - c * e) / den);
            const float tn = b * sv + f;
            if (tn < 0.0f) {
                t = 0.0f;
                sv = saturate(-c / a);
            } else if (tn > e) {
                t = 1.0f;
                sv = saturate((b - c) / a);
            } else {
                t = tn / e;
            }
        }
    }
    oa = a0 + d1 * sv;
    ob = b0 + d2 * t;
}

__device__ bool boxBox(f3 cA, float4 qA, f3 hA, f3 cB, float4 qB, f3 hB, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0.f, 0.f, 0.f};
    pen = 0.0f;
    const f3 axA[3] = {qRotate(qA, f3{1.f, 0.f, 0.f}), qRotate(qA, f3{0.f, 1.f, 0.f}), qRotate(qA, f3{0.f, 0.f, 1.f})};
    const f3 axB[3] = {qRotate(qB, f3{1.f, 0.f, 0.f}), qRotate(qB, f3{0.f, 1.f, 0.f}), qRotate(qB, f3{0.f, 0.f, 1.f})};
    const f3 cd = cB - cA;
    float minPen = 3.402823466e+38f;
    f3 best{0.f, 1.f, 0.f};
    uint32_t bType = 0u, bA = 0u, bB = 0u;
    for (uint32_t i = 0; i < 3u; ++i)
        if (!testObbAxis(axA[i], cd, axA, hA, axB, hB, 0u, i, 0u, minPen, best, bType, bA, bB)) return false;
    for (uint32_t i = 0; i < 3u; ++i)
        if (!testObbAxis(axB[i], cd, axA, hA, axB, hB, 1u, i, 0u, minPen, best, bType, bA, bB)) return false;
    for (uint32_t a = 0; a < 3u; ++a)
        for (uint32_t b = 0; b < 3u; ++b)
            if (!testObbAxis(cross(axA[a], axB[b]), cd, axA, hA, axB, hB, 2u, a, b, minPen, best, bType, bA, bB))
                return false;
    n = best;
    if (bType == 2u) {
        f3 ea0, ea1, eb0, eb1;
        boxSupportEdge(bA, cA, axA, hA, n, ea0, ea1);
        boxSupportEdge(bB, cB, axB, hB, -n, eb0, eb1);
        closestSegmentSegment(ea0, ea1, eb0, eb1, pA, pB);
    } else if (bType == 1u) {
        pB = boxSupportPoint(cB, qB, hB, -n);
        pA = closestPointOnBox(pB, cA, qA, hA);
    } else {
        pA = boxSupportPoint(cA, qA, hA, n);
        pB = closestPointOnBox(pA, cB, qB, hB);
    }
    pen = minPen;
    return pen > 0.0f;
}

__device__ bool segmentHitsAabbLocal(f3 a, f3 b, f3 h, f3 &hit)
{
    hit = a;
    float tMin = 0.0f, tMax = 1.0f;
    const f3 d = b - a;
    for (uint32_t ax = 0; ax < 3u; ++ax) {
        const float o = comp(a, ax), dl = comp(d, ax), lo = -comp(h, ax), hi = comp(h, ax);
        if (fabsf(dl) <= kEps) {
            if (o < lo || o > hi) {
                hit = a;
                return false;
            }
            continue;
        }
        const float inv = 1.0f / dl;
        float t0 = (lo - o) * inv, t1 = (hi - o) * inv;
        if (t0 > t1) {
            const float tmp = t0;
            t0 = t1;
            t1 = tmp;
        }
        tMin = mx(tMin, t0);
        tMax = mn(tMax, t1);
        if (tMin > tMax) {
            hit = a;
            return false;
        }
    }
    hit = a + d * tMin;
    return true;
}

__device__ __forceinline__ void segmentBoxCandidate(float t, f3 la, f3 lb, f3 h, float &bestD2, f3 &bestSeg, f3 &bestBox)
{
    if (t < 0.0f || t > 1.0f) return;
    const f3 sp = lerp3(la, lb, t);
    const f3 bp = clamp3(sp, -h, h);
    const float d2 = dot(sp - bp, sp - bp);
    if (d2 < bestD2) {
        bestD2 = d2;
        bestSeg = sp;
        bestBox = bp;
    }
}

__device__ void closestSegmentBox(f3 sa, f3 sb, f3 bc, float4 bq, f3 h, f3 &outSeg, f3 &outBox, bool &intersects)
{
    outSeg = sa;
    outBox = closestPointOnBox(sa, bc, bq, h);
    const f3 la = qInvRotate(bq, sa - bc), lb = qInvRotate(bq, sb - bc);
    f3 hitP;
    intersects = segmentHitsAabbLocal(la, lb, h, hitP);
    if (intersects) {
        outSeg = bc + qRotate(bq, hitP);
        outBox = outSeg;
        return;
    }
    float bestD2 = 3.402823466e+38f;
    f3 bestSeg = la, bestBox = clamp3(la, -h, h);
    const f3 d = lb - la;
    segmentBoxCandidate(0.0f, la, lb, h, bestD2, bestSeg, bestBox);
    segmentBoxCandidate(1.0f, la, lb, h, bestD2, bestSeg, bestBox);
    for (uint32_t ax = 0; ax < 3u; ++ax) {
        const float dl = comp(d, ax);
        if (fabsf(dl) > kEps) {
            segmentBoxCandidate((-comp(h, ax) - comp(la, ax)) / dl, la, lb, h, bestD2, bestSeg, bestBox);
            segmentBoxCandidate((comp(h, ax) - comp(la, ax)) / dl, la, lb, h, bestD2, bestSeg, bestBox);
        }
    }
    outSeg = bc + qRotate(bq, bestSeg);
    outBox = bc + qRotate(bq, bestBox);
}

__device__ bool boxCapsule(f3 bc, float4 bq, f3 h, f3 ca, f3 cb, float cr, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0.f, 0.f, 0.f};
    pen = 0.0f;
    f3 segP, boxP;
    bool inter = false;
    closestSegmentBox(ca, cb, bc, bq, h, segP, boxP, inter);
    if (!inter) {
        const f3 d = segP - boxP;
        const float d2 = dot(d, d);
        if (d2 > cr * cr) return false;
        const float dist = sqrtf(mx(d2, 0.0f));
        n = dist > kEps ? d / dist : f3{0.f, 1.f, 0.f};
        pA = boxP;
        pB = segP - n * cr;
        pen = penetrationFromPoints(pA, pB, n);
        return pen > 0.0f;
    }
    const f3 ls = qInvRotate(bq, segP - bc);
    const f3 lfn = closestFaceNormalLocal(ls, h);
    n = qRotate(bq, lfn);
    const float depth = mn(h.x - fabsf(ls.x), mn(h.y - fabsf(ls.y), h.z - fabsf(ls.z)));
    pA = bc + qRotate(bq, ls + lfn * depth);
    pB = segP - n * cr;
    pen = penetrationFromPoints(pA, pB, n);
    return pen > 0.0f;
}

// ------------------------------------------------------------ box-box manifold
// physics_rigid_box_box_manifold.hlsli: separating axis with a preference for face axes, then
// the incident face clipped against the reference face (or the edge pair, or corner recovery),
// reduced to at most kRigidPairContacts points (deepest first, then the farthest apart).
constexpr uint32_t kBoxCandidates = 16u;

__device__ bool boxBoxSat(f3 cA, const f3 *axA, f3 hA, f3 cB, const f3 *axB, f3 hB, f3 &nOut, float &penOut,
                          uint32_t &typeOut, uint32_t &aOut, uint32_t &bOut)
{
    nOut = f3{0.f, 0.f, 0.f};
    penOut = 0.0f;
    typeOut = 0u;
    aOut = bOut = 0u;
    const f3 cd = cB - cA;
    float bestFace = 3.402823466e+38f, bestEdge = 3.402823466e+38f;
    f3 faceAxis{0.f, 1.f, 0.f}, edgeAxis{0.f, 1.f, 0.f};
    uint32_t faceType = 0u, faceA = 0u, edgeA = 0u, edgeB = 0u;
    bool hasEdge = false;
    for (uint32_t side = 0; side < 2u; ++side)
        for (uint32_t i = 0; i < 3u; ++i) {
            f3 n = side == 0u ? axA[i] : axB[i];
            const float overlap = boxProjectionRadius(n, axA, hA) + boxProjectionRadius(n, axB, hB) - fabsf(dot(cd, n));
            if (overlap < 0.0f) return false;
            if (dot(cd, n) < 0.0f) n = -n;
            if (overlap < bestFace - 5.0e-4f) {
                bestFace = overlap;
                faceAxis = n;
                faceType = side;
                faceA = i;
            }
        }
    for (uint32_t a = 0; a < 3u; ++a)
        for (uint32_t b = 0; b < 3u; ++b) {
            const f3 axis = cross(axA[a], axB[b]);
            const float l2 = dot(axis, axis);
            if (l2 <= kEps) continue;
            hasEdge = true;
            f3 n = axis * (1.0f / sqrtf(l2));
            const float overlap = boxProjectionRadius(n, axA, hA) + boxProjectionRadius(n, axB, hB) - fabsf(dot(cd, n));
            if (overlap < 0.0f) return false;
            if (dot(cd, n) < 0.0f) n = -n;
            if (overlap < bestEdge) {
                bestEdge = overlap;
                edgeAxis = n;
                edgeA = a;
                edgeB = b;
            }
        }
    if (hasEdge && bestEdge < bestFace * 0.95f - 1.0e-3f) {
        nOut = edgeAxis;
        penOut = bestEdge;
        typeOut = 2u;
        aOut = edgeA;
        bOut = edgeB;
    } else {
        nOut = faceAxis;
        penOut = bestFace;
        typeOut = faceType;
        aOut = faceA;
        bOut = 0u;
    }
    return penOut > 0.0f;
}

struct BoxCandidate {
    f3 a, b;
    float pen;
};

__device__ void insertCandidate(f3 pa, f3 pb, float pen, float merge2, uint32_t &count, BoxCandidate *cand)
{
    if (pen <= kEps) return;
    const f3 mid = (pa + pb) * 0.5f;
    for (uint32_t i = 0; i < count; ++i) {
        const f3 d = (cand[i].a + cand[i].b) * 0.5f - mid;
        if (dot(d, d) <= merge2) {
            if (pen > cand[i].pen) cand[i] = BoxCandidate{pa, pb, pen};
            return;
        }
    }
    if (count < kBoxCandidates) {
        cand[count++] = BoxCandidate{pa, pb, pen};
        return;
    }
    uint32_t r = 0;
    float minPen = cand[0].pen;
    for (uint32_t i = 1; i < kBoxCandidates; ++i)
        if (cand[i].pen < minPen) {
            minPen = cand[i].pen;
            r = i;
        }
    if (pen > minPen) cand[r] = BoxCandidate{pa, pb, pen};
}

__device__ uint32_t clipAgainstPlane(const f3 *in, uint32_t inCount, f3 origin, f3 normal, float offset, bool keepLess,
                                     f3 *out)
{
    if (inCount == 0u) return 0u;
    uint32_t oc = 0;
    f3 prev = in[inCount - 1u];
    float prevC = dot(prev - origin, normal);
    bool prevIn = keepLess ? prevC <= offset : prevC >= offset;
    for (uint32_t i = 0; i < inCount && i < 8u; ++i) {
        const f3 cur = in[i];
        const float curC = dot(cur - origin, normal);
        const bool curIn = keepLess ? curC <= offset : curC >= offset;
        if (curIn != prevIn) {
            const float den = curC - prevC;
            const float t = fabsf(den) > kEps ? (offset - prevC) / den : 0.0f;
            if (oc < 8u) out[oc++] = lerp3(prev, cur, saturate(t));
        }
        if (curIn && oc < 8u) out[oc++] = cur;
        prev = cur;
        prevC = curC;
        prevIn = curIn;
    }
    return oc;
}

__device__ __forceinline__ f3 boxCorner(f3 c, float4 q, f3 h, uint32_t k)
{
    return c + qRotate(q, f3{(k & 1u) ? h.x : -h.x, (k & 2u) ? h.y : -h.y, (k & 4u) ? h.z : -h.z});
}

__device__ __forceinline__ bool insideBox(f3 p, f3 c, float4 q, f3 h)
{
    const f3 l = qInvRotate(q, p - c);
    return l.x >= -h.x && l.y >= -h.y && l.z >= -h.z && l.x <= h.x && l.y <= h.y && l.z <= h.z;
}

__device__ f3 projectInsideAlong(f3 p, f3 c, float4 q, f3 h, f3 dir)
{
    const f3 lp = qInvRotate(q, p - c);
    const f3 ld = qInvRotate(q, safeNormalize(dir, f3{0.f, 1.f, 0.f}));
    if (!(lp.x >= -h.x && lp.y >= -h.y && lp.z >= -h.z && lp.x <= h.x && lp.y <= h.y && lp.z <= h.z))
        return closestPointOnBox(p, c, q, h);
    float bestT = 3.402823466e+38f;
    for (uint32_t ax = 0; ax < 3u; ++ax) {
        const float d = comp(ld, ax);
        if (fabsf(d) <= kEps) continue;
        const float face = d > 0.0f ? comp(h, ax) : -comp(h, ax);
        const float t = (face - comp(lp, ax)) / d;
        if (t >= 0.0f && t < bestT) bestT = t;
    }
    f3 ls = lp;
    if (bestT < 3.402823466e+37f) {
        ls = lp + ld * bestT;
    } else {
        const f3 lfn = closestFaceNormalLocal(lp, h);
        ls = lp + lfn * mn(h.x - fabsf(lp.x), mn(h.y - fabsf(lp.y), h.z - fabsf(lp.z)));
    }
    return c + qRotate(q, ls);
}

// Returns the number of manifold points written to pts / pens (<= kRigidPairContacts), with
// the manifold normal in n.  0: the caller falls back to the single-point contact.
__device__ uint32_t boxBoxManifold(f3 cA, float4 qA, f3 hA, f3 cB, float4 qB, f3 hB, f3 nIn, float merge2, float slop,
                                   f3 &n, f3 *ptsA, f3 *ptsB, float *pens)
{
    BoxCandidate cand[kBoxCandidates];
    uint32_t count = 0;
    const f3 axA[3] = {qRotate(qA, f3{1.f, 0.f, 0.f}), qRotate(qA, f3{0.f, 1.f, 0.f}), qRotate(qA, f3{0.f, 0.f, 1.f})};
    const f3 axB[3] = {qRotate(qB, f3{1.f, 0.f, 0.f}), qRotate(qB, f3{0.f, 1.f, 0.f}), qRotate(qB, f3{0.f, 0.f, 1.f})};
    n = safeNormalize(nIn, f3{0.f, 1.f, 0.f});
    f3 satN;
    float satPen = 0.0f;
    uint32_t satType = 0u, satA = 0u, satB = 0u;
    const bool sat = boxBoxSat(cA, axA, hA, cB, axB, hB, satN, satPen, satType, satA, satB);
    if (sat) n = safeNormalize(satN, n);
    if (sat && satType == 2u) {
        f3 ea0, ea1, eb0, eb1, pa, pb;
        boxSupportEdge(satA, cA, axA, hA, n, ea0, ea1);
        boxSupportEdge(satB, cB, axB, hB, -n, eb0, eb1);
        closestSegmentSegment(ea0, ea1, eb0, eb1, pa, pb);
        insertCandidate(pa, pb, mx(satPen, penetrationFromPoints(pa, pb, n)), merge2, count, cand);
    }
    if (sat && satType < 2u) {
        const bool refA = satType == 0u;
        const f3 *rax = refA ? axA : axB;
        const f3 rc = refA ? cA : cB, rh = refA ? hA : hB;
        const float sign = dot(rax[satA], refA ? n : -n) >= 0.0f ? 1.0f : -1.0f;
        const uint32_t tu = (satA + 1u) % 3u, tv = (satA + 2u) % 3u;
        const f3 refN = rax[satA] * sign;
        const f3 refC = rc + refN * comp(rh, satA);
        const f3 refU = rax[tu], refV = rax[tv];
        const float halfU = comp(rh, tu), halfV = comp(rh, tv);
        // incident face: the other box's face most opposed to the reference normal
        const f3 *iax = refA ? axB : axA;
        const f3 ic = refA ? cB : cA, ih = refA ? hB : hA;
        uint32_t ia = 0u;
        float best = fabsf(dot(iax[0], refN));
        for (uint32_t i = 1; i < 3u; ++i) {
            const float al = fabsf(dot(iax[i], refN));
            if (al > best) {
                best = al;
                ia = i;
            }
        }
        const float isign = dot(iax[ia], refN) >= 0.0f ? -1.0f : 1.0f;
        const uint32_t iu = (ia + 1u) % 3u, iv = (ia + 2u) % 3u;
        const f3 iN = iax[ia] * isign;
        const f3 iC = ic + iN * comp(ih, ia);
        const f3 du = iax[iu] * comp(ih, iu), dv = iax[iv] * comp(ih, iv);
        f3 polyA[8], polyB[8];
        polyA[0] = iC + du + dv;
        polyA[1] = iC - du + dv;
        polyA[2] = iC - du - dv;
        polyA[3] = iC + du - dv;
        uint32_t pc = 4u;
        pc = clipAgainstPlane(polyA, pc, refC, refU, halfU, true, polyB);
        pc = clipAgainstPlane(polyB, pc, refC, refU, -halfU, false, polyA);
        pc = clipAgainstPlane(polyA, pc, refC, refV, halfV, true, polyB);
        pc = clipAgainstPlane(polyB, pc, refC, refV, -halfV, false, polyA);
        for (uint32_t i = 0; i < pc && i < 8u; ++i) {
            const f3 ip = polyA[i];
            const float sep = dot(ip - refC, refN);
            if (sep > slop) continue;
            const f3 rp = ip - refN * sep;
            const float pen = mx(0.0f, -sep);
            if (refA) insertCandidate(rp, ip, pen, merge2, count, cand);
            else insertCandidate(ip, rp, pen, merge2, count, cand);
        }
    }
    if (count == 0u) {
        for (uint32_t k = 0; k < 8u; ++k) {
            const f3 ca = boxCorner(cA, qA, hA, k);
            f3 pbA = closestPointOnBox(ca, cB, qB, hB);
            if (insideBox(ca, cB, qB, hB)) pbA = projectInsideAlong(ca, cB, qB, hB, -n);
            insertCandidate(ca, pbA, penetrationFromPoints(ca, pbA, n), merge2, count, cand);
            const f3 cb = boxCorner(cB, qB, hB, k);
            f3 paB = closestPointOnBox(cb, cA, qA, hA);
            if (insideBox(cb, cA, qA, hA)) paB = projectInsideAlong(cb, cA, qA, hA, n);
            insertCandidate(paB, cb, penetrationFromPoints(paB, cb, n), merge2, count, cand);
        }
    }
    if (count == 0u) return 0u;
    // reduce: deepest, then greedily the candidate farthest (in the contact plane) from those kept
    const f3 tx = safeNormalize(cross(fabsf(n.y) < 0.9f ? f3{0.f, 1.f, 0.f} : f3{1.f, 0.f, 0.f}, n), f3{1.f, 0.f, 0.f});
    const f3 ty = cross(n, tx);
    float mu[kBoxCandidates], mv[kBoxCandidates];
    bool sel[kBoxCandidates];
    for (uint32_t i = 0; i < count; ++i) {
        const f3 mid = (cand[i].a + cand[i].b) * 0.5f;
        mu[i] = dot(mid, tx);
        mv[i] = dot(mid, ty);
        sel[i] = false;
    }
    const uint32_t target = count < kRigidPairContacts ? count : kRigidPairContacts;
    uint32_t deepest = 0;
    for (uint32_t i = 1; i < count; ++i)
        if (cand[i].pen > cand[deepest].pen) deepest = i;
    sel[deepest] = true;
    uint32_t out = 0;
    ptsA[out] = cand[deepest].a;
    ptsB[out] = cand[deepest].b;
    pens[out++] = cand[deepest].pen;
    while (out < target) {
        uint32_t bi = 0;
        float bs = -1.0f;
        bool found = false;
        for (uint32_t i = 0; i < count; ++i) {
            if (sel[i]) continue;
            float md = 3.402823466e+38f;
            for (uint32_t j = 0; j < count; ++j) {
                if (!sel[j]) continue;
                const float du2 = mu[i] - mu[j], dv2 = mv[i] - mv[j];
                md = mn(md, du2 * du2 + dv2 * dv2);
            }
            const float score = md + cand[i].pen * 1.0e-4f;
            if (score > bs) {
                bs = score;
                bi = i;
                found = true;
            }
        }
        if (!found) break;
        sel[bi] = true;
        ptsA[out] = cand[bi].a;
        ptsB[out] = cand[bi].b;
        pens[out++] = cand[bi].pen;
    }
    return out;
}

// GenerateRigidContact (physics_rigid_contact_primitives.hlsli:520-641)
__device__ bool rigidContactPoints(uint32_t tA, f3 pA_, float4 qA, float4 prA, float4 sA, uint32_t tB, f3 pB_, float4 qB,
                                   float4 prB, float4 sB, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0.f, 0.f, 0.f};
    pen = 0.0f;
    const uint32_t S = CN_COLLIDER_SPHERE, X = CN_COLLIDER_BOX, K = CN_COLLIDER_CAPSULE;
    if (tA == S && tB == S) return sphereSphere(pA_, sphereRadius(prA, sA), pB_, sphereRadius(prB, sB), n, pA, pB, pen);
    if (tA == S && tB == X)
        return sphereBox(pA_, sphereRadius(prA, sA), pB_, qB, boxHalfExtents(prB, sB), n, pA, pB, pen);
    if (tA == X && tB == S) {
        f3 ns, ps, pb;
        const bool hit = sphereBox(pB_, sphereRadius(prB, sB), pA_, qA, boxHalfExtents(prA, sA), ns, ps, pb, pen);
        n = -ns;
        pA = pb;
        pB = ps;
        pen = penetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    if (tA == S && tB == K) {
        f3 b0, b1;
        float rB = 0.0f;
        capsuleSegment(pB_, qB, prB, sB, b0, b1, rB);
        return sphereCapsule(pA_, sphereRadius(prA, sA), b0, b1, rB, n, pA, pB, pen);
    }
    if (tA == K && tB == S) {
        f3 a0, a1;
        float rA = 0.0f;
        capsuleSegment(pA_, qA, prA, sA, a0, a1, rA);
        f3 ns, ps, pc;
        const bool hit = sphereCapsule(pB_, sphereRadius(prB, sB), a0, a1, rA, ns, ps, pc, pen);
        n = -ns;
        pA = pc;
        pB = ps;
        pen = penetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    if (tA == X && tB == X)
        return boxBox(pA_, qA, boxHalfExtents(prA, sA), pB_, qB, boxHalfExtents(prB, sB), n, pA, pB, pen);
    if (tA == K && tB == K) {
        f3 a0, a1, b0, b1, ca, cb;
        float rA = 0.0f, rB = 0.0f;
        capsuleSegment(pA_, qA, prA, sA, a0, a1, rA);
        capsuleSegment(pB_, qB, prB, sB, b0, b1, rB);
        closestSegmentSegment(a0, a1, b0, b1, ca, cb);
        return sphereSphere(ca, rA, cb, rB, n, pA, pB, pen);
    }
    if (tA == X && tB == K) {
        f3 b0, b1;
        float rB = 0.0f;
        capsuleSegment(pB_, qB, prB, sB, b0, b1, rB);
        return boxCapsule(pA_, qA, boxHalfExtents(prA, sA), b0, b1, rB, n, pA, pB, pen);
    }
    if (tA == K && tB == X) {
        f3 a0, a1;
        float rA = 0.0f;
        capsuleSegment(pA_, qA, prA, sA, a0, a1, rA);
        f3 nb, pbx, pcap;
        const bool hit = boxCapsule(pB_, qB, boxHalfExtents(prB, sB), a0, a1, rA, nb, pbx, pcap, pen);
        n = -nb;
        pA = pcap;
        pB = pbx;
        pen = penetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    return false;
}

__device__ __forceinline__ float4 colliderParams(const cn_collider_geometry &g)
{
    return make_float4(g.shape_params[0], g.shape_params[1], g.shape_params[2], g.shape_params[3]);
}

// physics_rigid_generate_contacts.cs.hlsl:37-190 (ProcessPair): the pair's kRigidPairContacts
// slots are cleared, then filled by the box-box manifold or by the single-point contact.
__global__ void k_rigidNarrowPhase(Scene s, Config cfg)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.meta_->rigidRigidPairCount) return;
    RigidPairContact *slot = s.rrContacts + size_t(p) * kRigidPairContacts;
    for (uint32_t k = 0; k < kRigidPairContacts; ++k) slot[k] = RigidPairContact{};
    const uint2 pr = s.rrPairs[p];
    const cn_collider_broadphase bpA = s.colBp[pr.x], bpB = s.colBp[pr.y];
    const uint32_t bA = bpA.owner_body, bB = bpB.owner_body;
    if (bA >= s.B || bB >= s.B || bA == bB) return;
    const uint32_t tyA = s.bodyType[bA], tyB = s.bodyType[bB];
    if (tyA != CN_BODY_DYNAMIC && tyB != CN_BODY_DYNAMIC) return;
    const float4 posA = s.predBodyPos[bA], posB = s.predBodyPos[bB];
    const float4 qA = qNormalize(s.predBodyRot[bA]), qB = qNormalize(s.predBodyRot[bB]);
    const cn_collider_geometry gA = s.colGeo[pr.x], gB = s.colGeo[pr.y];
    const float4 prmA = colliderParams(gA), prmB = colliderParams(gB);
    const float4 scA = s.bodyScale[bA], scB = s.bodyScale[bB];
    const f3 mat = combineContactMaterial(s.colMat[pr.x], s.colMat[pr.y]);
    const f3 cpA = xyz(posA) + qRotate(qA, f3{gA.local_position[0], gA.local_position[1], gA.local_position[2]} * xyz(scA));
    const f3 cpB = xyz(posB) + qRotate(qB, f3{gB.local_position[0], gB.local_position[1], gB.local_position[2]} * xyz(scB));
    const float4 cqA = qNormalize(qMul(qA, qNormalize(make_float4(gA.local_orientation[0], gA.local_orientation[1],
                                                                 gA.local_orientation[2], gA.local_orientation[3]))));
    const float4 cqB = qNormalize(qMul(qB, qNormalize(make_float4(gB.local_orientation[0], gB.local_orientation[1],
                                                                 gB.local_orientation[2], gB.local_orientation[3]))));
    f3 a0, a1, b0, b1;
    computeBodyAabb(bpA.shape_type, cpA, cqA, prmA, scA, a0, a1);
    computeBodyAabb(bpB.shape_type, cpB, cqB, prmB, scB, b0, b1);
    if (!aabbOverlaps(a0, a1, b0, b1)) return;
    auto write = [&](uint32_t k, f3 n, float pen, f3 pa, f3 pb) {
        RigidPairContact c{};
        c.bodyA = bA;
        c.bodyB = bB;
        c.active = 1u;
        c.normalPenetration = mk4(n, pen);
        c.material = mk4(mat, 0.0f);
        c.localPointA = mk4(qInvRotate(qA, pa - xyz(posA)), 1.0f);
        c.localPointB = mk4(qInvRotate(qB, pb - xyz(posB)), 1.0f);
        slot[k] = c;
    };
    if (bpA.shape_type == CN_COLLIDER_BOX && bpB.shape_type == CN_COLLIDER_BOX) {
        const f3 hA = boxHalfExtents(prmA, scA), hB = boxHalfExtents(prmB, scB);
        const f3 axA[3] = {qRotate(cqA, f3{1.f, 0.f, 0.f}), qRotate(cqA, f3{0.f, 1.f, 0.f}), qRotate(cqA, f3{0.f, 0.f, 1.f})};
        const f3 axB[3] = {qRotate(cqB, f3{1.f, 0.f, 0.f}), qRotate(cqB, f3{0.f, 1.f, 0.f}), qRotate(cqB, f3{0.f, 0.f, 1.f})};
        f3 satN;
        float satPen = 0.0f;
        uint32_t t0, t1, t2;
        if (!boxBoxSat(cpA, axA, hA, cpB, axB, hB, satN, satPen, t0, t1, t2)) return;
        const f3 cn0 = safeNormalize(satN, f3{0.f, 1.f, 0.f});
        f3 pa[kRigidPairContacts], pb[kRigidPairContacts], n;
        float pens[kRigidPairContacts];
        const float merge = cfg.manifoldMergeDistance;
        const uint32_t m = boxBoxManifold(cpA, cqA, hA, cpB, cqB, hB, cn0, merge * merge, cfg.slop, n, pa, pb, pens);
        if (m > 0u) {
            for (uint32_t k = 0; k < m; ++k) write(k, n, pens[k], pa[k], pb[k]);
            return;
        }
    }
    f3 n, pa, pb;
    float pen = 0.0f;
    if (!rigidContactPoints(bpA.shape_type, cpA, cqA, prmA, scA, bpB.shape_type, cpB, cqB, prmB, scB, n, pa, pb, pen) ||
        pen <= 0.0f)
        return;
    write(0u, safeNormalize(n, f3{0.f, 1.f, 0.f}), pen, pa, pb);
}

// physics_rigid_generate_proxy_contacts.cs.hlsl: proxy candidate k (a proxy particle of body A
// and a candidate body B) fills contact slot pairSlots + k with the deepest contact between the
// proxy sphere and B's enabled colliders (collider frames without the body scale, as
// ComposeColliderWorldPosition), or leaves it inactive.  Proxy particles lead the particle order
// and candidates are emitted particle by particle, so the proxies' candidates open the list; a
// slot per candidate keeps the contact order deterministic (the reference appends hits with an
// atomic counter).
__global__ void k_proxyRigidContacts(Scene s)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t last = s.nProxy - 1u;
    const uint32_t proxyCands = min(s.meta_->rigidPairCount, s.candOffset[last] + s.candCount[last]);
    const uint32_t used = min(proxyCands, s.proxyCapacity);
    const uint32_t base = kRigidPairContacts * s.meta_->rigidRigidPairCount;
    if (k == 0) {
        s.meta_->requiredProxyContacts = proxyCands;
        s.meta_->proxyContactSlots = used;
        s.meta_->rigidContactSlots = base + used;
    }
    if (k >= used) return;
    RigidPairContact out{};
    const uint2 pr = s.rigidPairs[k];
    const uint32_t p = pr.x, bB = pr.y;
    const uint32_t bA = s.ownerIdx[p];
    const float4 posA = s.predBodyPos[bA], posB = s.predBodyPos[bB];
    if (p >= s.nProxy || bA == bB || (posA.w <= kEps && posB.w <= kEps)) {
        s.rrContacts[base + k] = out;
        return;
    }
    const f3 sc = xyz(s.x[p]);
    const float sr = s.radii[p];
    const float4 qA = qNormalize(s.predBodyRot[bA]), qB = qNormalize(s.predBodyRot[bB]);
    const float4 scB = s.bodyScale[bB];
    const float4 proxyMat = s.bodyProxyMat[bA];
    const uint2 cr = s.bodyColRanges[bB];
    float best = 0.0f;
    f3 bestN{0.f, 1.f, 0.f}, bestA{0.f, 0.f, 0.f}, bestB{0.f, 0.f, 0.f}, bestMat{0.f, 0.f, 0.f};
    for (uint32_t i = 0; i < kColliderIterationCap; ++i) {
        if (i >= cr.y) break;
        const uint32_t c = s.bodyColIdx[cr.x + i];
        const cn_collider_broadphase bp = s.colBp[c];
        if (bp.enabled_flag == 0u) continue;
        const cn_collider_geometry g = s.colGeo[c];
        const f3 cwp = xyz(posB) + qRotate(qB, f3{g.local_position[0], g.local_position[1], g.local_position[2]});
        const float4 cwq = qNormalize(qMul(qB, qNormalize(make_float4(g.local_orientation[0], g.local_orientation[1],
                                                                     g.local_orientation[2], g.local_orientation[3]))));
        const float4 prm = colliderParams(g);
        f3 n, pa, pb;
        float pen = 0.0f;
        bool hit;
        if (bp.shape_type == CN_COLLIDER_SPHERE) {
            hit = sphereSphere(sc, sr, cwp, sphereRadius(prm, scB), n, pa, pb, pen);
        } else if (bp.shape_type == CN_COLLIDER_BOX) {
            hit = sphereBox(sc, sr, cwp, cwq, boxHalfExtents(prm, scB), n, pa, pb, pen);
        } else {
            f3 ca, cb;
            float capR = 0.0f;
            capsuleSegment(cwp, cwq, prm, scB, ca, cb, capR);
            hit = sphereCapsule(sc, sr, ca, cb, capR, n, pa, pb, pen);
        }
        if (!hit || pen <= best) continue;
        best = pen;
        bestN = safeNormalize(n, f3{0.f, 1.f, 0.f});
        bestA = pa;
        bestB = pb;
        bestMat = combineContactMaterial(proxyMat, s.colMat[c]);
    }
    if (best > 0.0f) {
        out.bodyA = bA;
        out.bodyB = bB;
        out.active = 1u;
        out.normalPenetration = mk4(bestN, best);
        out.localPointA = mk4(qInvRotate(qA, bestA - xyz(posA)), 0.0f);
        out.localPointB = mk4(qInvRotate(qB, bestB - xyz(posB)), 0.0f);
        out.material = mk4(bestMat, 0.0f);
    }
    s.rrContacts[base + k] = out;
}

// ------------------------------------------------------------------------- velocity groups
// Sort key of a contact: its canonical body pair (inactive contacts last).
__global__ void k_rigidGroupKeys(Scene s)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.meta_->rigidContactSlots) return;
    const RigidPairContact c = s.rrContacts[p];
    const uint32_t lo = min(c.bodyA, c.bodyB), hi = max(c.bodyA, c.bodyB);
    s.rrKeyA[p] = c.active ? lo * s.B + hi : 0xffffffffu;
}

__global__ void k_rigidGroupHeads(Scene s)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.rrSlotCapacity) return;
    const uint32_t n = s.meta_->rigidContactSlots;
    const uint32_t key = j < n ? s.rrKeyA[j] : 0xffffffffu;
    s.rrHead[j] = (j < n && key != 0xffffffffu && (j == 0u || s.rrKeyA[j - 1] != key)) ? 1u : 0u;
}

// CanonicalizeContact + the slot of physics_rigid_init_contact_velocities.cs.hlsl:208-236, for
// the first kRigidGroupContacts contacts of every body pair (the reference drops the rest).
__global__ void k_rigidGroupInit(Scene s, Config cfg, const uint32_t *groups)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) s.meta_->rigidGroupCount = *groups;
    const uint32_t n = s.meta_->rigidContactSlots;
    if (j >= n || s.rrHead[j] == 0u) return;
    const uint32_t key = s.rrKeyA[j];
    uint32_t cnt = 0;
    while (j + cnt < n && s.rrKeyA[j + cnt] == key && cnt < kRigidGroupContacts) {
        RigidPairContact c = s.rrContacts[s.rrValA[j + cnt]];
        if (c.bodyA > c.bodyB) {
            const uint32_t t = c.bodyA;
            c.bodyA = c.bodyB;
            c.bodyB = t;
            c.normalPenetration = mk4(-xyz(c.normalPenetration), c.normalPenetration.w);
            const float4 la = c.localPointA;
            c.localPointA = c.localPointB;
            c.localPointB = la;
        }
        RigidSlot sl;
        const f3 nrm = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
        sl.normal = mk4(nrm, saturate(c.material.x));
        sl.localA = mk4(xyz(c.localPointA), saturate(c.material.z));
        sl.localB = c.localPointB;
        sl.state = make_float4(0.f, 0.f, 0.f, 0.f);
        // ComputeContactNormalVelocity with the predicted velocities of this substep
        const float4 pA = s.predBodyPos[c.bodyA], pB = s.predBodyPos[c.bodyB];
        const float4 oA = qNormalize(s.predBodyRot[c.bodyA]), oB = qNormalize(s.predBodyRot[c.bodyB]);
        const f3 rA = (xyz(pA) + qRotate(oA, xyz(c.localPointA))) - xyz(pA);
        const f3 rB = (xyz(pB) + qRotate(oB, xyz(c.localPointB))) - xyz(pB);
        const f3 vA = xyz(s.predBodyLin[c.bodyA]) + cross(xyz(s.predBodyAng[c.bodyA]), rA);
        const f3 vB = xyz(s.predBodyLin[c.bodyB]) + cross(xyz(s.predBodyAng[c.bodyB]), rB);
        const float nv = dot(vB - vA, nrm);
        if (nv < -cfg.rigidRestitutionThreshold) sl.state.y = -saturate(c.material.y) * nv;
        s.rrSlots[j + cnt] = sl;
        ++cnt;
    }
    s.rrGroups[s.rrGroupOf[j]] = make_uint2(j, cnt);
}

// --------------------------------------------------------------------------- depenetration
// physics_rigid_depenetrate_contacts.cs.hlsl:22-137
__global__ void k_rigidDepenetrate(Scene s, Config cfg)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.meta_->rigidContactSlots) return;
    const RigidPairContact c = s.rrContacts[p];
    if (c.active == 0u) return;
    const uint32_t bA = c.bodyA, bB = c.bodyB;
    const float4 pA0 = s.predBodyPos[bA], pB0 = s.predBodyPos[bB];
    const float4 prA = s.prevBodyPos[bA], prB = s.prevBodyPos[bB];
    const uint32_t tyA = s.bodyType[bA], tyB = s.bodyType[bB];
    const float iA = tyA == CN_BODY_DYNAMIC ? pA0.w : 0.0f;
    const float iB = tyB == CN_BODY_DYNAMIC ? pB0.w : 0.0f;
    if (iA == 0.0f && iB == 0.0f) return;
    const float4 qA = qNormalize(s.predBodyRot[bA]), qB = qNormalize(s.predBodyRot[bB]);
    const float4 pqA = qNormalize(s.prevBodyRot[bA]), pqB = qNormalize(s.prevBodyRot[bB]);
    f3 inA = xyz(s.bodyInvInertia[bA]), inB = xyz(s.bodyInvInertia[bB]);
    if (iA == 0.0f) inA = f3{0.f, 0.f, 0.f};
    if (iB == 0.0f) inB = f3{0.f, 0.f, 0.f};
    const f3 ptA = xyz(pA0) + qRotate(qA, xyz(c.localPointA));
    const f3 ptB = xyz(pB0) + qRotate(qB, xyz(c.localPointB));
    const f3 ppA = xyz(prA) + qRotate(pqA, xyz(c.localPointA));
    const f3 ppB = xyz(prB) + qRotate(pqB, xyz(c.localPointB));
    const f3 n = safeNormalize(xyz(c.normalPenetration), f3{0.f, 1.f, 0.f});
    const float measured = -dot(ptB - ptA, n);
    const float raw = mx(measured - cfg.slop, 0.0f);
    const float pen = mn(raw * cfg.baumgarte, cfg.maxDepenetration);
    if (pen <= 0.0f) return;
    const f3 rA = ptA - xyz(pA0), rB = ptB - xyz(pB0);
    const float den = contactEffectiveMass(iA, inA, qA, rA, n) + contactEffectiveMass(iB, inB, qB, rB, n);
    if (den <= kEps) return;
    const float lambda = (pen / den) * cfg.depenetrationRelaxation;
    f3 tA = -n * (iA * lambda);
    f3 rotA = -mulWorldInvInertia(inA, qA, cross(rA, n)) * lambda;
    f3 tB = n * (iB * lambda);
    f3 rotB = mulWorldInvInertia(inB, qB, cross(rB, n)) * lambda;
    const f3 rel = (ptB - ppB) - (ptA - ppA);
    const f3 fd = positionFrictionDelta(projectOntoTangent(rel, n), pen, saturate(c.material.x), saturate(c.material.z),
                                        cfg.positionFrictionMinDistance);
    const float fdist = length(fd);
    if (fdist > 0.0f) {
        const f3 t = fd / fdist;
        const float tden = contactEffectiveMass(iA, inA, qA, rA, t) + contactEffectiveMass(iB, inB, qB, rB, t);
        if (tden > kEps) {
            const float tl = (fdist / tden) * cfg.depenetrationRelaxation;
            tA += t * (iA * tl);
            rotA += mulWorldInvInertia(inA, qA, cross(rA, t)) * tl;
            tB -= t * (iB * tl);
            rotB -= mulWorldInvInertia(inB, qB, cross(rB, t)) * tl;
        }
    }
    if (tyA == CN_BODY_DYNAMIC && iA != 0.0f) {
        atomicAdd(&s.bodyTransCorr[bA].x, tA.x); atomicAdd(&s.bodyTransCorr[bA].y, tA.y); atomicAdd(&s.bodyTransCorr[bA].z, tA.z);
        atomicAdd(&s.bodyRotCorr[bA].x, rotA.x); atomicAdd(&s.bodyRotCorr[bA].y, rotA.y); atomicAdd(&s.bodyRotCorr[bA].z, rotA.z);
    }
    if (tyB == CN_BODY_DYNAMIC && iB != 0.0f) {
        atomicAdd(&s.bodyTransCorr[bB].x, tB.x); atomicAdd(&s.bodyTransCorr[bB].y, tB.y); atomicAdd(&s.bodyTransCorr[bB].z, tB.z);
        atomicAdd(&s.bodyRotCorr[bB].x, rotB.x); atomicAdd(&s.bodyRotCorr[bB].y, rotB.y); atomicAdd(&s.bodyRotCorr[bB].z, rotB.z);
    }
}

// ------------------------------------------------------------------------- velocity solve
// physics_rigid_solve_contact_velocities.cs.hlsl: one body-pair group per thread, its slots in
// order, the contacts without a restitution target first; the velocity change goes to the
// bodies' corrections.
__global__ void k_rigidSolveVelocities(Scene s, Config cfg)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= s.meta_->rigidGroupCount) return;
    const uint2 gr = s.rrGroups[g];
    if (gr.y == 0u) return;
    const RigidPairContact c0 = s.rrContacts[s.rrValA[gr.x]];
    const uint32_t bA = min(c0.bodyA, c0.bodyB), bB = max(c0.bodyA, c0.bodyB);
    const float4 pA = s.predBodyPos[bA], pB = s.predBodyPos[bB];
    const float iA = s.bodyType[bA] == CN_BODY_DYNAMIC ? pA.w : 0.0f;
    const float iB = s.bodyType[bB] == CN_BODY_DYNAMIC ? pB.w : 0.0f;
    if (iA == 0.0f && iB == 0.0f) return;
    const float4 oA = qNormalize(s.predBodyRot[bA]), oB = qNormalize(s.predBodyRot[bB]);
    f3 inA = xyz(s.bodyInvInertia[bA]), inB = xyz(s.bodyInvInertia[bB]);
    if (iA == 0.0f) inA = f3{0.f, 0.f, 0.f};
    if (iB == 0.0f) inB = f3{0.f, 0.f, 0.f};
    const f3 lA0 = xyz(s.predBodyLin[bA]), lB0 = xyz(s.predBodyLin[bB]);
    const f3 aA0 = xyz(s.predBodyAng[bA]), aB0 = xyz(s.predBodyAng[bB]);
    f3 lA = lA0, lB = lB0, aA = aA0, aB = aB0;
    for (uint32_t pass = 0; pass < 2u; ++pass) {
        for (uint32_t k = 0; k < gr.y; ++k) {
            RigidSlot sl = s.rrSlots[gr.x + k];
            const bool hasRest = sl.state.y > 0.0f;
            if ((pass == 0u && hasRest) || (pass == 1u && !hasRest)) continue;
            const f3 n = safeNormalize(xyz(sl.normal), f3{0.f, 1.f, 0.f});
            const f3 ptA = xyz(pA) + qRotate(oA, xyz(sl.localA));
            const f3 ptB = xyz(pB) + qRotate(oB, xyz(sl.localB));
            const f3 rA = ptA - xyz(pA), rB = ptB - xyz(pB);
            const float nv = dot((lB + cross(aB, rB)) - (lA + cross(aA, rA)), n);
            const float pen = mx(penetrationFromPoints(ptA, ptB, n) - cfg.slop, 0.0f);
            const float nd = contactEffectiveMass(iA, inA, oA, rA, n) + contactEffectiveMass(iB, inB, oB, rB, n);
            if (nd <= kEps) continue;
            float vi = (sl.state.y - nv) / nd;
            if (vi < -sl.state.x) vi = -sl.state.x;
            const float pi = pen > 0.0f ? (cfg.velocityPenetrationStiffness * pen) / nd : 0.0f;
            const float applied = vi + pi;
            sl.state.x = sl.state.x + applied;
            if (fabsf(applied) > kEps) {
                const f3 imp = n * applied;
                if (iA > kEps) {
                    lA += -imp * iA;
                    aA += mulWorldInvInertia(inA, oA, cross(rA, -imp));
                }
                if (iB > kEps) {
                    lB += imp * iB;
                    aB += mulWorldInvInertia(inB, oB, cross(rB, imp));
                }
            }
            const float kf = saturate(sl.normal.w), sf = saturate(sl.localA.w);
            const f3 tv = projectOntoTangent((lB + cross(aB, rB)) - (lA + cross(aA, rA)), n);
            const float ts = length(tv);
            if (ts > 1.0e-5f) {
                const f3 t = tv / ts;
                const float td = contactEffectiveMass(iA, inA, oA, rA, t) + contactEffectiveMass(iB, inB, oB, rB, t);
                if (td > kEps) {
                    const float raw = -dot(tv, t) / td;
                    const float old = sl.state.z;
                    const float maxS = sf * sl.state.x, maxD = kf * sl.state.x;
                    const float un = old + raw;
                    float acc = un;
                    if (fabsf(un) > maxS) acc = mn(mx(un, -maxD), maxD);
                    const float at = acc - old;
                    sl.state.z = acc;
                    if (fabsf(at) > kEps) {
                        const f3 ti = t * at;
                        if (iA > kEps) {
                            lA += -ti * iA;
                            aA += mulWorldInvInertia(inA, oA, cross(rA, -ti));
                        }
                        if (iB > kEps) {
                            lB += ti * iB;
                            aB += mulWorldInvInertia(inB, oB, cross(rB, ti));
                        }
                    }
                }
            }
            s.rrSlots[gr.x + k] = sl;
        }
    }
    if (iA > kEps) {
        const f3 dl = lA - lA0, da = aA - aA0;
        atomicAdd(&s.bodyLinVelCorr[bA].x, dl.x); atomicAdd(&s.bodyLinVelCorr[bA].y, dl.y); atomicAdd(&s.bodyLinVelCorr[bA].z, dl.z);
        atomicAdd(&s.bodyAngVelCorr[bA].x, da.x); atomicAdd(&s.bodyAngVelCorr[bA].y, da.y); atomicAdd(&s.bodyAngVelCorr[bA].z, da.z);
    }
    if (iB > kEps) {
        const f3 dl = lB - lB0, da = aB - aB0;
        atomicAdd(&s.bodyLinVelCorr[bB].x, dl.x); atomicAdd(&s.bodyLinVelCorr[bB].y, dl.y); atomicAdd(&s.bodyLinVelCorr[bB].z, dl.z);
        atomicAdd(&s.bodyAngVelCorr[bB].x, da.x); atomicAdd(&s.bodyAngVelCorr[bB].y, da.y); atomicAdd(&s.bodyAngVelCorr[bB].z, da.z);
    }
}

// physics_rigid_apply_contact_velocities.cs.hlsl:14-58
__global__ void k_rigidApplyVelocityCorrections(Scene s, Config cfg)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.B) return;
    float4 lin = s.predBodyLin[b], ang = s.predBodyAng[b];
    if (s.bodyType[b] == CN_BODY_DYNAMIC) {
        f3 lc = xyz(s.bodyLinVelCorr[b]), ac = xyz(s.bodyAngVelCorr[b]);
        const float ll = length(lc), al = length(ac);
        if (ll > cfg.maxLinearVelocityCorrection && ll > kEps) lc = lc * (cfg.maxLinearVelocityCorrection / ll);
        if (al > cfg.maxAngularVelocityCorrection && al > kEps) ac = ac * (cfg.maxAngularVelocityCorrection / al);
        lin = mk4(xyz(lin) + lc, lin.w);
        ang = mk4(xyz(ang) + ac, ang.w);
    }
    s.predBodyLin[b] = lin;
    s.predBodyAng[b] = ang;
    s.bodyLinVelCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.bodyAngVelCorr[b] = make_float4(0.f, 0.f, 0.f, 0.f);
}

} // namespace

size_t rigidScratchBytes(uint32_t colliders, uint32_t pairs)
{
    const uint32_t n = colliders > pairs ? colliders : pairs;
    const size_t sortBytes = radixSortScratchBytes(n > 1u ? n : 1u);
    const size_t scan = scanScratchBytes(pairs > 1u ? pairs : 1u) + 4 * sizeof(uint32_t);
    return (sortBytes > scan ? sortBytes : scan) + 256;
}

void launchColliderBvh(const Scene &s, void *scratch, cudaStream_t st)
{
    const uint32_t n = s.colQueryCount;
    if (n < 2) return;
    void *work = static_cast<uint8_t *>(scratch) + 256;
    k_bvhBounds<<<1, kBoundsThreads, 0, st>>>(s);
    k_bvhMorton<<<blocksOf(n), kRigidThreads, 0, st>>>(s);
    radixSortPairs(s.bvhKeyA, s.bvhValA, s.bvhKeyB, s.bvhValB, n, work, &s.meta_->waitTimeouts, st);
    k_bvhBuild<<<blocksOf(n - 1), kRigidThreads, 0, st>>>(s);
    cudaMemsetAsync(s.bvhVisits, 0, sizeof(uint32_t) * (n - 1), st);
    k_bvhRefit<<<blocksOf(n), kRigidThreads, 0, st>>>(s);
}

void launchRigidBroadphaseAndContacts(const Scene &s, const Config &c, void *scratch, cudaStream_t st)
{
    const uint32_t n = s.colQueryCount;
    if (n < 2 || s.activeMovingCount == 0 || s.rrCapacity == 0) { // no collider pairs: proxy contacts alone
        cudaMemsetAsync(&s.meta_->rigidRigidPairCount, 0, 6 * sizeof(uint32_t), st);
        return;
    }
    uint32_t *total = static_cast<uint32_t *>(scratch);
    void *work = static_cast<uint8_t *>(scratch) + 256;
    if (!s.colBvh) launchColliderBvh(s, scratch, st); // else built after the rigid predict already
    // one warp per block: the walks are latency-bound chains, so they go to as many SMs as possible
    const unsigned pairBlocks = unsigned((s.activeMovingCount + 31u) / 32u);
    k_rigidPairsCount<<<pairBlocks, 32, 0, st>>>(s);
    exclusiveScan(s.rrCount, s.rrOffset, s.activeMovingCount, total, work, st);
    k_rigidPairsEmit<<<pairBlocks, 32, 0, st>>>(s, total);
    k_rigidNarrowPhase<<<blocksOf(s.rrCapacity), kRigidThreads, 0, st>>>(s, c);
}

void launchProxyRigidContacts(const Scene &s, cudaStream_t st)
{
    if (s.proxyCapacity == 0 || s.nProxy == 0) return;
    k_proxyRigidContacts<<<blocksOf(s.proxyCapacity), kRigidThreads, 0, st>>>(s);
}

void launchRigidVelocityInit(const Scene &s, const Config &c, void *scratch, cudaStream_t st)
{
    if (s.rrSlotCapacity == 0) return;
    uint32_t *total = static_cast<uint32_t *>(scratch);
    void *work = static_cast<uint8_t *>(scratch) + 256;
    const uint32_t slots = s.rrSlotCapacity;
    k_rigidGroupKeys<<<blocksOf(slots), kRigidThreads, 0, st>>>(s);
    radixSortPairs(s.rrKeyA, s.rrValA, s.rrKeyB, s.rrValB, slots, work, &s.meta_->waitTimeouts, st,
                   &s.meta_->rigidContactSlots);
    k_rigidGroupHeads<<<blocksOf(slots), kRigidThreads, 0, st>>>(s);
    exclusiveScan(s.rrHead, s.rrGroupOf, slots, total, work, st);
    k_rigidGroupInit<<<blocksOf(slots), kRigidThreads, 0, st>>>(s, c, total);
}

void launchRigidDepenetration(const Scene &s, const Config &c, cudaStream_t st)
{
    if (s.rrSlotCapacity == 0) return;
    k_rigidDepenetrate<<<blocksOf(s.rrSlotCapacity), kRigidThreads, 0, st>>>(s, c);
}

void launchRigidContactVelocitySolve(const Scene &s, const Config &c, uint32_t iterations, uint32_t contactIterations,
                                     cudaStream_t st)
{
    if (s.B == 0) return;
    for (uint32_t it = 0; it < iterations; ++it) {
        if (it < contactIterations && s.rrSlotCapacity)
            k_rigidSolveVelocities<<<blocksOf(s.rrSlotCapacity), kRigidThreads, 0, st>>>(s, c);
        k_rigidApplyVelocityCorrections<<<blocksOf(s.B), kRigidThreads, 0, st>>>(s, c);
    }
}

} // namespace cn
