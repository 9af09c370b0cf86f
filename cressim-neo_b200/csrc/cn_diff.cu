// cn_diff.cu -- differentiable XPBD rollout: forward substeps with checkpoints and a hand-written
// adjoint (no reference counterpart: the reference has no gradients).
//
// The rollout is the soft-body substep of the particle path -- predict, `iterations` Jacobi
// iterations of edge-distance then tet-volume constraints (solve writes per-constraint correction
// records, apply gathers them per particle in ascending constraint order), velocity update --
// with pinned particles and no contacts.  The forward math below follows the product kernels
// (k_predictKeys, k_solveEdges, k_applyPair, k_solveTets, k_applyQuad, k_updateVelocities)
// expression for expression, so in float it reproduces their bits.
//
// The adjoint runs the iterations backwards: per constraint, the Jacobian of (corrections,
// lambda') with respect to (positions, lambda, compliance) comes from the same templated
// constraint code evaluated on forward-mode dual numbers, and the vector-Jacobian products are
// written as per-constraint records that each particle gathers in ascending constraint order
// (deterministic, no atomics).  Positions and velocities are checkpointed at the start of every
// `checkpoint_interval`-th substep; backward recomputes one segment of substeps from its
// checkpoint, then one substep's iteration states at a time.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_internal.h"

using cn::setError;

namespace {

constexpr int kDiffThreads = 256;
inline unsigned gridOf(size_t n) { return n == 0 ? 1u : unsigned((n + kDiffThreads - 1) / kDiffThreads); }

// ---------------------------------------------------------------- scalar types
// A value with K tangents (forward mode).  Only the operations the constraint code uses.
template <class T, int K> struct Dual {
    T v;
    T d[K];
};
template <class T> __host__ __device__ __forceinline__ T val(T x) { return x; }
template <class T, int K> __host__ __device__ __forceinline__ T val(const Dual<T, K> &x) { return x.v; }

template <class T, int K> __device__ __forceinline__ Dual<T, K> mkc(T c)
{
    Dual<T, K> r;
    r.v = c;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = T(0);
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> operator+(const Dual<T, K> &a, const Dual<T, K> &b)
{
    Dual<T, K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> operator-(const Dual<T, K> &a, const Dual<T, K> &b)
{
    Dual<T, K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> operator-(const Dual<T, K> &a)
{
    Dual<T, K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> operator*(const Dual<T, K> &a, const Dual<T, K> &b)
{
    Dual<T, K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> operator/(const Dual<T, K> &a, const Dual<T, K> &b)
{
    Dual<T, K> r;
    r.v = a.v / b.v;
    const T inv = T(1) / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
template <class T, int K> __device__ __forceinline__ Dual<T, K> sqrtD(const Dual<T, K> &a)
{
    Dual<T, K> r;
    r.v = sqrt(a.v);
    const T h = T(0.5) / r.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
    return r;
}
__device__ __forceinline__ float sqrtD(float a) { return sqrtf(a); }
__device__ __forceinline__ double sqrtD(double a) { return sqrt(a); }

// a scalar constant of the same type as `like`
template <class T> __device__ __forceinline__ T cst(T, double c) { return T(c); }
template <class T, int K> __device__ __forceinline__ Dual<T, K> cst(const Dual<T, K> &, double c) { return mkc<T, K>(T(c)); }

template <class S> struct V3 {
    S x, y, z;
};
template <class S> __device__ __forceinline__ V3<S> operator+(const V3<S> &a, const V3<S> &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> __device__ __forceinline__ V3<S> operator-(const V3<S> &a, const V3<S> &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> __device__ __forceinline__ V3<S> operator-(const V3<S> &a) { return {-a.x, -a.y, -a.z}; }
template <class S> __device__ __forceinline__ V3<S> operator*(const V3<S> &a, const S &s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> __device__ __forceinline__ V3<S> operator*(const S &s, const V3<S> &a) { return {s * a.x, s * a.y, s * a.z}; }
template <class S> __device__ __forceinline__ V3<S> operator/(const V3<S> &a, const S &s) { return {a.x / s, a.y / s, a.z / s}; }
template <class S> __device__ __forceinline__ S dot3(const V3<S> &a, const V3<S> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> __device__ __forceinline__ V3<S> cross3(const V3<S> &a, const V3<S> &b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <class T> struct P4 {
    T x, y, z, w;
};

// ---------------------------------------------------------------- constraint math
// physics_soft_solve_edge_constraints.cs.hlsl:10-74 (k_solveEdges).  Returns false when the
// record is written as zeros (disabled, no mass, zero length, no denominator): then lambda' = lambda.
template <class S, class T>
__device__ __forceinline__ bool edgeProject(const V3<S> &a, const V3<S> &b, T wA, T wB, T rest, const S &compliance,
                                            const S &lambda, T dt, T relax, V3<S> &cA, V3<S> &cB, S &lambdaOut)
{
    const T eps = T(1.0e-6);
    const T wSum = wA + wB;
    const V3<S> delta = b - a;
    const S l2 = dot3(delta, delta);
    lambdaOut = lambda;
    if (!(wSum > eps && val(l2) > eps)) return false;
    const S len = sqrtD(l2);
    const V3<S> gA = (-delta) / len;
    const V3<S> gB = -gA;
    const T dt2 = dt * dt;
    const S alpha = compliance / cst(l2, dt2 > eps ? dt2 : eps); // max(compliance, 0): compliance > 0 here
    const S Cv = len - cst(l2, rest);
    const S den = cst(l2, wSum) + alpha;
    if (!(val(den) > eps)) return false;
    const S dl = -(Cv + alpha * lambda) / den;
    lambdaOut = lambda + dl;
    cA = ((cst(l2, wA) * dl) * gA) * cst(l2, relax);
    cB = ((cst(l2, wB) * dl) * gB) * cst(l2, relax);
    return true;
}

// |x| given the sign s of x: fabs for plain scalars (bit-exact), s * x on duals (the derivative).
__device__ __forceinline__ float absSigned(float x, float) { return fabsf(x); }
__device__ __forceinline__ double absSigned(double x, double) { return fabs(x); }
template <class T, int K> __device__ __forceinline__ Dual<T, K> absSigned(const Dual<T, K> &x, const Dual<T, K> &s)
{
    return s * x;
}

// physics_soft_solve_tet_constraints.cs.hlsl:15-87 (k_solveTets).  Returns false when the
// reference keeps the previous record (no mass, no denominator).
template <class S, class T>
__device__ __forceinline__ bool tetProject(const V3<S> p[4], const T w[4], T rest, const S &compliance,
                                           const S &lambda, T dt, T relax, V3<S> out[4], S &lambdaOut)
{
    const T eps = T(1.0e-6);
    lambdaOut = lambda;
    if ((w[0] + w[1] + w[2] + w[3]) <= eps) return false;
    const S sv = dot3(cross3(p[1] - p[0], p[2] - p[0]), p[3] - p[0]) / cst(lambda, 6.0);
    const T vsv = val(sv) >= T(0) ? T(1) : T(-1);
    const S vs = cst(lambda, vsv);
    const S Cv = absSigned(sv, vs) - cst(lambda, rest > T(0) ? rest : T(0));
    const S k6 = vs / cst(lambda, 6.0);
    const V3<S> g0 = cross3(p[3] - p[1], p[2] - p[1]) * k6;
    const V3<S> g1 = cross3(p[2] - p[0], p[3] - p[0]) * k6;
    const V3<S> g2 = cross3(p[3] - p[0], p[1] - p[0]) * k6;
    const V3<S> g3 = cross3(p[1] - p[0], p[2] - p[0]) * k6;
    const S sg = cst(lambda, w[0]) * dot3(g0, g0) + cst(lambda, w[1]) * dot3(g1, g1) +
                 cst(lambda, w[2]) * dot3(g2, g2) + cst(lambda, w[3]) * dot3(g3, g3);
    const T dt2 = dt * dt;
    const S alpha = compliance / cst(lambda, dt2 > eps ? dt2 : eps);
    const S den = sg + alpha;
    if (!(val(den) > eps)) return false;
    const S dl = -(Cv + alpha * lambda) / den;
    lambdaOut = lambda + dl;
    const V3<S> g[4] = {g0, g1, g2, g3};
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = ((cst(lambda, w[k]) * dl) * g[k]) * cst(lambda, relax);
    return true;
}


// ---------------------------------------------------------------- device scene
template <class T> struct DScene {
    uint32_t N = 0, E = 0, T_ = 0;
    const T *w = nullptr;          // inverse mass
    const T *damp = nullptr;       // per-particle velocity damping (contact material .z)
    const uint2 *edgePair = nullptr;
    const T *edgeRest = nullptr, *edgeCompliance = nullptr;
    const uint32_t *edgeEnabled = nullptr;
    const uint4 *tetIdx = nullptr;
    const T *tetRest = nullptr;
    const uint2 *edgeRanges = nullptr, *edgeInc = nullptr, *tetRanges = nullptr, *tetInc = nullptr;
    T g[3] = {T(0), T(0), T(0)};
    T relax = T(0.2);
};

template <class T> __device__ __forceinline__ V3<T> xyzOf(const P4<T> &p) { return {p.x, p.y, p.z}; }

// k_predictKeys for a solid particle (gravity scale 1)
template <class T> __global__ void k_dPredict(DScene<T> s, P4<T> *x, P4<T> *v, P4<T> *xprev, T dt)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    const P4<T> p = x[i];
    xprev[i] = {p.x, p.y, p.z, T(0)};
    if (s.w[i] <= T(1.0e-6)) {
        v[i] = {T(0), T(0), T(0), T(0)};
        return;
    }
    const P4<T> vv = v[i];
    const T gs = dt * T(1);
    const V3<T> vel = V3<T>{vv.x, vv.y, vv.z} + V3<T>{s.g[0], s.g[1], s.g[2]} * gs;
    const V3<T> pp = V3<T>{p.x, p.y, p.z} + vel * dt;
    v[i] = {vel.x, vel.y, vel.z, T(0)};
    x[i] = {pp.x, pp.y, pp.z, p.w};
}

template <class T>
__global__ void k_dEdges(DScene<T> s, const P4<T> *x, T *lambda, P4<T> *corr, T dt)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= s.E) return;
    const uint2 ab = s.edgePair[e];
    V3<T> cA{T(0), T(0), T(0)}, cB = cA;
    T lo = lambda[e];
    if (s.edgeEnabled[e] != 0u)
        edgeProject<T, T>(xyzOf(x[ab.x]), xyzOf(x[ab.y]), s.w[ab.x], s.w[ab.y], s.edgeRest[e],
                          s.edgeCompliance[e] > T(0) ? s.edgeCompliance[e] : T(0), lambda[e], dt, s.relax, cA, cB, lo);
    lambda[e] = lo;
    corr[2 * e] = {cA.x, cA.y, cA.z, T(0)};
    corr[2 * e + 1] = {cB.x, cB.y, cB.z, T(0)};
}

template <class T>
__global__ void k_dTets(DScene<T> s, const P4<T> *x, const T *compliance, T *lambda, P4<T> *corr, T dt)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s.T_) return;
    const uint4 q = s.tetIdx[t];
    const uint32_t id[4] = {q.x, q.y, q.z, q.w};
    V3<T> p[4];
    T w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        p[k] = xyzOf(x[id[k]]);
        w[k] = s.w[id[k]];
    }
    V3<T> out[4];
    T lo;
    if (!tetProject<T, T>(p, w, s.tetRest[t], compliance[t] > T(0) ? compliance[t] : T(0), lambda[t], dt, s.relax,
                          out, lo))
        return; // the previous record stays (the reference's behaviour)
    lambda[t] = lo;
#pragma unroll
    for (int k = 0; k < 4; ++k) corr[4 * t + k] = {out[k].x, out[k].y, out[k].z, T(0)};
}

// k_applyPair / k_applyQuad
template <class T, int kPer>
__global__ void k_dApply(DScene<T> s, P4<T> *x, const uint2 *ranges, const uint2 *inc, const P4<T> *corr)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    if (s.w[i] <= T(1.0e-6)) return;
    const P4<T> p = x[i];
    const uint2 r = ranges[i];
    V3<T> total{T(0), T(0), T(0)};
    for (uint32_t k = 0; k < r.y; ++k) {
        const uint2 ref = inc[r.x + k];
        const P4<T> c = corr[kPer * ref.x + (kPer == 2 ? (ref.y == 0u ? 0u : 1u) : (ref.y > 3u ? 3u : ref.y))];
        total = total + V3<T>{c.x, c.y, c.z};
    }
    const V3<T> n = V3<T>{p.x, p.y, p.z} + total;
    x[i] = {n.x, n.y, n.z, p.w};
}

// k_updateVelocities for a solid particle
template <class T> __global__ void k_dVelocity(DScene<T> s, const P4<T> *x, const P4<T> *xprev, P4<T> *v, T dt)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    if (s.w[i] <= T(1.0e-6) || dt <= T(1.0e-6)) {
        v[i] = {T(0), T(0), T(0), T(0)};
        return;
    }
    const T d = s.damp[i] > T(0) ? s.damp[i] : T(0);
    const T a = T(1) - d * dt;
    const T ds = a > T(0) ? a : T(0);
    const V3<T> vel = ((xyzOf(x[i]) - xyzOf(xprev[i])) / dt) * ds;
    v[i] = {vel.x, vel.y, vel.z, T(0)};
}

// ---------------------------------------------------------------- adjoint kernels
// Edge: inputs (a xyz, b xyz, lambda, compliance) -> outputs (cA, cB, lambda').  Writes the
// adjoints of a and b as records (2 per edge), accumulates d loss / d lambda into gLambda
// (replaced by the adjoint of the input lambda).  Edge compliance is not a parameter here.
template <class T>
__global__ void k_dEdgesBack(DScene<T> s, const P4<T> *x, const T *lambdaIn, const P4<T> *gX, T *gLambda,
                             P4<T> *rec, T dt)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= s.E) return;
    const uint2 ab = s.edgePair[e];
    typedef Dual<T, 7> D;
    V3<D> a, b;
    const V3<T> xa = xyzOf(x[ab.x]), xb = xyzOf(x[ab.y]);
    a = {mkc<T, 7>(xa.x), mkc<T, 7>(xa.y), mkc<T, 7>(xa.z)};
    b = {mkc<T, 7>(xb.x), mkc<T, 7>(xb.y), mkc<T, 7>(xb.z)};
    a.x.d[0] = a.y.d[1] = a.z.d[2] = T(1);
    b.x.d[3] = b.y.d[4] = b.z.d[5] = T(1);
    D lam = mkc<T, 7>(lambdaIn[e]);
    lam.d[6] = T(1);
    const D comp = mkc<T, 7>(s.edgeCompliance[e] > T(0) ? s.edgeCompliance[e] : T(0));
    V3<D> cA{mkc<T, 7>(T(0)), mkc<T, 7>(T(0)), mkc<T, 7>(T(0))}, cB = cA;
    D lo = lam;
    bool wrote = false;
    if (s.edgeEnabled[e] != 0u)
        wrote = edgeProject<D, T>(a, b, s.w[ab.x], s.w[ab.y], s.edgeRest[e], comp, lam, dt, s.relax, cA, cB, lo);
    // upstream adjoints: corrections reach particles with mass only (the apply skips the rest)
    const T gl = gLambda[e];
    T gin[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) gin[k] = gl * lo.d[k];
    if (wrote) {
        const P4<T> ga = s.w[ab.x] > T(1.0e-6) ? gX[ab.x] : P4<T>{T(0), T(0), T(0), T(0)};
        const P4<T> gb = s.w[ab.y] > T(1.0e-6) ? gX[ab.y] : P4<T>{T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int k = 0; k < 7; ++k)
            gin[k] += ga.x * cA.x.d[k] + ga.y * cA.y.d[k] + ga.z * cA.z.d[k] + gb.x * cB.x.d[k] + gb.y * cB.y.d[k] +
                      gb.z * cB.z.d[k];
    }
    rec[2 * e] = {gin[0], gin[1], gin[2], T(0)};
    rec[2 * e + 1] = {gin[3], gin[4], gin[5], T(0)};
    gLambda[e] = gin[6];
}

// Tet: inputs (4 positions, lambda, compliance) -> outputs (4 corrections, lambda').
template <class T>
__global__ void k_dTetsBack(DScene<T> s, const P4<T> *x, const T *compliance, const T *lambdaIn, const P4<T> *gX,
                            T *gLambda, P4<T> *rec, T *gCompliance, T dt)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s.T_) return;
    typedef Dual<T, 14> D;
    const uint4 q = s.tetIdx[t];
    const uint32_t id[4] = {q.x, q.y, q.z, q.w};
    V3<D> p[4];
    T w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const V3<T> xp = xyzOf(x[id[k]]);
        p[k] = {mkc<T, 14>(xp.x), mkc<T, 14>(xp.y), mkc<T, 14>(xp.z)};
        p[k].x.d[3 * k] = p[k].y.d[3 * k + 1] = p[k].z.d[3 * k + 2] = T(1);
        w[k] = s.w[id[k]];
    }
    D lam = mkc<T, 14>(lambdaIn[t]);
    lam.d[12] = T(1);
    const T c0 = compliance[t];
    D comp = mkc<T, 14>(c0 > T(0) ? c0 : T(0));
    comp.d[13] = c0 > T(0) ? T(1) : T(0);
    V3<D> out[4];
    D lo;
    const bool wrote = tetProject<D, T>(p, w, s.tetRest[t], comp, lam, dt, s.relax, out, lo);
    const T gl = gLambda[t];
    T gin[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) gin[k] = wrote ? gl * lo.d[k] : (k == 12 ? gl : T(0));
    if (wrote) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (w[j] <= T(1.0e-6)) continue;
            const P4<T> g = gX[id[j]];
#pragma unroll
            for (int k = 0; k < 14; ++k) gin[k] += g.x * out[j].x.d[k] + g.y * out[j].y.d[k] + g.z * out[j].z.d[k];
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) rec[4 * t + j] = {gin[3 * j], gin[3 * j + 1], gin[3 * j + 2], T(0)};
    gLambda[t] = gin[12];
    gCompliance[t] += gin[13];
}

// gX_in[i] = gX_out[i] + sum of the records of i's incident constraints (ascending order)
template <class T, int kPer>
__global__ void k_dGather(DScene<T> s, const P4<T> *gOut, P4<T> *gIn, const uint2 *ranges, const uint2 *inc,
                          const P4<T> *rec)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    const P4<T> g = gOut[i];
    const uint2 r = ranges[i];
    V3<T> total{g.x, g.y, g.z};
    for (uint32_t k = 0; k < r.y; ++k) {
        const uint2 ref = inc[r.x + k];
        const P4<T> c = rec[kPer * ref.x + (kPer == 2 ? (ref.y == 0u ? 0u : 1u) : (ref.y > 3u ? 3u : ref.y))];
        total = total + V3<T>{c.x, c.y, c.z};
    }
    gIn[i] = {total.x, total.y, total.z, T(0)};
}

// Velocity update + predict, backwards.  In: gX (adjoint of the substep's end positions),
// gV (of its end velocities), gX0 is overwritten: first with the adjoint entering the last
// iteration, later (k_dPredictBack) with the adjoint of the substep's start positions.
template <class T> __global__ void k_dVelocityBack(DScene<T> s, const P4<T> *gX, const P4<T> *gV, P4<T> *gXI, T dt)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    P4<T> g = gX[i];
    if (s.w[i] > T(1.0e-6) && dt > T(1.0e-6)) {
        const T d = s.damp[i] > T(0) ? s.damp[i] : T(0);
        const T a = T(1) - d * dt;
        const T k = (a > T(0) ? a : T(0)) / dt;
        const P4<T> gv = gV[i];
        g.x += gv.x * k;
        g.y += gv.y * k;
        g.z += gv.z * k;
    }
    gXI[i] = g;
}

template <class T>
__global__ void k_dPredictBack(DScene<T> s, const P4<T> *gX0, const P4<T> *gV, P4<T> *gXs, P4<T> *gVs, T dt)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.N) return;
    const P4<T> g0 = gX0[i];
    P4<T> gx = {g0.x, g0.y, g0.z, T(0)};
    P4<T> gv = {T(0), T(0), T(0), T(0)};
    if (s.w[i] > T(1.0e-6)) {
        if (dt > T(1.0e-6)) {
            const T d = s.damp[i] > T(0) ? s.damp[i] : T(0);
            const T a = T(1) - d * dt;
            const T k = (a > T(0) ? a : T(0)) / dt;
            const P4<T> g = gV[i];
            gx.x -= g.x * k;
            gx.y -= g.y * k;
            gx.z -= g.z * k;
        }
        gv = {g0.x * dt, g0.y * dt, g0.z * dt, T(0)};
    }
    gXs[i] = gx;
    gVs[i] = gv;
}

// ---------------------------------------------------------------- host engine
template <class T> struct Engine {
    DScene<T> s;
    uint32_t iterations = 1, substeps = 1, interval = 8;
    T dt = T(0);
    // owned device buffers
    std::vector<void *> owned;
    P4<T> *x = nullptr, *v = nullptr, *xprev = nullptr;
    T *lamE = nullptr, *lamT = nullptr;
    P4<T> *corrE = nullptr, *corrT = nullptr;
    P4<T> *ckX = nullptr, *ckV = nullptr;     // checkpoints: (substeps / interval + 1) x N
    P4<T> *segX = nullptr, *segV = nullptr;   // one segment's substep starts: interval x N
    P4<T> *itX0 = nullptr, *itX1 = nullptr;   // one substep's iteration states: iterations x N
    T *itLE = nullptr, *itLT = nullptr;       // iterations x E, iterations x T
    P4<T> *gX = nullptr, *gV = nullptr, *gA = nullptr, *gB = nullptr;
    T *gLE = nullptr, *gLT = nullptr;
    P4<T> *recE = nullptr, *recT = nullptr;
    const T *compliance = nullptr;            // the forward's tet compliances (caller's device buffer)
    bool forwardDone = false;

    template <class U> U *alloc(size_t n)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(U)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        owned.push_back(p); // a null entry marks a failed allocation
        return static_cast<U *>(p);
    }
    void release()
    {
        for (void *p : owned)
            if (p) cudaFree(p);
        owned.clear();
    }
};

void copyAsync(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
}

template <class T> void runIteration(Engine<T> &g, P4<T> *x, cudaStream_t st)
{
    const DScene<T> &s = g.s;
    if (s.E) {
        k_dEdges<T><<<gridOf(s.E), kDiffThreads, 0, st>>>(s, x, g.lamE, g.corrE, g.dt);
        k_dApply<T, 2><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, s.edgeRanges, s.edgeInc, g.corrE);
    }
    if (s.T_) {
        k_dTets<T><<<gridOf(s.T_), kDiffThreads, 0, st>>>(s, x, g.compliance, g.lamT, g.corrT, g.dt);
        k_dApply<T, 4><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, s.tetRanges, s.tetInc, g.corrT);
    }
}

// One substep from (x, v) in place; with `record`, the iteration states for the adjoint.
template <class T> void runSubstep(Engine<T> &g, P4<T> *x, P4<T> *v, bool record, cudaStream_t st)
{
    const DScene<T> &s = g.s;
    const size_t nb = sizeof(P4<T>) * s.N;
    k_dPredict<T><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, v, g.xprev, g.dt);
    if (s.E) cudaMemsetAsync(g.lamE, 0, sizeof(T) * s.E, st);
    if (s.T_) cudaMemsetAsync(g.lamT, 0, sizeof(T) * s.T_, st);
    for (uint32_t it = 0; it < g.iterations; ++it) {
        if (record) {
            copyAsync(g.itX0 + size_t(it) * s.N, x, nb, st);
            copyAsync(g.itLE + size_t(it) * s.E, g.lamE, sizeof(T) * s.E, st);
        }
        if (s.E) {
            k_dEdges<T><<<gridOf(s.E), kDiffThreads, 0, st>>>(s, x, g.lamE, g.corrE, g.dt);
            k_dApply<T, 2><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, s.edgeRanges, s.edgeInc, g.corrE);
        }
        if (record) {
            copyAsync(g.itX1 + size_t(it) * s.N, x, nb, st);
            copyAsync(g.itLT + size_t(it) * s.T_, g.lamT, sizeof(T) * s.T_, st);
        }
        if (s.T_) {
            k_dTets<T><<<gridOf(s.T_), kDiffThreads, 0, st>>>(s, x, g.compliance, g.lamT, g.corrT, g.dt);
            k_dApply<T, 4><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, s.tetRanges, s.tetInc, g.corrT);
        }
    }
    k_dVelocity<T><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, x, g.xprev, v, g.dt);
}

template <class T> cn_status forward(Engine<T> &g, const T *compliance, const P4<T> *x0, const P4<T> *v0, P4<T> *xOut,
                                     P4<T> *vOut, cudaStream_t st)
{
    const size_t nb = sizeof(P4<T>) * g.s.N;
    g.compliance = compliance;
    copyAsync(g.x, x0, nb, st);
    copyAsync(g.v, v0, nb, st);
    // corrections start at zero (the solver's upload clears them)
    if (g.s.E) cudaMemsetAsync(g.corrE, 0, sizeof(P4<T>) * 2 * g.s.E, st);
    if (g.s.T_) cudaMemsetAsync(g.corrT, 0, sizeof(P4<T>) * 4 * g.s.T_, st);
    for (uint32_t sub = 0; sub < g.substeps; ++sub) {
        if (sub % g.interval == 0) {
            const size_t c = sub / g.interval;
            copyAsync(g.ckX + c * g.s.N, g.x, nb, st);
            copyAsync(g.ckV + c * g.s.N, g.v, nb, st);
        }
        runSubstep(g, g.x, g.v, false, st);
    }
    if (xOut) copyAsync(xOut, g.x, nb, st);
    if (vOut) copyAsync(vOut, g.v, nb, st);
    g.forwardDone = true;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return setError(CN_ERR_CUDA, std::string("cn_diff_forward: ") + cudaGetErrorString(e));
    return CN_OK;
}

// The stale-record case of the tet solve (a record kept from an earlier iteration) carries no
// derivative here: it only arises for tets whose four particles are all pinned (their records are
// never applied) or whose denominator vanishes.
template <class T> cn_status backward(Engine<T> &g, const P4<T> *gXOut, const P4<T> *gVOut, T *gCompliance,
                                      P4<T> *gX0, P4<T> *gV0, cudaStream_t st)
{
    if (!g.forwardDone) return setError(CN_ERR_NOT_INITIALIZED, "cn_diff_backward: run cn_diff_forward first");
    const DScene<T> &s = g.s;
    const size_t nb = sizeof(P4<T>) * s.N;
    if (gXOut) copyAsync(g.gX, gXOut, nb, st); else cudaMemsetAsync(g.gX, 0, nb, st);
    if (gVOut) copyAsync(g.gV, gVOut, nb, st); else cudaMemsetAsync(g.gV, 0, nb, st);
    if (s.T_) cudaMemsetAsync(gCompliance, 0, sizeof(T) * s.T_, st);
    const uint32_t segments = (g.substeps + g.interval - 1) / g.interval;
    for (int seg = int(segments) - 1; seg >= 0; --seg) {
        const uint32_t first = uint32_t(seg) * g.interval;
        const uint32_t count = std::min(g.interval, g.substeps - first);
        // recompute the segment's substep starts from its checkpoint
        copyAsync(g.x, g.ckX + size_t(seg) * s.N, nb, st);
        copyAsync(g.v, g.ckV + size_t(seg) * s.N, nb, st);
        if (s.E) cudaMemsetAsync(g.corrE, 0, sizeof(P4<T>) * 2 * s.E, st);
        if (s.T_) cudaMemsetAsync(g.corrT, 0, sizeof(P4<T>) * 4 * s.T_, st);
        for (uint32_t k = 0; k < count; ++k) {
            copyAsync(g.segX + size_t(k) * s.N, g.x, nb, st);
            copyAsync(g.segV + size_t(k) * s.N, g.v, nb, st);
            if (k + 1 < count) runSubstep(g, g.x, g.v, false, st);
        }
        for (int k = int(count) - 1; k >= 0; --k) {
            // this substep's iteration states
            copyAsync(g.x, g.segX + size_t(k) * s.N, nb, st);
            copyAsync(g.v, g.segV + size_t(k) * s.N, nb, st);
            runSubstep(g, g.x, g.v, true, st);
            // velocity update backwards: gA = adjoint entering the last iteration's output
            k_dVelocityBack<T><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, g.gX, g.gV, g.gA, g.dt);
            if (s.E) cudaMemsetAsync(g.gLE, 0, sizeof(T) * s.E, st);
            if (s.T_) cudaMemsetAsync(g.gLT, 0, sizeof(T) * s.T_, st);
            for (int it = int(g.iterations) - 1; it >= 0; --it) {
                if (s.T_) {
                    k_dTetsBack<T><<<gridOf(s.T_), kDiffThreads, 0, st>>>(
                        s, g.itX1 + size_t(it) * s.N, g.compliance, g.itLT + size_t(it) * s.T_, g.gA, g.gLT, g.recT,
                        gCompliance, g.dt);
                    k_dGather<T, 4><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, g.gA, g.gB, s.tetRanges, s.tetInc,
                                                                         g.recT);
                    std::swap(g.gA, g.gB);
                }
                if (s.E) {
                    k_dEdgesBack<T><<<gridOf(s.E), kDiffThreads, 0, st>>>(
                        s, g.itX0 + size_t(it) * s.N, g.itLE + size_t(it) * s.E, g.gA, g.gLE, g.recE, g.dt);
                    k_dGather<T, 2><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, g.gA, g.gB, s.edgeRanges, s.edgeInc,
                                                                         g.recE);
                    std::swap(g.gA, g.gB);
                }
            }
            // predict backwards: (gX, gV) of the substep start
            k_dPredictBack<T><<<gridOf(s.N), kDiffThreads, 0, st>>>(s, g.gA, g.gV, g.gX, g.gV, g.dt);
        }
    }
    if (gX0) copyAsync(gX0, g.gX, nb, st);
    if (gV0) copyAsync(gV0, g.gV, nb, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return setError(CN_ERR_CUDA, std::string("cn_diff_backward: ") + cudaGetErrorString(e));
    return CN_OK;
}

template <class T> cn_status build(Engine<T> &g, const cn_world_soa &w, const cn_diff_desc &d)
{
    const uint32_t N = w.particle_count, E = w.edge_count, TT = w.tet_count;
    DScene<T> &s = g.s;
    s.N = N; s.E = E; s.T_ = TT;
    g.iterations = std::max<uint32_t>(d.iterations, 1u);
    g.substeps = std::max<uint32_t>(d.substeps, 1u);
    g.interval = std::max<uint32_t>(d.checkpoint_interval, 1u);
    g.dt = T(d.substep_dt);
    s.relax = T(d.relaxation);
    for (int k = 0; k < 3; ++k) s.g[k] = T(d.gravity[k]);
    std::vector<T> wv(N), damp(N);
    for (uint32_t i = 0; i < N; ++i) {
        wv[i] = T(w.positions_inv_mass[4 * i + 3]);
        const uint32_t m = w.material_indices[i];
        damp[i] = m < w.contact_material_count ? T(w.contact_materials[4 * m + 2]) : T(0);
    }
    std::vector<uint2> pairs(E);
    std::vector<T> rest(E), ecomp(E);
    std::vector<uint32_t> en(E);
    for (uint32_t e = 0; e < E; ++e) {
        pairs[e] = make_uint2(w.edges[e].particle_a, w.edges[e].particle_b);
        rest[e] = T(w.edges[e].rest_length);
        ecomp[e] = T(w.edges[e].compliance);
        en[e] = w.edges[e].enabled;
    }
    std::vector<uint4> tets(TT);
    std::vector<T> trest(TT);
    for (uint32_t t = 0; t < TT; ++t) {
        const cn_soft_tet &q = w.tets[t];
        tets[t] = make_uint4(q.particle_indices[0], q.particle_indices[1], q.particle_indices[2], q.particle_indices[3]);
        trest[t] = T(q.rest_volume);
    }
    const cn::Incidence eI = cn::buildIncidence(N, E, 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? w.edges[c].particle_a : w.edges[c].particle_b;
    });
    const cn::Incidence tI = cn::buildIncidence(N, TT, 4, [&](uint32_t c, uint32_t k) { return w.tets[c].particle_indices[k]; });
    auto upload = [&](auto *dst, const auto &vec) {
        if (!vec.empty()) cudaMemcpy(dst, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice);
    };
    T *dw = g.template alloc<T>(N), *ddamp = g.template alloc<T>(N);
    uint2 *dpairs = g.template alloc<uint2>(E);
    T *drest = g.template alloc<T>(E), *decomp = g.template alloc<T>(E);
    uint32_t *den = g.template alloc<uint32_t>(E);
    uint4 *dtets = g.template alloc<uint4>(TT);
    T *dtrest = g.template alloc<T>(TT);
    uint2 *eR = g.template alloc<uint2>(N), *eInc = g.template alloc<uint2>(eI.inc.size());
    uint2 *tR = g.template alloc<uint2>(N), *tInc = g.template alloc<uint2>(tI.inc.size());
    const size_t ck = g.substeps / g.interval + 1;
    g.x = g.template alloc<P4<T>>(N); g.v = g.template alloc<P4<T>>(N); g.xprev = g.template alloc<P4<T>>(N);
    g.lamE = g.template alloc<T>(E); g.lamT = g.template alloc<T>(TT);
    g.corrE = g.template alloc<P4<T>>(size_t(E) * 2); g.corrT = g.template alloc<P4<T>>(size_t(TT) * 4);
    g.ckX = g.template alloc<P4<T>>(ck * N); g.ckV = g.template alloc<P4<T>>(ck * N);
    g.segX = g.template alloc<P4<T>>(size_t(g.interval) * N); g.segV = g.template alloc<P4<T>>(size_t(g.interval) * N);
    g.itX0 = g.template alloc<P4<T>>(size_t(g.iterations) * N); g.itX1 = g.template alloc<P4<T>>(size_t(g.iterations) * N);
    g.itLE = g.template alloc<T>(size_t(g.iterations) * E); g.itLT = g.template alloc<T>(size_t(g.iterations) * TT);
    g.gX = g.template alloc<P4<T>>(N); g.gV = g.template alloc<P4<T>>(N);
    g.gA = g.template alloc<P4<T>>(N); g.gB = g.template alloc<P4<T>>(N);
    g.gLE = g.template alloc<T>(E); g.gLT = g.template alloc<T>(TT);
    g.recE = g.template alloc<P4<T>>(size_t(E) * 2); g.recT = g.template alloc<P4<T>>(size_t(TT) * 4);
    for (void *p : g.owned)
        if (!p) return setError(CN_ERR_OUT_OF_MEMORY, "cn_diff_set_scene: device allocation failed");
    upload(dw, wv); upload(ddamp, damp); upload(dpairs, pairs); upload(drest, rest); upload(decomp, ecomp);
    upload(den, en); upload(dtets, tets); upload(dtrest, trest);
    upload(eR, eI.ranges); upload(eInc, eI.inc); upload(tR, tI.ranges); upload(tInc, tI.inc);
    s.w = dw; s.damp = ddamp; s.edgePair = dpairs; s.edgeRest = drest; s.edgeCompliance = decomp; s.edgeEnabled = den;
    s.tetIdx = dtets; s.tetRest = dtrest; s.edgeRanges = eR; s.edgeInc = eInc; s.tetRanges = tR; s.tetInc = tInc;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return setError(CN_ERR_CUDA, std::string("cn_diff_set_scene: ") + cudaGetErrorString(e));
    return CN_OK;
}

} // namespace

struct cn_diff {
    cn_diff_desc desc{};
    int device = 0;
    cudaStream_t ownStream = nullptr;
    Engine<float> f32;
    Engine<double> f64;
    bool ready = false;
    uint32_t N = 0, T = 0;
};

extern "C" {

CN_API void cn_diff_desc_defaults(cn_diff_desc *d)
{
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->gravity[1] = -9.81f;
    d->substeps = 32;
    d->iterations = 20;
    d->substep_dt = 1.0f / 60.0f / 32.0f;
    d->relaxation = 0.2f;
    d->checkpoint_interval = 8;
    d->precision = 4;
}

CN_API cn_status cn_diff_create(const cn_diff_desc *d, int device, cn_diff **out)
{
    if (!d || !out) return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_create: null argument");
    *out = nullptr;
    if (d->precision != 4 && d->precision != 8) return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_create: precision is 4 or 8");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return setError(CN_ERR_NO_DEVICE, "cn_diff_create: no CUDA device");
    }
    if (device < 0 || device >= count) return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_create: bad device");
    auto *g = new cn_diff();
    g->desc = *d;
    g->device = device;
    cudaSetDevice(device);
    cudaStreamCreateWithFlags(&g->ownStream, cudaStreamNonBlocking);
    *out = g;
    return CN_OK;
}

CN_API void cn_diff_destroy(cn_diff *g)
{
    if (!g) return;
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    g->f32.release();
    g->f64.release();
    if (g->ownStream) cudaStreamDestroy(g->ownStream);
    delete g;
}

CN_API cn_status cn_diff_set_scene(cn_diff *g, const cn_world_soa *w)
{
    if (!g || !w) return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_set_scene: null argument");
    if (w->bend_count || w->dihedral_count || w->strand_segment_count || w->strand_joint_count ||
        w->strand_distance_count || w->collider_count)
        return setError(CN_ERR_UNSUPPORTED, "cn_diff_set_scene: the differentiable rollout covers edges and tets "
                                            "without colliders");
    for (uint32_t i = 0; i < w->particle_count; ++i)
        if (w->kinds[i] == CN_PARTICLE_FLUID || (w->owner_types && w->owner_types[i] == CN_OWNER_RIGID_BODY))
            return setError(CN_ERR_UNSUPPORTED, "cn_diff_set_scene: fluid or rigid proxy particles");
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    g->f32.release();
    g->f64.release();
    g->f32 = Engine<float>();
    g->f64 = Engine<double>();
    const cn_status st = g->desc.precision == 8 ? build(g->f64, *w, g->desc) : build(g->f32, *w, g->desc);
    if (st != CN_OK) return st;
    g->ready = true;
    g->N = w->particle_count;
    g->T = w->tet_count;
    return CN_OK;
}

CN_API cn_status cn_diff_forward(cn_diff *g, const void *tet_compliance, const void *x0, const void *v0, void *x_out,
                                 void *v_out, void *stream)
{
    if (!g || !g->ready || !tet_compliance || !x0 || !v0)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_forward: no scene or null buffer");
    cudaSetDevice(g->device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->ownStream;
    if (g->desc.precision == 8)
        return forward(g->f64, static_cast<const double *>(tet_compliance), static_cast<const P4<double> *>(x0),
                       static_cast<const P4<double> *>(v0), static_cast<P4<double> *>(x_out),
                       static_cast<P4<double> *>(v_out), st);
    return forward(g->f32, static_cast<const float *>(tet_compliance), static_cast<const P4<float> *>(x0),
                   static_cast<const P4<float> *>(v0), static_cast<P4<float> *>(x_out), static_cast<P4<float> *>(v_out),
                   st);
}

CN_API cn_status cn_diff_backward(cn_diff *g, const void *grad_x_out, const void *grad_v_out, void *grad_tet_compliance,
                                  void *grad_x0, void *grad_v0, void *stream)
{
    if (!g || !g->ready || !grad_tet_compliance)
        return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_backward: no scene or null buffer");
    cudaSetDevice(g->device);
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->ownStream;
    if (g->desc.precision == 8)
        return backward(g->f64, static_cast<const P4<double> *>(grad_x_out), static_cast<const P4<double> *>(grad_v_out),
                        static_cast<double *>(grad_tet_compliance), static_cast<P4<double> *>(grad_x0),
                        static_cast<P4<double> *>(grad_v0), st);
    return backward(g->f32, static_cast<const P4<float> *>(grad_x_out), static_cast<const P4<float> *>(grad_v_out),
                    static_cast<float *>(grad_tet_compliance), static_cast<P4<float> *>(grad_x0),
                    static_cast<P4<float> *>(grad_v0), st);
}

CN_API cn_status cn_diff_memory(cn_diff *g, uint64_t *bytes)
{
    if (!g || !bytes) return setError(CN_ERR_INVALID_ARGUMENT, "cn_diff_memory: null argument");
    const Engine<float> &a = g->f32;
    const Engine<double> &b = g->f64;
    const size_t es = g->desc.precision == 8 ? 8 : 4;
    const uint32_t iters = g->desc.precision == 8 ? b.iterations : a.iterations;
    const uint32_t subs = g->desc.precision == 8 ? b.substeps : a.substeps;
    const uint32_t interval = g->desc.precision == 8 ? b.interval : a.interval;
    const uint32_t E = g->desc.precision == 8 ? b.s.E : a.s.E;
    const size_t N = g->N, T = g->T;
    // the state saved for the adjoint: checkpoints, one segment, one substep's iterations
    *bytes = uint64_t((subs / interval + 1) * 2 * N * 4 * es + size_t(interval) * 2 * N * 4 * es +
                      size_t(iters) * (2 * N * 4 * es + (E + T) * es));
    return CN_OK;
}

} // extern "C"
