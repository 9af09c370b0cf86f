// cn_math.cuh -- float3/float4 and quaternion helpers for the particle substep kernels.
//
// Each helper evaluates in the same operation order as the reference HLSL helper it
// names (assets/shaders/include/physics/core/physics_math.hlsli,
// collision/physics_shape_common.hlsli, rigid/physics_rigid_solver_shared.hlsli,
// fluid/physics_fluid_common.hlsli).  The library is compiled with --fmad=false and
// IEEE division / square root, so a kernel that follows the reference's expression
// order produces the same float32 bits as a CPU evaluation of that order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cn {

constexpr float kEps = 1.0e-6f;           // physics_base.hlsli:7
constexpr uint32_t kInvalid = 0xffffffffu; // physics_base.hlsli:6

struct f3 { float x, y, z; };

__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 xyz(float4 v) { return f3{v.x, v.y, v.z}; }
__host__ __device__ __forceinline__ float4 mk4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ f3 &operator+=(f3 &a, f3 b) { a = a + b; return a; }
__host__ __device__ __forceinline__ f3 &operator-=(f3 &a, f3 b) { a = a - b; return a; }
__host__ __device__ __forceinline__ float4 add4(float4 a, float4 b)
{
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__host__ __device__ __forceinline__ float4 scale4(float4 a, float s)
{
    return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float dot4(float4 a, float4 b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b)
{
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// std::max / std::min semantics (first operand returned on ties), shared with the oracle.
__host__ __device__ __forceinline__ float mx(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float mn(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float length(f3 v) { return sqrtf(dot(v, v)); }
__host__ __device__ __forceinline__ float saturate(float v) { return mn(mx(v, 0.0f), 1.0f); }
__host__ __device__ __forceinline__ f3 fabs3(f3 v) { return f3{fabsf(v.x), fabsf(v.y), fabsf(v.z)}; }
__host__ __device__ __forceinline__ f3 clamp3(f3 v, f3 lo, f3 hi)
{
    return f3{mn(mx(v.x, lo.x), hi.x), mn(mx(v.y, lo.y), hi.y), mn(mx(v.z, lo.z), hi.z)};
}
__host__ __device__ __forceinline__ f3 min3(f3 a, f3 b) { return f3{mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)}; }
__host__ __device__ __forceinline__ f3 max3(f3 a, f3 b) { return f3{mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)}; }
__host__ __device__ __forceinline__ f3 lerp3(f3 a, f3 b, float t) { return a + (b - a) * t; }

// physics_math.hlsli:6-20 (rsqrt evaluated as 1/sqrt)
__host__ __device__ __forceinline__ f3 safeNormalize(f3 v, f3 fallback)
{
    const float l2 = dot(v, v);
    if (l2 <= kEps) return fallback;
    return v * (1.0f / sqrtf(l2));
}
__host__ __device__ __forceinline__ float4 qNormalize(float4 q)
{
    const float l2 = dot4(q, q);
    if (l2 <= kEps) return make_float4(0.f, 0.f, 0.f, 1.f);
    return scale4(q, 1.0f / sqrtf(l2));
}
__host__ __device__ __forceinline__ float4 qConj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
// physics_math.hlsli:24-31
__host__ __device__ __forceinline__ float4 qMul(float4 a, float4 b)
{
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                       a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                       a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
                       a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
// physics_math.hlsli:33-37
__host__ __device__ __forceinline__ f3 qRotate(float4 q, f3 v)
{
    const f3 qv = xyz(q);
    const f3 t = 2.0f * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
__host__ __device__ __forceinline__ f3 qInvRotate(float4 q, f3 v) { return qRotate(qConj(q), v); }

// physics_math.hlsli:71-89
__device__ __forceinline__ f3 angularVelocityFromQuaternionDelta(float4 prev, float4 cur, float dt)
{
    if (dt <= kEps) return f3{0.f, 0.f, 0.f};
    float4 d = qMul(qNormalize(cur), qConj(qNormalize(prev)));
    if (d.w < 0.0f) d = make_float4(-d.x, -d.y, -d.z, -d.w);
    const f3 im = xyz(d);
    const float l2 = dot(im, im);
    if (l2 <= kEps) return im * (2.0f / dt);
    const float l = sqrtf(l2);
    const float angle = 2.0f * atan2f(l, d.w);
    return im * (angle / (l * dt));
}

// physics_math.hlsli:55-73: rotation-vector quaternion and orientation integration
__device__ __forceinline__ float4 qFromRotationVector(f3 rv)
{
    const float a2 = dot(rv, rv);
    if (a2 <= kEps) return qNormalize(mk4(rv * 0.5f, 1.0f));
    const float angle = sqrtf(a2);
    const float half = 0.5f * angle;
    const float sc = sinf(half) / angle;
    return qNormalize(mk4(rv * sc, cosf(half)));
}
__device__ __forceinline__ float4 integrateOrientation(float4 q, f3 w, float dt)
{
    return qNormalize(qMul(qFromRotationVector(w * dt), q));
}

// physics_shape_common.hlsli:24-42
__host__ __device__ __forceinline__ float sphereRadius(float4 p, float4 s)
{
    const f3 a = fabs3(xyz(s));
    return p.x * mx(a.x, mx(a.y, a.z));
}
__host__ __device__ __forceinline__ f3 boxHalfExtents(float4 p, float4 s) { return xyz(p) * fabs3(xyz(s)); }
__host__ __device__ __forceinline__ void capsuleSegment(f3 pos, float4 q, float4 p, float4 s, f3 &a, f3 &b,
                                                        float &r)
{
    const f3 as = fabs3(xyz(s));
    r = p.x * mx(as.x, as.z);
    const float hh = p.y * as.y;
    const f3 axis = qRotate(q, f3{0.f, 1.f, 0.f});
    a = pos - axis * hh;
    b = pos + axis * hh;
}
// physics_shape_common.hlsli:97-105
__host__ __device__ __forceinline__ f3 closestFaceNormalLocal(f3 lp, f3 h)
{
    const f3 d = h - fabs3(lp);
    if (d.x <= d.y && d.x <= d.z) return f3{lp.x >= 0.0f ? 1.0f : -1.0f, 0.f, 0.f};
    if (d.y <= d.z) return f3{0.f, lp.y >= 0.0f ? 1.0f : -1.0f, 0.f};
    return f3{0.f, 0.f, lp.z >= 0.0f ? 1.0f : -1.0f};
}
// physics_shape_common.hlsli:45-98: box axes, ComputeBodyAabb, closest point and support point
__host__ __device__ __forceinline__ void computeBodyAabb(uint32_t shape, f3 pos, float4 q, float4 p, float4 sc, f3 &mnv, f3 &mxv)
{
    f3 e{0.f, 0.f, 0.f};
    if (shape == CN_COLLIDER_SPHERE) {
        const float r = sphereRadius(p, sc);
        e = f3{r, r, r};
    } else if (shape == CN_COLLIDER_BOX) {
        const f3 h = boxHalfExtents(p, sc);
        e = fabs3(qRotate(q, f3{1.f, 0.f, 0.f})) * h.x + fabs3(qRotate(q, f3{0.f, 1.f, 0.f})) * h.y +
            fabs3(qRotate(q, f3{0.f, 0.f, 1.f})) * h.z;
    } else {
        f3 a, b;
        float r = 0.0f;
        capsuleSegment(pos, q, p, sc, a, b, r);
        const f3 axis = fabs3(qRotate(q, f3{0.f, 1.f, 0.f}));
        e = axis * (0.5f * length(b - a)) + f3{r, r, r};
    }
    mnv = pos - e;
    mxv = pos + e;
}

__host__ __device__ __forceinline__ f3 closestPointOnBox(f3 q, f3 c, float4 o, f3 h)
{
    const f3 lp = qInvRotate(o, q - c);
    return c + qRotate(o, clamp3(lp, -h, h));
}
__host__ __device__ __forceinline__ f3 boxSupportPoint(f3 c, float4 o, f3 h, f3 dir)
{
    const f3 ld = qInvRotate(o, dir);
    return c + qRotate(o, f3{ld.x >= 0.0f ? h.x : -h.x, ld.y >= 0.0f ? h.y : -h.y, ld.z >= 0.0f ? h.z : -h.z});
}
// physics_shape_common.hlsli:75-80
__host__ __device__ __forceinline__ bool aabbOverlaps(f3 minA, f3 maxA, f3 minB, f3 maxB)
{
    return minA.x <= maxB.x && maxA.x >= minB.x && minA.y <= maxB.y && maxA.y >= minB.y &&
           minA.z <= maxB.z && maxA.z >= minB.z;
}

// physics_rigid_solver_shared.hlsli:8-68
__host__ __device__ __forceinline__ f3 mulWorldInvInertia(f3 inv, float4 q, f3 v)
{
    const f3 ax = qRotate(q, f3{1.f, 0.f, 0.f});
    const f3 ay = qRotate(q, f3{0.f, 1.f, 0.f});
    const f3 az = qRotate(q, f3{0.f, 0.f, 1.f});
    return ax * (inv.x * dot(ax, v)) + ay * (inv.y * dot(ay, v)) + az * (inv.z * dot(az, v));
}
__host__ __device__ __forceinline__ float contactEffectiveMass(float invMass, f3 inv, float4 q, f3 r, f3 dir)
{
    if (invMass <= kEps) return 0.0f;
    const f3 am = mulWorldInvInertia(inv, q, cross(r, dir));
    return invMass + dot(cross(am, r), dir);
}
__host__ __device__ __forceinline__ f3 combineContactMaterial(float4 a, float4 b)
{
    const float friction = sqrtf(mx(0.0f, a.x) * mx(0.0f, b.x));
    const float restitution = mx(mx(0.0f, a.y), mx(0.0f, b.y));
    const float stat = sqrtf(mx(0.0f, a.w) * mx(0.0f, b.w));
    return f3{friction, restitution, stat};
}
__host__ __device__ __forceinline__ f3 projectOntoTangent(f3 v, f3 n) { return v - n * dot(v, n); }
__host__ __device__ __forceinline__ f3 positionFrictionDelta(f3 tdisp, float pen, float kinetic, float stat,
                                                             float minDistance)
{
    const float td = length(tdisp);
    if (td <= minDistance || pen <= kEps) return f3{0.f, 0.f, 0.f};
    const float sl = saturate(stat) * pen;
    if (td <= sl) return tdisp;
    return tdisp * mn(saturate(kinetic) * pen / td, 1.0f);
}

// physics_fluid_common.hlsli:17-66.  The shaders divide by the smoothing radius and by the pair
// distance; SPIR-V's OpFDiv is specified to 2.5 ulp, not correctly rounded, and these kernels
// (and the oracle) take each such quotient as the product with the correctly rounded reciprocal
// -- one reciprocal per particle (1 / h) or per pair (1 / d) -- at most 1.5 ulp from the exact
// quotient.  The normalisation 15 / (pi h^3) is passed in, computed once per particle.
__host__ __device__ __forceinline__ float spikyK(float h)
{
    const float h3 = h * h * h;
    return 15.0f / (3.14159265359f * h3);
}
__host__ __device__ __forceinline__ float spikyWk(float d, float h, float invH, float k)
{
    if (d >= h) return 0.0f;
    const float om = 1.0f - d * invH;
    return k * om * om;
}
__host__ __device__ __forceinline__ float spikyDWk(float d, float h, float invH, float k)
{
    if (d <= kEps || d >= h) return 0.0f;
    const float om = 1.0f - d * invH;
    return -2.0f * k * om * invH;
}
__host__ __device__ __forceinline__ f3 spikyGradK(f3 delta, float d, float h, float invH, float k)
{
    if (d <= kEps || d >= h) return f3{0.f, 0.f, 0.f};
    const float dw = spikyDWk(d, h, invH, k);
    return dw * (delta * (1.0f / d));
}
__host__ __device__ __forceinline__ float cohesionW(float d, float h, float invH, float c1, float c2)
{
    if (d <= kEps || d >= h) return 0.0f;
    const float q = d * invH;
    return c1 * q * q * q + c2 * q * q - 1.0f;
}

// physics_particle_grid.hlsli:4-10
__host__ __device__ __forceinline__ uint32_t cellKey(int gx, int gy, int gz)
{
    uint32_t seed = uint32_t(gx) * 73856093u;
    seed ^= uint32_t(gy) * 19349663u;
    seed ^= uint32_t(gz) * 83492791u;
    return seed;
}

// Slot hash for the cell table (murmur3 finaliser; the cell key itself is the reference's).
__host__ __device__ __forceinline__ uint32_t mixKey(uint32_t k)
{
    k ^= k >> 16;
    k *= 0x85ebca6bu;
    k ^= k >> 13;
    k *= 0xc2b2ae35u;
    k ^= k >> 16;
    return k;
}

} // namespace cn
