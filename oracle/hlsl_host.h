// hlsl_host.h -- TEST INFRASTRUCTURE ONLY.
//
// A small host-side model of the HLSL compute language, written for this project, so that the
// reference's own compute shaders (assets/shaders/physics/**/*.cs.hlsl of CRESSim-Neo) can be
// compiled with g++ and executed thread by thread on the CPU.  oracle/ref_build.py preprocesses
// each shader, rewrites the few constructs C++ cannot parse (attributes, semantics, cbuffer
// blocks, out/inout parameters, swizzles, float literals) and compiles it against this header
// into oracle/_ref/.  The results pin the CPU restatement in oracle/cn_oracle.cpp to the
// reference's code; nothing in the product includes this file.
//
// Arithmetic is IEEE float32 without contraction (build with -ffp-contract=off).  Choices where
// HLSL leaves the precision to the implementation follow the restatement's documented choices:
// rsqrt is the correctly rounded 1 / sqrt, length is sqrt(dot), normalize is v * rsqrt(dot).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace hlsl {

typedef uint32_t uint;
typedef uint32_t dword;

template <class T, int N> struct vec;

// A swizzle such as v.xyz or v.yz: a copy of the selected components (so it reads as, and
// converts like, the swizzle's vector type) that also writes assignments back to them.  The
// scalar constructor gives HLSL's promotion of a scalar in `c ? v.xyz : 0.0`.
template <class V, int... I> struct swz : V {
    typedef typename V::scalar S;
    S *b;
    explicit swz(S *p) : V(p[I]...), b(p) {}
    swz(S s) : V(s), b(nullptr) {}
    swz(const swz &) = default;
    swz &operator=(const V &v)
    {
        V::operator=(v);
        int k = 0;
        ((b[I] = v[k++]), ...);
        return *this;
    }
    swz &operator=(const swz &o) { return *this = static_cast<const V &>(o); }
    swz &operator+=(const V &v) { return *this = static_cast<const V &>(*this) + v; }
    swz &operator-=(const V &v) { return *this = static_cast<const V &>(*this) - v; }
    swz &operator*=(const V &v) { return *this = static_cast<const V &>(*this) * v; }
    swz &operator/=(const V &v) { return *this = static_cast<const V &>(*this) / v; }
    swz &operator*=(S s) { return *this = static_cast<const V &>(*this) * s; }
    swz &operator/=(S s) { return *this = static_cast<const V &>(*this) / s; }
};

#define HLSL_VEC_COMMON(N)                                                                              \
    typedef T scalar;                                                                                   \
    static constexpr int size = N;                                                                      \
    T &operator[](int i) { return (&x)[i]; }                                                            \
    const T &operator[](int i) const { return (&x)[i]; }                                                \
    template <class U> explicit vec(const vec<U, N> &o) { for (int i = 0; i < N; ++i) (*this)[i] = T(o[i]); } \
    friend vec operator+(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
    friend vec operator-(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
    friend vec operator*(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
    friend vec operator/(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
    friend vec operator+(const vec &a, T s) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] + s; return r; } \
    friend vec operator-(const vec &a, T s) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] - s; return r; } \
    friend vec operator*(const vec &a, T s) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] * s; return r; } \
    friend vec operator/(const vec &a, T s) { vec r; for (int i = 0; i < N; ++i) r[i] = a[i] / s; return r; } \
    friend vec operator+(T s, const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = s + a[i]; return r; } \
    friend vec operator-(T s, const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = s - a[i]; return r; } \
    friend vec operator*(T s, const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = s * a[i]; return r; } \
    friend vec operator/(T s, const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = s / a[i]; return r; } \
    friend vec operator-(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; }   \
    friend vec<bool, N> operator<(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] < b[i]; return r; } \
    friend vec<bool, N> operator<=(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] <= b[i]; return r; } \
    friend vec<bool, N> operator>(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] > b[i]; return r; } \
    friend vec<bool, N> operator>=(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] >= b[i]; return r; } \
    friend vec<bool, N> operator==(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] == b[i]; return r; } \
    friend vec<bool, N> operator!=(const vec &a, const vec &b) { vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] != b[i]; return r; } \
    vec &operator+=(const vec &o) { return *this = *this + o; }                                      \
    vec &operator-=(const vec &o) { return *this = *this - o; }                                      \
    vec &operator*=(const vec &o) { return *this = *this * o; }                                      \
    vec &operator/=(const vec &o) { return *this = *this / o; }                                      \
    vec &operator*=(T s) { return *this = *this * s; }                                               \
    vec &operator/=(T s) { return *this = *this / s; }                                               \
    friend T dot(const vec &a, const vec &b) { T r = a[0] * b[0]; for (int i = 1; i < N; ++i) r = r + a[i] * b[i]; return r; } \
    friend vec min(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = hmin(a[i], b[i]); return r; } \
    friend vec max(const vec &a, const vec &b) { vec r; for (int i = 0; i < N; ++i) r[i] = hmax(a[i], b[i]); return r; } \
    friend vec clamp(const vec &a, const vec &lo, const vec &hi) { return min(max(a, lo), hi); }     \
    friend vec abs(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = habs(a[i]); return r; } \
    friend vec floor(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = std::floor(a[i]); return r; } \
    friend vec sqrt(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = std::sqrt(a[i]); return r; } \
    friend vec saturate(const vec &a) { return min(max(a, vec(T(0))), vec(T(1))); }                   \
    friend vec sign(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = T(a[i] > T(0)) - T(a[i] < T(0)); return r; } \
    friend vec lerp(const vec &a, const vec &b, const vec &t) { return a + t * (b - a); }             \
    friend vec lerp(const vec &a, const vec &b, T t) { return a + (b - a) * t; }                      \
    friend T length(const vec &a) { return std::sqrt(dot(a, a)); }                                    \
    friend T distance(const vec &a, const vec &b) { return length(b - a); }                           \
    friend vec normalize(const vec &a) { return a * (T(1) / std::sqrt(dot(a, a))); }                 \
    friend vec rsqrt(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = T(1) / std::sqrt(a[i]); return r; } \
    friend vec rcp(const vec &a) { vec r; for (int i = 0; i < N; ++i) r[i] = T(1) / a[i]; return r; }

template <class T> inline T hmin(T a, T b) { return b < a ? b : a; }
template <class T> inline T hmax(T a, T b) { return a < b ? b : a; }
template <class T> inline T habs(T a) { return a < T(0) ? -a : a; }
inline bool habs(bool a) { return a; }
inline uint32_t habs(uint32_t a) { return a; }

template <class T> struct vec<T, 2> {
    T x, y;
    vec() = default;
    vec(T s) : x(s), y(s) {}
    vec(T a, T b) : x(a), y(b) {}
    vec(const vec<T, 3> &o) : x(o.x), y(o.y) {}   // HLSL's implicit truncation
    vec(const vec<T, 4> &o) : x(o.x), y(o.y) {}
    HLSL_VEC_COMMON(2)
    swz<vec, 1, 0> yx() { return swz<vec, 1, 0>(&x); }
    swz<vec<T, 3>, 0, 0, 0> xxx() { return swz<vec<T, 3>, 0, 0, 0>(&x); }
};

template <class T> struct vec<T, 3> {
    T x, y, z;
    vec() = default;
    vec(T s) : x(s), y(s), z(s) {}
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    vec(const vec<T, 2> &a, T c) : x(a.x), y(a.y), z(c) {}
    vec(T a, const vec<T, 2> &b) : x(a), y(b.x), z(b.y) {}
    vec(const vec<T, 4> &o) : x(o.x), y(o.y), z(o.z) {}   // HLSL's implicit truncation
    HLSL_VEC_COMMON(3)
    swz<vec, 0, 1, 2> xyz() { return swz<vec, 0, 1, 2>(&x); }
    vec xyz() const { return *this; }
    swz<vec<T, 2>, 0, 1> xy() { return swz<vec<T, 2>, 0, 1>(&x); }
    swz<vec<T, 2>, 1, 2> yz() { return swz<vec<T, 2>, 1, 2>(&x); }
    swz<vec<T, 2>, 0, 2> xz() { return swz<vec<T, 2>, 0, 2>(&x); }
    swz<vec<T, 3>, 0, 0, 0> xxx() { return swz<vec<T, 3>, 0, 0, 0>(&x); }
    swz<vec<T, 3>, 1, 1, 1> yyy() { return swz<vec<T, 3>, 1, 1, 1>(&x); }
    swz<vec<T, 3>, 2, 2, 2> zzz() { return swz<vec<T, 3>, 2, 2, 2>(&x); }
    swz<vec<T, 3>, 1, 2, 0> yzx() { return swz<vec<T, 3>, 1, 2, 0>(&x); }
    swz<vec<T, 3>, 2, 0, 1> zxy() { return swz<vec<T, 3>, 2, 0, 1>(&x); }
    friend vec cross(const vec &a, const vec &b)
    {
        return vec(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    }
};

template <class T> struct vec<T, 4> {
    T x, y, z, w;
    vec() = default;
    vec(T s) : x(s), y(s), z(s), w(s) {}
    vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    vec(const vec<T, 3> &a, T d) : x(a.x), y(a.y), z(a.z), w(d) {}
    vec(T a, const vec<T, 3> &b) : x(a), y(b.x), z(b.y), w(b.z) {}
    vec(const vec<T, 2> &a, const vec<T, 2> &b) : x(a.x), y(a.y), z(b.x), w(b.y) {}
    vec(const vec<T, 2> &a, T c, T d) : x(a.x), y(a.y), z(c), w(d) {}
    HLSL_VEC_COMMON(4)
    swz<vec<T, 3>, 0, 1, 2> xyz() { return swz<vec<T, 3>, 0, 1, 2>(&x); }
    vec<T, 3> xyz() const { return vec<T, 3>(x, y, z); }
    swz<vec<T, 2>, 0, 1> xy() { return swz<vec<T, 2>, 0, 1>(&x); }
    vec<T, 2> xy() const { return vec<T, 2>(x, y); }
    swz<vec<T, 2>, 1, 2> yz() { return swz<vec<T, 2>, 1, 2>(&x); }
    swz<vec<T, 2>, 2, 3> zw() { return swz<vec<T, 2>, 2, 3>(&x); }
    swz<vec<T, 3>, 0, 0, 0> xxx() { return swz<vec<T, 3>, 0, 0, 0>(&x); }
    swz<vec<T, 3>, 1, 2, 3> yzw() { return swz<vec<T, 3>, 1, 2, 3>(&x); }
};

#undef HLSL_VEC_COMMON

template <int N> inline bool all(const vec<bool, N> &v) { for (int i = 0; i < N; ++i) if (!v[i]) return false; return true; }
template <int N> inline bool any(const vec<bool, N> &v) { for (int i = 0; i < N; ++i) if (v[i]) return true; return false; }
inline bool all(bool v) { return v; }
inline bool any(bool v) { return v; }

typedef vec<float, 2> float2;
typedef vec<float, 3> float3;
typedef vec<float, 4> float4;
typedef vec<uint32_t, 2> uint2;
typedef vec<uint32_t, 3> uint3;
typedef vec<uint32_t, 4> uint4;
typedef vec<int32_t, 2> int2;
typedef vec<int32_t, 3> int3;
typedef vec<int32_t, 4> int4;
typedef vec<bool, 2> bool2;
typedef vec<bool, 3> bool3;
typedef vec<bool, 4> bool4;

// Scalar and vector .xxx swizzles (a splat of the first component).
inline float3 splat3(float s) { return float3(s, s, s); }
template <class T, int N> inline vec<T, 3> splat3(const vec<T, N> &v) { return vec<T, 3>(v.x, v.x, v.x); }

// Row-major 3x3 matrix (HLSL float3x3): m[r] is row r.
struct float3x3 {
    float3 r[3];
    float3x3() = default;
    float3x3(float a, float b, float c, float d, float e, float f, float g, float h, float i)
    {
        r[0] = float3(a, b, c);
        r[1] = float3(d, e, f);
        r[2] = float3(g, h, i);
    }
    float3x3(const float3 &a, const float3 &b, const float3 &c) { r[0] = a; r[1] = b; r[2] = c; }
    float3 &operator[](int i) { return r[i]; }
    const float3 &operator[](int i) const { return r[i]; }
    friend float3x3 operator+(const float3x3 &a, const float3x3 &b) { return float3x3(a.r[0] + b.r[0], a.r[1] + b.r[1], a.r[2] + b.r[2]); }
    friend float3x3 operator-(const float3x3 &a, const float3x3 &b) { return float3x3(a.r[0] - b.r[0], a.r[1] - b.r[1], a.r[2] - b.r[2]); }
    friend float3x3 operator*(const float3x3 &a, float s) { return float3x3(a.r[0] * s, a.r[1] * s, a.r[2] * s); }
    friend float3x3 operator*(float s, const float3x3 &a) { return float3x3(s * a.r[0], s * a.r[1], s * a.r[2]); }
    float3x3 &operator+=(const float3x3 &o) { return *this = *this + o; }
};
inline float3 mul(const float3x3 &m, const float3 &v) { return float3(dot(m.r[0], v), dot(m.r[1], v), dot(m.r[2], v)); }
inline float3 mul(const float3 &v, const float3x3 &m) { return m.r[0] * v.x + m.r[1] * v.y + m.r[2] * v.z; }
inline float3x3 transpose(const float3x3 &m)
{
    return float3x3(m.r[0].x, m.r[1].x, m.r[2].x, m.r[0].y, m.r[1].y, m.r[2].y, m.r[0].z, m.r[1].z, m.r[2].z);
}

// Scalar intrinsics.
inline float min(float a, float b) { return hmin(a, b); }
inline float max(float a, float b) { return hmax(a, b); }
inline uint32_t min(uint32_t a, uint32_t b) { return hmin(a, b); }
inline uint32_t max(uint32_t a, uint32_t b) { return hmax(a, b); }
inline int32_t min(int32_t a, int32_t b) { return hmin(a, b); }
inline int32_t max(int32_t a, int32_t b) { return hmax(a, b); }
inline float clamp(float v, float lo, float hi) { return min(max(v, lo), hi); }
inline uint32_t clamp(uint32_t v, uint32_t lo, uint32_t hi) { return min(max(v, lo), hi); }
inline int32_t clamp(int32_t v, int32_t lo, int32_t hi) { return min(max(v, lo), hi); }
inline float saturate(float v) { return min(max(v, 0.0f), 1.0f); }
inline float abs(float v) { return std::fabs(v); }
inline int32_t abs(int32_t v) { return v < 0 ? -v : v; }
inline float sqrt(float v) { return std::sqrt(v); }
inline float rsqrt(float v) { return 1.0f / std::sqrt(v); }
inline float rcp(float v) { return 1.0f / v; }
inline float floor(float v) { return std::floor(v); }
inline float ceil(float v) { return std::ceil(v); }
inline float round(float v) { return std::nearbyint(v); }
inline float frac(float v) { return v - std::floor(v); }
inline float sin(float v) { return std::sin(v); }
inline float cos(float v) { return std::cos(v); }
inline float tan(float v) { return std::tan(v); }
inline float acos(float v) { return std::acos(v); }
inline float asin(float v) { return std::asin(v); }
inline float atan(float v) { return std::atan(v); }
inline float atan2(float y, float x) { return std::atan2(y, x); }
inline float exp(float v) { return std::exp(v); }
inline float log(float v) { return std::log(v); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float fmod(float a, float b) { return std::fmod(a, b); }
inline float sign(float v) { return float(v > 0.0f) - float(v < 0.0f); }
inline float lerp(float a, float b, float t) { return a + t * (b - a); }
inline float step(float e, float v) { return v >= e ? 1.0f : 0.0f; }
inline float smoothstep(float a, float b, float v)
{
    const float t = saturate((v - a) / (b - a));
    return t * t * (3.0f - 2.0f * t);
}
inline bool isnan(float v) { return std::isnan(v); }
inline bool isinf(float v) { return std::isinf(v); }
inline bool isfinite(float v) { return std::isfinite(v); }
inline uint32_t asuint(float v) { uint32_t r; std::memcpy(&r, &v, 4); return r; }
inline uint32_t asuint(uint32_t v) { return v; }
inline uint32_t asuint(int32_t v) { return uint32_t(v); }
inline int32_t asint(float v) { int32_t r; std::memcpy(&r, &v, 4); return r; }
inline int32_t asint(uint32_t v) { return int32_t(v); }
inline float asfloat(uint32_t v) { float r; std::memcpy(&r, &v, 4); return r; }
inline float asfloat(int32_t v) { float r; std::memcpy(&r, &v, 4); return r; }
inline float asfloat(float v) { return v; }
template <int N> inline vec<uint32_t, N> asuint(const vec<float, N> &v) { vec<uint32_t, N> r; for (int i = 0; i < N; ++i) r[i] = asuint(v[i]); return r; }
template <int N> inline vec<float, N> asfloat(const vec<uint32_t, N> &v) { vec<float, N> r; for (int i = 0; i < N; ++i) r[i] = asfloat(v[i]); return r; }
inline uint32_t firstbithigh(uint32_t v) { return v == 0u ? 0xffffffffu : 31u - uint32_t(__builtin_clz(v)); }
inline uint32_t firstbitlow(uint32_t v) { return v == 0u ? 0xffffffffu : uint32_t(__builtin_ctz(v)); }
inline uint32_t countbits(uint32_t v) { return uint32_t(__builtin_popcount(v)); }
inline uint32_t reversebits(uint32_t v)
{
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) r |= ((v >> i) & 1u) << (31 - i);
    return r;
}

// Interlocked operations: the host executes one thread at a time, so they are plain updates.
template <class T, class U> inline void InterlockedAdd(T &d, U v) { d = T(d + T(v)); }
template <class T, class U> inline void InterlockedAdd(T &d, U v, T &orig) { orig = d; d = T(d + T(v)); }
template <class T, class U> inline void InterlockedMax(T &d, U v) { d = hmax(d, T(v)); }
template <class T, class U> inline void InterlockedMax(T &d, U v, T &orig) { orig = d; d = hmax(d, T(v)); }
template <class T, class U> inline void InterlockedMin(T &d, U v) { d = hmin(d, T(v)); }
template <class T, class U> inline void InterlockedMin(T &d, U v, T &orig) { orig = d; d = hmin(d, T(v)); }
template <class T, class U> inline void InterlockedOr(T &d, U v) { d = T(d | T(v)); }
template <class T, class U> inline void InterlockedOr(T &d, U v, T &orig) { orig = d; d = T(d | T(v)); }
template <class T, class U> inline void InterlockedAnd(T &d, U v) { d = T(d & T(v)); }
template <class T, class U> inline void InterlockedAnd(T &d, U v, T &orig) { orig = d; d = T(d & T(v)); }
template <class T, class U> inline void InterlockedExchange(T &d, U v, T &orig) { orig = d; d = T(v); }
template <class T, class U, class W> inline void InterlockedCompareExchange(T &d, U cmp, W v, T &orig)
{
    orig = d;
    if (d == T(cmp)) d = T(v);
}
template <class T, class U, class W> inline void InterlockedCompareStore(T &d, U cmp, W v)
{
    if (d == T(cmp)) d = T(v);
}

// Barriers cannot be honoured by one-thread-at-a-time execution; kernels that need them are not
// run by the host driver, and reaching one is reported.
extern int g_barrierCalls;
inline void GroupMemoryBarrierWithGroupSync() { ++g_barrierCalls; }
inline void GroupMemoryBarrier() {}
inline void DeviceMemoryBarrier() {}
inline void AllMemoryBarrier() {}
inline void DeviceMemoryBarrierWithGroupSync() { ++g_barrierCalls; }
inline void AllMemoryBarrierWithGroupSync() { ++g_barrierCalls; }

// Structured buffers bound to host memory.  Out-of-range reads return zero and out-of-range
// writes are dropped, as robust buffer access does on the GPU; each is counted.
extern uint64_t g_outOfRange;
template <class T> struct StructuredBuffer {
    T *data = nullptr;
    uint64_t count = 0;
    T &operator[](uint64_t i)
    {
        if (i < count) return data[i];
        ++g_outOfRange;
        static T dummy;
        std::memset(static_cast<void *>(&dummy), 0, sizeof(T));
        return dummy;
    }
    uint64_t elementSize() const { return sizeof(T); }
    void GetDimensions(uint32_t &n, uint32_t &stride) const { n = uint32_t(count); stride = sizeof(T); }
    void GetDimensions(uint32_t &n) const { n = uint32_t(count); }
};
template <class T> using RWStructuredBuffer = StructuredBuffer<T>;

// Raw (byte-address) buffers over 32-bit words.
struct ByteAddressBuffer {
    uint32_t *data = nullptr;
    uint64_t count = 0;   // words
    uint32_t &word(uint32_t byteOffset)
    {
        const uint64_t i = byteOffset / 4u;
        if (i < count) return data[i];
        ++g_outOfRange;
        static uint32_t dummy;
        dummy = 0;
        return dummy;
    }
    uint32_t Load(uint32_t o) { return word(o); }
    uint2 Load2(uint32_t o) { return uint2(word(o), word(o + 4u)); }
    uint3 Load3(uint32_t o) { return uint3(word(o), word(o + 4u), word(o + 8u)); }
    uint4 Load4(uint32_t o) { return uint4(word(o), word(o + 4u), word(o + 8u), word(o + 12u)); }
    void Store(uint32_t o, uint32_t v) { word(o) = v; }
    void Store2(uint32_t o, const uint2 &v) { word(o) = v.x; word(o + 4u) = v.y; }
    void Store3(uint32_t o, const uint3 &v) { word(o) = v.x; word(o + 4u) = v.y; word(o + 8u) = v.z; }
    void Store4(uint32_t o, const uint4 &v) { word(o) = v.x; word(o + 4u) = v.y; word(o + 8u) = v.z; word(o + 12u) = v.w; }
    void InterlockedAdd(uint32_t o, uint32_t v) { word(o) += v; }
    void InterlockedAdd(uint32_t o, uint32_t v, uint32_t &orig) { orig = word(o); word(o) += v; }
    void InterlockedCompareExchange(uint32_t o, uint32_t cmp, uint32_t v, uint32_t &orig)
    {
        orig = word(o);
        if (orig == cmp) word(o) = v;
    }
    void InterlockedMax(uint32_t o, uint32_t v) { word(o) = hmax(word(o), v); }
    void InterlockedMin(uint32_t o, uint32_t v) { word(o) = hmin(word(o), v); }
    void InterlockedOr(uint32_t o, uint32_t v) { word(o) |= v; }
    uint64_t elementSize() const { return 4; }
};
typedef ByteAddressBuffer RWByteAddressBuffer;

} // namespace hlsl
