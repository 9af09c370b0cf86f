// cn_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of CRESSim-Neo's particle physics substep, used as the parity
// checker for the CUDA path and as the timed CPU baseline ("port").  Nothing in
// the product links, loads or calls this file; only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg do.
//
// Each pass restates one HLSL compute kernel of the reference and cites it
// (paths are relative to the reference project root).  Passes run in the order
// PhysicsSolver::step dispatches them (src/physics/physics_solver.cpp:336-1401).
// Arithmetic is float32 with the reference's expression order; build with
// -ffp-contract=off so no multiply-add is fused.
//
// Parity status: the reference's GPU path (Vulkan/D3D12 through Diligent + DXC)
// cannot be built or run here, but its compute shaders can: oracle/ref_build.py
// compiles them for the host and oracle/ref_driver.py runs them in the solver's
// pass order.  Built with -DCN_ORACLE_QUOTIENTS (the shaders' own quotients in the
// fluid kernels) this restatement reproduces those runs bit for bit on every
// golden scene (tests/golden/ref_*.npz, tests/test_reference_pinned.py); the
// default build differs only by the reciprocal products documented below.
//
// Deliberate restatement choices (documented where they occur):
//  * rigid-BVH traversal order is replaced by "moving colliders, then static
//    colliders, each ascending by collider index"; the candidate SETS are the
//    reference's (leaf AABB = union of previous/predicted collider AABB +/- 0.05).
//  * float atomics are accumulated in contact-index order (the reference's order
//    is whatever the GPU schedules).
#include "../include/cn_physics.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr float kEps = 1.0e-6f;            // physics_base.hlsli:7
constexpr uint32_t kInvalid = 0xffffffffu; // physics_base.hlsli:6
constexpr uint32_t kRigidDedup = 16u;      // physics_particle_types.hlsli:23
constexpr uint32_t kColliderCap = 64u;     // physics_particle_types.hlsli:24
constexpr float kBroadPhaseMargin = 0.05f; // physics_shape_common.hlsli:10

struct f3 { float x, y, z; };
struct f4 { float x, y, z, w; };
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 xyz(const f4 &v) { return f3{v.x, v.y, v.z}; }
inline f4 mk4(f3 v, float w) { return f4{v.x, v.y, v.z, w}; }
inline f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
inline f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
inline f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
inline f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
inline f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
inline f3 &operator+=(f3 &a, f3 b) { a = a + b; return a; }
inline f3 &operator-=(f3 &a, f3 b) { a = a - b; return a; }
inline f4 operator+(f4 a, f4 b) { return f4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline f4 operator*(f4 a, float s) { return f4{a.x * s, a.y * s, a.z * s, a.w * s}; }
inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot4(f4 a, f4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline f3 cross(f3 a, f3 b)
{
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(f3 v) { return std::sqrt(dot(v, v)); }
inline float saturate(float v) { return std::min(std::max(v, 0.0f), 1.0f); }
inline f3 fabs3(f3 v) { return f3{std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)}; }
inline f3 clamp3(f3 v, f3 lo, f3 hi)
{
    return f3{std::min(std::max(v.x, lo.x), hi.x), std::min(std::max(v.y, lo.y), hi.y),
              std::min(std::max(v.z, lo.z), hi.z)};
}
inline f3 min3(f3 a, f3 b) { return f3{std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline f3 max3(f3 a, f3 b) { return f3{std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
inline f3 lerp3(f3 a, f3 b, float t) { return a + (b - a) * t; }

// physics_math.hlsli:6-20
inline f3 SafeNormalize(f3 v, f3 fallback)
{
    const float l2 = dot(v, v);
    if (l2 <= kEps) return fallback;
    return v * (1.0f / std::sqrt(l2));
}
inline f4 QNormalize(f4 q)
{
    const float l2 = dot4(q, q);
    if (l2 <= kEps) return f4{0, 0, 0, 1};
    return q * (1.0f / std::sqrt(l2));
}
inline f4 QConj(f4 q) { return f4{-q.x, -q.y, -q.z, q.w}; }
// physics_math.hlsli:24-31
inline f4 QMul(f4 a, f4 b)
{
    return f4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
              a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
// physics_math.hlsli:33-37
inline f3 QRotate(f4 q, f3 v)
{
    const f3 qv = xyz(q);
    const f3 t = 2.0f * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
inline f3 QInvRotate(f4 q, f3 v) { return QRotate(QConj(q), v); }
// physics_math.hlsli:71-89
inline f3 AngularVelocityFromQuaternionDelta(f4 prev, f4 cur, float dt)
{
    if (dt <= kEps) return f3{0, 0, 0};
    f4 d = QMul(QNormalize(cur), QConj(QNormalize(prev)));
    if (d.w < 0.0f) d = f4{-d.x, -d.y, -d.z, -d.w};
    const f3 im = xyz(d);
    const float l2 = dot(im, im);
    if (l2 <= kEps) return im * (2.0f / dt);
    const float l = std::sqrt(l2);
    const float angle = 2.0f * std::atan2(l, d.w);
    return im * (angle / (l * dt));
}

// physics_math.hlsli:55-73
inline f4 QuaternionFromRotationVector(f3 rv)
{
    const float a2 = dot(rv, rv);
    if (a2 <= kEps) return QNormalize(mk4(rv * 0.5f, 1.0f));
    const float angle = std::sqrt(a2);
    const float half = 0.5f * angle;
    const float sc = std::sin(half) / angle;
    return QNormalize(mk4(rv * sc, std::cos(half)));
}
inline f4 IntegrateOrientation(f4 q, f3 w, float dt) { return QNormalize(QMul(QuaternionFromRotationVector(w * dt), q)); }
inline f3 ClampLength(f3 v, float maxLen)
{
    const float l = length(v);
    if (l > maxLen && l > kEps) v = v * (maxLen / l);
    return v;
}

// physics_shape_common.hlsli:24-42
inline float SphereRadius(f4 p, f4 s)
{
    const f3 a = fabs3(xyz(s));
    return p.x * std::max(a.x, std::max(a.y, a.z));
}
inline f3 BoxHalfExtents(f4 p, f4 s) { return xyz(p) * fabs3(xyz(s)); }
inline void CapsuleSegment(f3 pos, f4 q, f4 p, f4 s, f3 &a, f3 &b, float &r)
{
    const f3 as = fabs3(xyz(s));
    r = p.x * std::max(as.x, as.z);
    const float hh = p.y * as.y;
    const f3 axis = QRotate(q, f3{0, 1, 0});
    a = pos - axis * hh;
    b = pos + axis * hh;
}
// physics_shape_common.hlsli:49-73
inline void ComputeBodyAabb(uint32_t shape, f3 pos, f4 q, f4 p, f4 s, f3 &mn, f3 &mx)
{
    f3 e{0, 0, 0};
    if (shape == CN_COLLIDER_SPHERE) {
        const float r = SphereRadius(p, s);
        e = f3{r, r, r};
    } else if (shape == CN_COLLIDER_BOX) {
        const f3 h = BoxHalfExtents(p, s);
        e = fabs3(QRotate(q, f3{1, 0, 0})) * h.x + fabs3(QRotate(q, f3{0, 1, 0})) * h.y +
            fabs3(QRotate(q, f3{0, 0, 1})) * h.z;
    } else {
        f3 a, b;
        float r = 0.0f;
        CapsuleSegment(pos, q, p, s, a, b, r);
        const f3 axis = fabs3(QRotate(q, f3{0, 1, 0}));
        e = axis * (0.5f * length(b - a)) + f3{r, r, r};
    }
    mn = pos - e;
    mx = pos + e;
}
// physics_shape_common.hlsli:75-80
inline bool AabbOverlaps(f3 minA, f3 maxA, f3 minB, f3 maxB)
{
    return minA.x <= maxB.x && maxA.x >= minB.x && minA.y <= maxB.y && maxA.y >= minB.y &&
           minA.z <= maxB.z && maxA.z >= minB.z;
}
// physics_shape_common.hlsli:97-105
inline f3 ClosestFaceNormalLocal(f3 lp, f3 h)
{
    const f3 d = h - fabs3(lp);
    if (d.x <= d.y && d.x <= d.z) return f3{lp.x >= 0.0f ? 1.0f : -1.0f, 0, 0};
    if (d.y <= d.z) return f3{0, lp.y >= 0.0f ? 1.0f : -1.0f, 0};
    return f3{0, 0, lp.z >= 0.0f ? 1.0f : -1.0f};
}

// physics_rigid_solver_shared.hlsli:8-68
inline f3 MulWorldInvInertia(f3 inv, f4 q, f3 v)
{
    const f3 ax = QRotate(q, f3{1, 0, 0});
    const f3 ay = QRotate(q, f3{0, 1, 0});
    const f3 az = QRotate(q, f3{0, 0, 1});
    return ax * (inv.x * dot(ax, v)) + ay * (inv.y * dot(ay, v)) + az * (inv.z * dot(az, v));
}
inline float ContactEffectiveMass(float invMass, f3 inv, f4 q, f3 r, f3 dir)
{
    if (invMass <= kEps) return 0.0f;
    const f3 am = MulWorldInvInertia(inv, q, cross(r, dir));
    return invMass + dot(cross(am, r), dir);
}
inline f3 CombineContactMaterial(f4 a, f4 b)
{
    const float friction = std::sqrt(std::max(0.0f, a.x) * std::max(0.0f, b.x));
    const float restitution = std::max(std::max(0.0f, a.y), std::max(0.0f, b.y));
    const float stat = std::sqrt(std::max(0.0f, a.w) * std::max(0.0f, b.w));
    return f3{friction, restitution, stat};
}
inline f3 ProjectOntoTangent(f3 v, f3 n) { return v - n * dot(v, n); }

// physics_fluid_common.hlsli:17-41.  A quotient by the smoothing radius or by a pair distance is
// taken as the product with the correctly rounded reciprocal (SPIR-V's OpFDiv, which the shaders
// compile to, is specified to 2.5 ulp rather than correctly rounded); the kernels do the same.
// Built with CN_ORACLE_QUOTIENTS the oracle keeps the shaders' quotients instead: that build is
// compared bit for bit with the reference's own kernels executed on the host (oracle/_ref).
#ifdef CN_ORACLE_QUOTIENTS
#define CN_DIV(a, b) ((a) / (b))
#else
#define CN_DIV(a, b) ((a) * (1.0f / (b)))
#endif
inline float SpikyW(float d, float h)
{
    if (d >= h) return 0.0f;
    const float om = 1.0f - CN_DIV(d, h);
    const float h3 = h * h * h;
    const float k = 15.0f / (3.14159265359f * h3);
    return k * om * om;
}
inline float SpikyDW(float d, float h)
{
    if (d <= kEps || d >= h) return 0.0f;
    const float om = 1.0f - CN_DIV(d, h);
    const float h3 = h * h * h;
    const float k = 15.0f / (3.14159265359f * h3);
    return CN_DIV(-2.0f * k * om, h);
}
inline f3 divv(f3 v, float d)
{
#ifdef CN_ORACLE_QUOTIENTS
    return v / d;
#else
    return v * (1.0f / d);
#endif
}
inline f3 SpikyGrad(f3 delta, float d, float h)
{
    if (d <= kEps || d >= h) return f3{0, 0, 0};
    const float dw = SpikyDW(d, h);
    return dw * divv(delta, d);
}
inline float CohesionW(float d, float h, float c1, float c2)
{
    if (d <= kEps || d >= h) return 0.0f;
    const float q = CN_DIV(d, h);
    return c1 * q * q * q + c2 * q * q - 1.0f;
}

// physics_particle_grid.hlsli:4-10
inline uint32_t CellKey(int gx, int gy, int gz)
{
    uint32_t seed = uint32_t(gx) * 73856093u;
    seed ^= uint32_t(gy) * 19349663u;
    seed ^= uint32_t(gz) * 83492791u;
    return seed;
}

uint32_t nextPow2(uint32_t v)
{
    if (v <= 1u) return 1u;
    --v;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1u;
}

struct Range { uint32_t start, count; };
struct Incident { uint32_t index, slot; };
struct CellRange { uint32_t key, start, end, pad; };
struct RigidContact {   // GpuParticleRigidContact, physics_particle_types.hlsli:74-83
    uint32_t particle, body, collider, active;
    f4 normalPenetration, rigidLocalPoint, material;
};
struct ParticleContact { // GpuParticleContact
    uint32_t a, b, active, pad;
    f4 normalPenetration, material;
};

template <class T> void copyArr(std::vector<T> &dst, const void *src, size_t n)
{
    dst.resize(n);
    if (n && src) std::memcpy(dst.data(), src, n * sizeof(T));
}

void buildIncidence(uint32_t n, const std::vector<std::vector<Incident>> &refs,
                    std::vector<Range> &ranges, std::vector<Incident> &flat)
{
    // physics_scene_gpu_state.cpp:3255-3420: per-particle lists in ascending constraint order.
    ranges.assign(n, Range{0, 0});
    flat.clear();
    for (uint32_t i = 0; i < n; ++i) {
        ranges[i].start = uint32_t(flat.size());
        ranges[i].count = uint32_t(refs[i].size());
        flat.insert(flat.end(), refs[i].begin(), refs[i].end());
    }
}

} // namespace

struct cno_solver {
    cn_solver_desc desc{};
    uint32_t N = 0;
    // particles
    std::vector<f4> x, xprev, v;
    std::vector<float> radii;
    std::vector<uint32_t> kinds, matIdx, fluidMatIdx, ownerTypes, ownerIdx;
    std::vector<uint32_t> meta; // uint4 per particle
    std::vector<uint32_t> adjOff, adjCnt, adjIdx;
    float cellSize = 1.0f;
    std::vector<f4> contactMaterials;
    std::vector<cn_fluid_material> fluidMaterials;
    // constraints
    std::vector<cn_soft_edge> edges;
    std::vector<cn_soft_bend> bends;
    std::vector<cn_cloth_dihedral> dihedrals;
    std::vector<cn_soft_tet> tets;
    std::vector<cn_strand_segment> segs;
    std::vector<f4> segOrient;
    std::vector<cn_strand_joint> joints;
    std::vector<cn_strand_distance> dists;
    // incidence
    std::vector<Range> edgeRanges, bendRanges, tetRanges, segRanges, segJointRanges;
    std::vector<Incident> edgeInc, bendInc, tetInc, segInc, segJointInc;
    // rigid
    uint32_t B = 0, C = 0;
    std::vector<f4> bodyPos, bodyRot, bodyLin, bodyAng, bodyScale, bodyInvInertia;
    std::vector<uint32_t> bodyType, bodyKinFlags;
    std::vector<f4> bodyKinPos, bodyKinRot;
    std::vector<uint32_t> bodyColRanges, bodyColIdx;
    std::vector<cn_collider_geometry> colGeo;
    std::vector<cn_collider_broadphase> colBp;
    std::vector<f4> colMat;
    std::vector<f4> prevBodyPos, prevBodyRot, predBodyPos, predBodyRot, predBodyLin, predBodyAng;
    std::vector<f3> colAabbMin, colAabbMax;
    // dynamic bodies: summed position / velocity corrections of a pass
    bool hasDynamic = false;
    std::vector<f3> bodyTransCorr, bodyRotCorr, bodyLinVelCorr, bodyAngVelCorr;
    // rigid-rigid contacts: candidate collider pairs, one contact each, body-pair groups
    struct RigidPairContact {
        uint32_t bodyA = 0, bodyB = 0;
        bool active = false;
        f4 normalPenetration{0, 0, 0, 0}, localA{0, 0, 0, 0}, localB{0, 0, 0, 0}, material{0, 0, 0, 0};
    };
    struct RigidSlot { f4 normal, localA, localB, state; };
    std::vector<std::pair<uint32_t, uint32_t>> rrPairs;
    std::vector<RigidPairContact> rrContacts;
    std::vector<std::vector<RigidSlot>> rrGroups;
    std::vector<std::pair<uint32_t, uint32_t>> rrGroupBodies;
    uint32_t requiredRigidRigidPairs = 0;
    // rigid proxy particles: the leading nProxy particles, carried with their bodies
    uint32_t nProxy = 0;
    std::vector<f4> proxyLocal, bodyProxyMat;
    uint32_t proxyContactSlots = 0, requiredProxyContacts = 0;
    std::vector<uint32_t> colliderQueryOrder; // moving colliders first, then static
    uint32_t activeMovingCount = 0;
    // transient state
    std::vector<int32_t> entries;     // int4 per particle (cx, cy, cz, key)
    std::vector<uint32_t> sortedKey, sortedIdx;
    std::vector<CellRange> cellRanges;
    uint32_t cellRangeCapacity = 0;
    std::vector<uint32_t> nbrCount, nbrList;
    std::vector<f4> fluidDelta, fluidNormalC, fluidDx, fluidVorticity;
    std::vector<std::vector<uint32_t>> boundaryCand; // collider indices per particle (fluids)
    std::vector<std::pair<uint32_t, uint32_t>> rigidPairs;    // (particle, body)
    std::vector<std::pair<uint32_t, uint32_t>> particlePairs; // (a, b)
    uint32_t requiredRigidPairs = 0, requiredParticlePairs = 0;
    std::vector<RigidContact> rigidContacts, activeRigidContacts;
    std::vector<ParticleContact> particleContacts, activeParticleContacts;
    std::vector<f4> posCorr, velCorr;
    std::vector<float> edgeLambda, bendLambda, tetLambda, distLambda;
    std::vector<f4> segLambda, jointLambda;
    std::vector<f4> edgeCorr;      // 2 per edge
    std::vector<f4> bendCorr;      // 4 per bend/dihedral
    std::vector<f4> tetCorr;       // 4 per tet
    std::vector<f4> segCorr;       // 3 per segment
    std::vector<f4> jointCorr;     // 5 per joint
    std::vector<f4> distCorr;      // 2 per distance
    // coloured XPBD schedules (desc.soft.xpbd_schedule != 0): per family (edges, strand
    // segments, bends + dihedrals, strand joints, strand distances, tets) the constraints grouped
    // by colour, the colour boundaries, and the colour-Jacobi sums
    std::vector<uint32_t> colOrder[6], colStarts[6];
    std::vector<f4> softAcc, orientAcc;
    uint32_t truncations = 0;
    bool postUpdateNeighbors = true; // physics_solver.cpp:1262-1268
    // surface render data (SurfaceDeformableRenderDataHost) and outputs
    std::vector<cn_surface_vertex_binding> surfBind;
    std::vector<f4> surfFallback;
    std::vector<cn_surface_triangle_range> surfRanges;
    std::vector<uint32_t> surfIdx;
    std::vector<uint32_t> surfTri;            // uint4 per triangle
    std::vector<uint32_t> surfChunks;         // uint4 per chunk (surface, start, count, 0)
    std::vector<uint32_t> surfChunkRanges;    // uint2 per surface (start, count)
    std::vector<f4> surfPos, surfNrm, surfTriN, surfChunkAabb, surfWorldAabb;

    // settings shorthands (physics_solver_config.hlsli:27-62)
    float slop() const { return desc.contact.slop; }
};

namespace {

void setupWorld(cno_solver &s, const cn_world_soa &w)
{
    s.N = w.particle_count;
    const uint32_t N = s.N;
    copyArr(s.x, w.positions_inv_mass, N);
    copyArr(s.v, w.velocities, N);
    s.xprev.assign(N, f4{0, 0, 0, 0});
    for (uint32_t i = 0; i < N; ++i) s.xprev[i] = mk4(xyz(s.x[i]), 0.0f);
    copyArr(s.radii, w.radii, N);
    copyArr(s.kinds, w.kinds, N);
    copyArr(s.meta, w.metadata, size_t(N) * 4);
    copyArr(s.matIdx, w.material_indices, N);
    copyArr(s.fluidMatIdx, w.fluid_material_indices, N);
    copyArr(s.ownerTypes, w.owner_types, N);
    copyArr(s.ownerIdx, w.owner_indices, N);
    s.nProxy = 0;
    while (s.nProxy < N && s.ownerTypes[s.nProxy] == CN_OWNER_RIGID_BODY) ++s.nProxy;
    if (s.nProxy) {
        copyArr(s.proxyLocal, w.rigid_proxy_local_positions, s.nProxy);
        copyArr(s.bodyProxyMat, w.body_proxy_contact_materials, w.rigid_body_count);
    }
    copyArr(s.adjOff, w.adjacency_offsets, N);
    copyArr(s.adjCnt, w.adjacency_counts, N);
    copyArr(s.adjIdx, w.adjacency_indices, w.adjacency_index_count);
    s.cellSize = w.particle_grid_cell_size;
    copyArr(s.contactMaterials, w.contact_materials, w.contact_material_count);
    copyArr(s.fluidMaterials, w.fluid_materials, w.fluid_material_count);
    copyArr(s.edges, w.edges, w.edge_count);
    copyArr(s.bends, w.bends, w.bend_count);
    copyArr(s.dihedrals, w.dihedrals, w.dihedral_count);
    copyArr(s.tets, w.tets, w.tet_count);
    copyArr(s.segs, w.strand_segments, w.strand_segment_count);
    copyArr(s.segOrient, w.strand_segment_orientations, w.strand_segment_count);
    copyArr(s.joints, w.strand_joints, w.strand_joint_count);
    copyArr(s.dists, w.strand_distances, w.strand_distance_count);
    s.B = w.rigid_body_count;
    s.C = w.collider_count;
    copyArr(s.bodyPos, w.body_positions_inv_mass, s.B);
    copyArr(s.bodyRot, w.body_orientations, s.B);
    copyArr(s.bodyLin, w.body_linear_velocities, s.B);
    copyArr(s.bodyAng, w.body_angular_velocities, s.B);
    copyArr(s.bodyScale, w.body_scales, s.B);
    copyArr(s.bodyInvInertia, w.body_inverse_inertia, s.B);
    copyArr(s.bodyType, w.body_types, s.B);
    copyArr(s.bodyKinPos, w.body_kinematic_target_positions, s.B);
    copyArr(s.bodyKinRot, w.body_kinematic_target_orientations, s.B);
    copyArr(s.bodyKinFlags, w.body_kinematic_target_flags, s.B);
    copyArr(s.bodyColRanges, w.body_collider_ranges, size_t(s.B) * 2);
    copyArr(s.bodyColIdx, w.body_collider_indices, w.body_collider_index_count);
    copyArr(s.colGeo, w.collider_geometry, s.C);
    copyArr(s.colBp, w.collider_broadphase, s.C);
    copyArr(s.colMat, w.collider_materials, s.C);

    // Incidence tables (physics_scene_gpu_state.cpp:3273-3420).
    std::vector<std::vector<Incident>> refs(N);
    for (uint32_t e = 0; e < s.edges.size(); ++e) {
        if (s.edges[e].particle_a < N) refs[s.edges[e].particle_a].push_back({e, 0});
        if (s.edges[e].particle_b < N) refs[s.edges[e].particle_b].push_back({e, 1});
    }
    buildIncidence(N, refs, s.edgeRanges, s.edgeInc);
    refs.assign(N, {});
    for (uint32_t b = 0; b < s.bends.size(); ++b) {
        const uint32_t p[3] = {s.bends[b].particle0, s.bends[b].particle1, s.bends[b].particle2};
        for (uint32_t k = 0; k < 3; ++k)
            if (p[k] < N) refs[p[k]].push_back({b, k});
    }
    const uint32_t off = uint32_t(s.bends.size());
    for (uint32_t d = 0; d < s.dihedrals.size(); ++d) {
        const cn_cloth_dihedral &h = s.dihedrals[d];
        const uint32_t p[4] = {h.edge_particle0, h.edge_particle1, h.opposite_particle0,
                               h.opposite_particle1};
        for (uint32_t k = 0; k < 4; ++k)
            if (p[k] < N) refs[p[k]].push_back({off + d, k});
    }
    buildIncidence(N, refs, s.bendRanges, s.bendInc);
    refs.assign(N, {});
    for (uint32_t t = 0; t < s.tets.size(); ++t)
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t p = s.tets[t].particle_indices[k];
            if (p < N) refs[p].push_back({t, k});
        }
    buildIncidence(N, refs, s.tetRanges, s.tetInc);
    refs.assign(N, {});
    for (uint32_t g = 0; g < s.segs.size(); ++g) {
        if (s.segs[g].particle_a < N) refs[s.segs[g].particle_a].push_back({g, 0});
        if (s.segs[g].particle_b < N) refs[s.segs[g].particle_b].push_back({g, 1});
    }
    buildIncidence(N, refs, s.segRanges, s.segInc);
    std::vector<std::vector<Incident>> srefs(s.segs.size());
    for (uint32_t j = 0; j < s.joints.size(); ++j) {
        if (s.joints[j].segment_a >= s.segs.size() || s.joints[j].segment_b >= s.segs.size())
            continue;
        srefs[s.joints[j].segment_a].push_back({j, 0});
        srefs[s.joints[j].segment_b].push_back({j, 1});
    }
    buildIncidence(uint32_t(s.segs.size()), srefs, s.segJointRanges, s.segJointInc);

    // Transient buffers start zeroed (fresh allocations).
    s.entries.assign(size_t(N) * 4, 0);
    s.sortedKey.assign(N, 0);
    s.sortedIdx.assign(N, 0);
    s.cellRangeCapacity = nextPow2(std::max<uint32_t>(N * 2u, 1u));
    s.cellRanges.assign(s.cellRangeCapacity, CellRange{kInvalid, 0, 0, 0});
    s.nbrCount.assign(N, 0);
    s.nbrList.assign(size_t(N) * s.desc.max_fluid_neighborhood, 0);
    s.fluidDelta.assign(N, f4{0, 0, 0, 0});
    s.fluidNormalC.assign(N, f4{0, 0, 0, 0});
    s.fluidDx.assign(N, f4{0, 0, 0, 0});
    s.boundaryCand.assign(N, {});
    s.posCorr.assign(N, f4{0, 0, 0, 0});
    s.velCorr.assign(N, f4{0, 0, 0, 0});
    s.edgeLambda.assign(s.edges.size(), 0.0f);
    s.bendLambda.assign(s.bends.size() + s.dihedrals.size(), 0.0f);
    s.tetLambda.assign(s.tets.size(), 0.0f);
    s.distLambda.assign(s.dists.size(), 0.0f);
    s.segLambda.assign(s.segs.size(), f4{0, 0, 0, 0});
    s.jointLambda.assign(s.joints.size(), f4{0, 0, 0, 0});
    s.edgeCorr.assign(s.edges.size() * 2, f4{0, 0, 0, 0});
    s.bendCorr.assign((s.bends.size() + s.dihedrals.size()) * 4, f4{0, 0, 0, 0});
    s.tetCorr.assign(s.tets.size() * 4, f4{0, 0, 0, 0});
    s.segCorr.assign(s.segs.size() * 3, f4{0, 0, 0, 0});
    s.jointCorr.assign(s.joints.size() * 5, f4{0, 0, 0, 0});
    s.distCorr.assign(s.dists.size() * 2, f4{0, 0, 0, 0});
    s.prevBodyPos = s.bodyPos; s.prevBodyRot = s.bodyRot;
    s.predBodyPos = s.bodyPos; s.predBodyRot = s.bodyRot;
    s.predBodyLin = s.bodyLin; s.predBodyAng = s.bodyAng;
    s.colAabbMin.assign(s.C, f3{0, 0, 0});
    s.colAabbMax.assign(s.C, f3{0, 0, 0});
    for (uint32_t b = 0; b < s.B; ++b) s.hasDynamic = s.hasDynamic || s.bodyType[b] == CN_BODY_DYNAMIC;
    s.bodyTransCorr.assign(s.B, f3{0, 0, 0}); s.bodyRotCorr.assign(s.B, f3{0, 0, 0});
    s.bodyLinVelCorr.assign(s.B, f3{0, 0, 0}); s.bodyAngVelCorr.assign(s.B, f3{0, 0, 0});
    if (const cn_surface_render_data *sr = w.surface_render) {
        const uint32_t V = sr->vertex_count, T = sr->triangle_count, S = sr->surface_count;
        s.surfBind.assign(sr->vertex_bindings, sr->vertex_bindings + V);
        s.surfFallback.resize(V);
        for (uint32_t v = 0; v < V; ++v)
            s.surfFallback[v] = f4{sr->fallback_normals[4 * v], sr->fallback_normals[4 * v + 1],
                                   sr->fallback_normals[4 * v + 2], sr->fallback_normals[4 * v + 3]};
        s.surfRanges.assign(sr->vertex_triangle_ranges, sr->vertex_triangle_ranges + V);
        s.surfIdx.assign(sr->vertex_triangle_indices, sr->vertex_triangle_indices + sr->vertex_triangle_index_count);
        s.surfTri.assign(sr->triangle_particle_indices, sr->triangle_particle_indices + size_t(T) * 4);
        // 64-particle bounds chunks per surface (physics_scene_gpu_state.cpp:3482-3500)
        for (uint32_t k = 0; k < S; ++k) {
            const uint32_t off = sr->surface_particle_ranges[2 * k], cnt = sr->surface_particle_ranges[2 * k + 1];
            s.surfChunkRanges.push_back(uint32_t(s.surfChunks.size() / 4));
            uint32_t n = 0;
            for (uint32_t o = 0; o < cnt; o += 64u, ++n)
                s.surfChunks.insert(s.surfChunks.end(), {k, off + o, std::min(64u, cnt - o), 0u});
            s.surfChunkRanges.push_back(n);
        }
        s.surfPos.assign(V, f4{0, 0, 0, 0});
        s.surfNrm.assign(V, f4{0, 0, 0, 0});
        s.surfTriN.assign(T, f4{0, 0, 0, 0});
        s.surfChunkAabb.assign(s.surfChunks.size() / 4 * 2, f4{0, 0, 0, 0});
        s.surfWorldAabb.assign(size_t(S) * 2, f4{0, 0, 0, 0});
    }
}

// ---------------------------------------------------------------------------
// Surface render passes (PhysicsSolver::step, physics_solver.cpp:1310-1337).
// ---------------------------------------------------------------------------
// physics_surface_skin_render_vertices.cs.hlsl:14-36
void skinSurfaceVertices(cno_solver &s)
{
    for (size_t v = 0; v < s.surfBind.size(); ++v) {
        const cn_surface_vertex_binding &b = s.surfBind[v];
        f3 acc{0.f, 0.f, 0.f};
        for (int k = 0; k < 4; ++k) acc += b.weights[k] * xyz(s.x[b.particle_indices[k]]);
        s.surfPos[v] = mk4(acc, 1.0f);
    }
}

// physics_surface_update_triangle_normals.cs.hlsl:8-24
void updateSurfaceTriangleNormals(cno_solver &s)
{
    for (size_t t = 0; t < s.surfTriN.size(); ++t) {
        const f3 p0 = xyz(s.x[s.surfTri[4 * t]]), p1 = xyz(s.x[s.surfTri[4 * t + 1]]), p2 = xyz(s.x[s.surfTri[4 * t + 2]]);
        s.surfTriN[t] = mk4(cross(p2 - p0, p1 - p0), 0.0f);
    }
}

// physics_surface_update_render_normals.cs.hlsl:18-48; rsqrt taken as the correctly rounded
// 1 / sqrt (the shader's is a hardware approximation)
void updateSurfaceVertexNormals(cno_solver &s)
{
    for (size_t v = 0; v < s.surfRanges.size(); ++v) {
        const cn_surface_triangle_range &r = s.surfRanges[v];
        f3 acc{0.f, 0.f, 0.f};
        for (uint32_t k = 0; k < r.count; ++k) acc += xyz(s.surfTriN[s.surfIdx[r.start + k]]);
        f3 n = acc;
        const float lenSq = dot(n, n);
        if (lenSq <= 1.0e-12f) n = xyz(s.surfFallback[v]);
        else n = n * (1.0f / std::sqrt(lenSq));
        s.surfNrm[v] = mk4(n, 0.0f);
    }
}

// physics_surface_update_bounds.cs.hlsl:12-65 and physics_surface_finalize_bounds.cs.hlsl:12-66
void updateSurfaceBounds(cno_solver &s)
{
    const float big = 3.402823e+38f;
    const size_t chunks = s.surfChunks.size() / 4;
    for (size_t c = 0; c < chunks; ++c) {
        const uint32_t start = s.surfChunks[4 * c + 1], count = s.surfChunks[4 * c + 2];
        if (count == 0u) {
            s.surfChunkAabb[2 * c] = s.surfChunkAabb[2 * c + 1] = f4{0, 0, 0, 0};
            continue;
        }
        f3 lo{big, big, big}, hi{-big, -big, -big};
        for (uint32_t k = 0; k < count; ++k) {
            lo = min3(lo, xyz(s.x[start + k]));
            hi = max3(hi, xyz(s.x[start + k]));
        }
        s.surfChunkAabb[2 * c] = mk4(lo, 0.0f);
        s.surfChunkAabb[2 * c + 1] = mk4(hi, 0.0f);
    }
    const size_t S = s.surfChunkRanges.size() / 2;
    for (size_t k = 0; k < S; ++k) {
        const uint32_t start = s.surfChunkRanges[2 * k], count = s.surfChunkRanges[2 * k + 1];
        if (count == 0u) {
            s.surfWorldAabb[2 * k] = s.surfWorldAabb[2 * k + 1] = f4{0, 0, 0, 0};
            continue;
        }
        f3 lo{big, big, big}, hi{-big, -big, -big};
        for (uint32_t c = 0; c < count; ++c) {
            lo = min3(lo, xyz(s.surfChunkAabb[2 * (start + c)]));
            hi = max3(hi, xyz(s.surfChunkAabb[2 * (start + c) + 1]));
        }
        s.surfWorldAabb[2 * k] = mk4(lo, 0.0f);
        s.surfWorldAabb[2 * k + 1] = mk4(hi, 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Rigid predict (static / kinematic branches): physics_rigid_predict.cs.hlsl:20-81,
// then the collider world AABBs: physics_rigid_update_world_aabbs.cs.hlsl:23-100.
// ---------------------------------------------------------------------------
void predictRigid(cno_solver &s, float dt)
{
    const f3 g{s.desc.gravity[0], s.desc.gravity[1], s.desc.gravity[2]};
    for (uint32_t b = 0; b < s.B; ++b) {
        const f4 p = s.bodyPos[b];
        const f4 q = QNormalize(s.bodyRot[b]);
        f4 lin = s.bodyLin[b], ang = s.bodyAng[b];
        const bool kinEnabled = (s.bodyKinFlags[b] & 1u) != 0u;
        const f4 kq = QNormalize(s.bodyKinRot[b]);
        s.prevBodyPos[b] = p;
        s.prevBodyRot[b] = q;
        if (s.bodyType[b] == CN_BODY_STATIC) {
            s.predBodyPos[b] = p; s.predBodyRot[b] = q;
            s.predBodyLin[b] = f4{0, 0, 0, 0}; s.predBodyAng[b] = f4{0, 0, 0, 0};
            continue;
        }
        if (s.bodyType[b] == CN_BODY_KINEMATIC) {
            const f3 pp = kinEnabled ? xyz(s.bodyKinPos[b]) : xyz(p);
            const f4 pq = kinEnabled ? kq : q;
            const f3 l = (pp - xyz(p)) / std::max(dt, kEps);
            const f3 a = AngularVelocityFromQuaternionDelta(q, pq, std::max(dt, kEps));
            s.predBodyPos[b] = mk4(pp, p.w); s.predBodyRot[b] = pq;
            s.predBodyLin[b] = mk4(l, lin.w); s.predBodyAng[b] = mk4(a, ang.w);
            continue;
        }
        f3 l = xyz(lin) + g * dt;
        s.predBodyPos[b] = mk4(xyz(p) + l * dt, p.w);
        s.predBodyRot[b] = IntegrateOrientation(q, xyz(ang), dt);
        s.predBodyLin[b] = mk4(l, lin.w);
        s.predBodyAng[b] = ang;
    }
    s.activeMovingCount = 0;
    std::vector<uint32_t> moving, stat;
    for (uint32_t c = 0; c < s.C; ++c) {
        const cn_collider_broadphase &bp = s.colBp[c];
        const uint32_t ob = bp.owner_body;
        if (ob >= s.B || bp.enabled_flag == 0u) {
            s.colAabbMin[c] = f3{0, 0, 0}; s.colAabbMax[c] = f3{0, 0, 0};
            continue;
        }
        const f4 sc = s.bodyScale[ob];
        const cn_collider_geometry &cg = s.colGeo[c];
        const f4 params{cg.shape_params[0], cg.shape_params[1], cg.shape_params[2], cg.shape_params[3]};
        const f3 lp = f3{cg.local_position[0], cg.local_position[1], cg.local_position[2]} * xyz(sc);
        const f4 lq = QNormalize(f4{cg.local_orientation[0], cg.local_orientation[1],
                                    cg.local_orientation[2], cg.local_orientation[3]});
        const f4 bq = QNormalize(s.predBodyRot[ob]);
        const f4 pbq = QNormalize(s.prevBodyRot[ob]);
        const f3 cp = xyz(s.predBodyPos[ob]) + QRotate(bq, lp);
        const f4 cq = QNormalize(QMul(bq, lq));
        const f3 pcp = xyz(s.prevBodyPos[ob]) + QRotate(pbq, lp);
        const f4 pcq = QNormalize(QMul(pbq, lq));
        f3 mn, mx, pmn, pmx;
        ComputeBodyAabb(bp.shape_type, cp, cq, params, sc, mn, mx);
        ComputeBodyAabb(bp.shape_type, pcp, pcq, params, sc, pmn, pmx);
        mn = min3(mn, pmn);
        mx = max3(mx, pmx);
        s.colAabbMin[c] = mn - f3{kBroadPhaseMargin, kBroadPhaseMargin, kBroadPhaseMargin};
        s.colAabbMax[c] = mx + f3{kBroadPhaseMargin, kBroadPhaseMargin, kBroadPhaseMargin};
        if (s.bodyType[ob] == CN_BODY_STATIC) stat.push_back(c);
        else moving.push_back(c);
    }
    s.activeMovingCount = uint32_t(moving.size());
    s.colliderQueryOrder = moving;
    s.colliderQueryOrder.insert(s.colliderQueryOrder.end(), stat.begin(), stat.end());
}

// physics_soft_predict.cs.hlsl:12-47
void predictSoft(cno_solver &s, float dt)
{
    const f3 g{s.desc.gravity[0], s.desc.gravity[1], s.desc.gravity[2]};
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f4 pim = s.x[i];
        s.xprev[i] = mk4(xyz(pim), 0.0f);
        if (pim.w <= kEps) {
            s.v[i] = f4{0, 0, 0, 0};
            continue;
        }
        f3 vel = xyz(s.v[i]);
        float gs = 1.0f;
        if (s.kinds[i] == CN_PARTICLE_FLUID) gs = s.fluidMaterials[s.fluidMatIdx[i]].gravity_scale;
        vel = vel + g * (dt * gs);
        const f3 pp = xyz(pim) + vel * dt;
        s.v[i] = mk4(vel, 0.0f);
        s.x[i] = mk4(pp, pim.w);
    }
}

// physics_particle_sync_rigid_proxy_particles.cs.hlsl:13-39: a proxy particle at its body's
// predicted pose (the inverse mass kept)
void syncRigidProxies(cno_solver &s)
{
    for (uint32_t i = 0; i < s.nProxy; ++i) {
        const uint32_t b = s.ownerIdx[i];
        const f4 q = QNormalize(s.predBodyRot[b]);
        s.x[i] = mk4(xyz(s.predBodyPos[b]) + QRotate(q, xyz(s.proxyLocal[i])), s.x[i].w);
    }
}

// physics_particle_build_broad_phase_entries.cs.hlsl:9-35 + _keys.cs.hlsl:8-23 +
// the stable 32-pass split radix sort (physics_pass_dispatcher.cpp:3963-4057) +
// cell ranges (mark_cell_range_starts / clear_cell_ranges / build_cell_ranges).
void broadphase(cno_solver &s)
{
    const uint32_t N = s.N;
    const float safe = std::max(s.cellSize, 1.0e-4f);
    const float inv = 1.0f / safe;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f3 p = xyz(s.x[i]);
        const int gx = int(std::floor(p.x * inv));
        const int gy = int(std::floor(p.y * inv));
        const int gz = int(std::floor(p.z * inv));
        s.entries[4 * i + 0] = gx;
        s.entries[4 * i + 1] = gy;
        s.entries[4 * i + 2] = gz;
        s.entries[4 * i + 3] = int32_t(CellKey(gx, gy, gz));
    }
    std::vector<uint64_t> kv(N);
    for (uint32_t i = 0; i < N; ++i) kv[i] = (uint64_t(uint32_t(s.entries[4 * i + 3])) << 32) | i;
    // Sorting (key, index) lexicographically is the permutation of a stable sort by key.
    std::sort(kv.begin(), kv.end());
    for (uint32_t i = 0; i < N; ++i) {
        s.sortedKey[i] = uint32_t(kv[i] >> 32);
        s.sortedIdx[i] = uint32_t(kv[i] & 0xffffffffu);
    }
    s.cellRangeCapacity = nextPow2(std::max<uint32_t>(N * 2u, 1u));
    s.cellRanges.assign(s.cellRangeCapacity, CellRange{kInvalid, 0, 0, 0});
    uint32_t rangeIndex = 0;
    for (uint32_t i = 0; i < N; ++i) {
        if (i != 0 && s.sortedKey[i - 1] == s.sortedKey[i]) continue;
        uint32_t end = i + 1;
        while (end < N && s.sortedKey[end] == s.sortedKey[i]) ++end;
        if (rangeIndex < s.cellRangeCapacity)
            s.cellRanges[rangeIndex] = CellRange{s.sortedKey[i], i, end, 0};
        ++rangeIndex;
    }
}

// physics_fluid_neighbor_build.hlsli:6-46 (identical to FindCellRange in
// physics_particle_broad_phase_query.hlsli:8-48)
inline CellRange FindCellRange(const cno_solver &s, uint32_t key)
{
    const CellRange missing{kInvalid, 0, 0, 0};
    if (s.cellRangeCapacity == 0) return missing;
    uint32_t lo = 0, hi = s.cellRangeCapacity;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        if (s.cellRanges[mid].key < key) lo = mid + 1u;
        else hi = mid;
    }
    if (lo < s.cellRangeCapacity && s.cellRanges[lo].key == key) return s.cellRanges[lo];
    return missing;
}

// physics_particle_broad_phase_query.hlsli:50-117
bool IsAdjacent(const cno_solver &s, uint32_t p, uint32_t c)
{
    const uint32_t o = s.adjOff[p], n = s.adjCnt[p];
    for (uint32_t i = 0; i < n; ++i)
        if (s.adjIdx[o + i] == c) return true;
    return false;
}
bool ValidParticleParticleCandidate(const cno_solver &s, uint32_t p, f3 pos, float r, uint32_t kind,
                                    uint32_t env, uint32_t phase, uint32_t layer, uint32_t mask,
                                    uint32_t other)
{
    if (other <= p) return false;
    const uint32_t *om = &s.meta[4 * other];
    if (om[0] != env) return false;
    if ((mask & om[2]) == 0u || (om[3] & layer) == 0u) return false;
    const uint32_t ok = s.kinds[other];
    if (kind == CN_PARTICLE_FLUID && ok == CN_PARTICLE_FLUID) return false;
    if (kind == CN_PARTICLE_SOLID && ok == CN_PARTICLE_SOLID &&
        (phase & CN_PHASE_GROUP_MASK) == (om[1] & CN_PHASE_GROUP_MASK)) {
        const bool a = (phase & CN_PHASE_SELF_COLLIDE) != 0u;
        const bool b = (om[1] & CN_PHASE_SELF_COLLIDE) != 0u;
        if (!a || !b || IsAdjacent(s, p, other)) return false;
    }
    const f3 op = xyz(s.x[other]);
    const float cr = r + s.radii[other];
    const f3 d = op - pos;
    return dot(d, d) <= cr * cr;
}

// count/finalize/emit_particle_particle_candidates.cs.hlsl
void buildParticleParticleCandidates(cno_solver &s)
{
    const uint32_t N = s.N;
    std::vector<std::vector<uint32_t>> per(N);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ii = 0; ii < int64_t(N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const int32_t *e = &s.entries[4 * i];
        const f3 pos = xyz(s.x[i]);
        const float r = s.radii[i];
        const uint32_t *m = &s.meta[4 * i];
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const CellRange rg = FindCellRange(s, CellKey(e[0] + dx, e[1] + dy, e[2] + dz));
                    if (rg.key == kInvalid) continue;
                    for (uint32_t si = rg.start; si < rg.end; ++si) {
                        const uint32_t c = s.sortedIdx[si];
                        const int32_t *ce = &s.entries[4 * c];
                        if (ce[0] != e[0] + dx || ce[1] != e[1] + dy || ce[2] != e[2] + dz) continue;
                        if (ValidParticleParticleCandidate(s, i, pos, r, s.kinds[i], m[0], m[1], m[2],
                                                           m[3], c))
                            per[i].push_back(c);
                    }
                }
    }
    const uint32_t cap = std::max<uint32_t>(N * 8u, 64u);
    s.particlePairs.clear();
    uint64_t required = 0;
    for (uint32_t i = 0; i < N; ++i) {
        for (uint32_t c : per[i]) {
            if (required < cap) s.particlePairs.push_back({i, c});
            ++required;
        }
    }
    s.requiredParticlePairs = uint32_t(required);
}

// count/finalize/emit_particle_rigid_candidates.cs.hlsl:113-151 (BVH replaced by the
// collider query order; TryAppendRigidBody dedup cache of 16 bodies kept).
void buildParticleRigidCandidates(cno_solver &s)
{
    const uint32_t N = s.N;
    std::vector<std::vector<uint32_t>> per(N);
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f3 p = xyz(s.x[i]);
        const float r = s.radii[i];
        const f3 qmin = p - f3{r, r, r}, qmax = p + f3{r, r, r};
        const uint32_t *m = &s.meta[4 * i];
        const bool proxyOwner = s.ownerTypes[i] == CN_OWNER_RIGID_BODY;
        uint32_t seen[kRigidDedup];
        uint32_t seenCount = 0;
        for (uint32_t k = 0; k < s.colliderQueryOrder.size(); ++k) {
            const uint32_t c = s.colliderQueryOrder[k];
            const bool isMoving = k < s.activeMovingCount;
            if (isMoving && s.activeMovingCount == 0) continue;
            if (!AabbOverlaps(qmin, qmax, s.colAabbMin[c], s.colAabbMax[c])) continue;
            const cn_collider_broadphase &bp = s.colBp[c];
            const uint32_t b = bp.owner_body;
            if (proxyOwner && b == s.ownerIdx[i]) continue;
            const uint32_t bt = s.bodyType[b];
            if (!(bp.enabled_flag != 0u && bp.environment_index == m[0] &&
                  (m[3] & bp.collision_layer) != 0u && (bp.collision_mask & m[2]) != 0u &&
                  (s.kinds[i] == CN_PARTICLE_SOLID || bt == CN_BODY_DYNAMIC) &&
                  s.bodyColRanges[2 * b + 1] > 0u))
                continue;
            bool fresh = true;
            for (uint32_t q = 0; q < seenCount; ++q)
                if (seen[q] == b) { fresh = false; break; }
            if (!fresh) continue;
            if (seenCount < kRigidDedup) seen[seenCount++] = b;
            per[i].push_back(b);
        }
    }
    // max(particles x 8, 64) (physics_scene_gpu_state.cpp:726-727); the rate is a setting here
    const uint32_t rate = s.desc.particle_rigid_pairs_per_particle ? s.desc.particle_rigid_pairs_per_particle : 8u;
    const uint32_t cap = std::max<uint32_t>(N * rate, 64u);
    s.rigidPairs.clear();
    uint64_t required = 0;
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t b : per[i]) {
            if (required < cap) s.rigidPairs.push_back({i, b});
            ++required;
        }
    s.requiredRigidPairs = uint32_t(required);
}

// count/emit_fluid_boundary_candidates.cs.hlsl (per-particle candidate lists)
void buildFluidBoundaryCandidates(cno_solver &s)
{
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        s.boundaryCand[i].clear();
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const f3 p = xyz(s.x[i]);
        const float pr = std::max(s.radii[i], 0.0f);
        const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[i]];
        const float support = std::max(fm.smoothing_radius, pr);
        const float reuse = std::max(std::max(fm.cfl_radius, pr), support);
        const float qr = support + reuse;
        const f3 qmin = p - f3{qr, qr, qr}, qmax = p + f3{qr, qr, qr};
        const uint32_t *m = &s.meta[4 * i];
        for (uint32_t k = 0; k < s.colliderQueryOrder.size(); ++k) {
            const uint32_t c = s.colliderQueryOrder[k];
            if (!AabbOverlaps(qmin, qmax, s.colAabbMin[c], s.colAabbMax[c])) continue;
            const cn_collider_broadphase &bp = s.colBp[c];
            const uint32_t bt = s.bodyType[bp.owner_body];
            if (bp.enabled_flag != 0u && bp.environment_index == m[0] && bt != CN_BODY_DYNAMIC &&
                (m[3] & bp.collision_layer) != 0u && (bp.collision_mask & m[2]) != 0u)
                s.boundaryCand[i].push_back(c);
        }
    }
}

// physics_fluid_boundary_common.hlsli:11-83
bool FluidBoundaryContactInfo(const cno_solver &s, uint32_t c, f3 pos, float &sd, f3 &n)
{
    sd = 0.0f;
    n = f3{0, 1, 0};
    const cn_collider_broadphase &bp = s.colBp[c];
    if (bp.enabled_flag == 0u) return false;
    const uint32_t b = bp.owner_body;
    const f3 bpos = xyz(s.predBodyPos[b]);
    const f4 bq = QNormalize(s.predBodyRot[b]);
    const f4 sc = s.bodyScale[b];
    const cn_collider_geometry &cg = s.colGeo[c];
    const f3 cwp = bpos + QRotate(bq, f3{cg.local_position[0], cg.local_position[1], cg.local_position[2]});
    const f4 cwq = QNormalize(QMul(bq, QNormalize(f4{cg.local_orientation[0], cg.local_orientation[1],
                                                      cg.local_orientation[2], cg.local_orientation[3]})));
    const f4 sp{cg.shape_params[0], cg.shape_params[1], cg.shape_params[2], cg.shape_params[3]};
    if (bp.shape_type == CN_COLLIDER_SPHERE) {
        const f3 d = pos - cwp;
        const float dist = length(d);
        const float r = SphereRadius(sp, sc);
        n = dist > kEps ? (d / dist) : f3{0, 1, 0};
        sd = dist - r;
    } else if (bp.shape_type == CN_COLLIDER_BOX) {
        const f3 he = BoxHalfExtents(sp, sc);
        const f3 lp = QInvRotate(cwq, pos - cwp);
        const f3 cl = clamp3(lp, -he, he);
        const f3 d = lp - cl;
        const float dl = length(d);
        if (dl > kEps) {
            n = QRotate(cwq, d / dl);
            sd = dl;
        } else {
            const f3 ds = he - fabs3(lp);
            n = QRotate(cwq, ClosestFaceNormalLocal(lp, he));
            sd = -std::min(ds.x, std::min(ds.y, ds.z));
        }
    } else {
        f3 a, b2;
        float cr = 0.0f;
        CapsuleSegment(cwp, cwq, sp, sc, a, b2, cr);
        const f3 seg = b2 - a;
        const float l2 = dot(seg, seg);
        float t = 0.0f;
        if (l2 > kEps) t = saturate(dot(pos - a, seg) / l2);
        const f3 cl = lerp3(a, b2, t);
        const f3 d = pos - cl;
        const float dist = length(d);
        n = dist > kEps ? (d / dist) : f3{0, 1, 0};
        sd = dist - cr;
    }
    return true;
}
bool FluidGhostDelta(const cno_solver &s, uint32_t c, f3 pos, float h, f3 &ghost)
{
    ghost = f3{0, 0, 0};
    float sd = 0.0f;
    f3 n{0, 1, 0};
    if (!FluidBoundaryContactInfo(s, c, pos, sd, n)) return false;
    if (sd < 0.0f || sd >= h) return false;
    ghost = n * (2.0f * sd);
    return true;
}

// physics_fluid_build_neighbors.cs.hlsl:21-147
void buildFluidNeighbors(cno_solver &s, uint32_t iter)
{
    const uint32_t maxN = s.desc.max_fluid_neighborhood;
    uint32_t trunc = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : trunc)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const f4 self = s.x[i];
        if (self.w <= kEps) continue;
        if (maxN == 0) { s.nbrCount[i] = 0; continue; }
        const f3 sd = iter > 0 ? xyz(s.fluidDelta[i]) : f3{0, 0, 0};
        const f3 sp = xyz(self) + sd;
        const float h = std::max(s.fluidMaterials[s.fluidMatIdx[i]].smoothing_radius, 1.0e-4f);
        const uint32_t *m = &s.meta[4 * i];
        const int32_t *e = &s.entries[4 * i];
        uint32_t count = 0;
        bool truncated = false;
        uint32_t *out = &s.nbrList[size_t(i) * maxN];
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int tx = e[0] + dx, ty = e[1] + dy, tz = e[2] + dz;
                    const CellRange rg = FindCellRange(s, CellKey(tx, ty, tz));
                    if (rg.key == kInvalid) continue;
                    for (uint32_t si = rg.start; si < rg.end; ++si) {
                        const uint32_t c = s.sortedIdx[si];
                        const int32_t *ce = &s.entries[4 * c];
                        if (ce[0] != tx || ce[1] != ty || ce[2] != tz) continue;
                        // ShouldProcessFluidNeighbor (physics_fluid_neighbor_build.hlsli:48-69)
                        if (c == i || s.kinds[c] != CN_PARTICLE_FLUID) continue;
                        const uint32_t *om = &s.meta[4 * c];
                        if (om[0] != m[0]) continue;
                        if (!((m[3] & om[2]) != 0u && (om[3] & m[2]) != 0u)) continue;
                        const f4 np = s.x[c];
                        if (np.w <= kEps) continue;
                        const f3 nd = iter > 0 ? xyz(s.fluidDelta[c]) : f3{0, 0, 0};
                        const f3 delta = sp - (xyz(np) + nd);
                        if (length(delta) >= h) continue;
                        if (count >= maxN) { truncated = true; continue; }
                        out[count++] = c;
                    }
                }
        s.nbrCount[i] = count;
        trunc += truncated ? 1u : 0u;
    }
    s.truncations += trunc;
}

// physics_fluid_compute_density_lambda.cs.hlsl:26-115
void fluidDensity(cno_solver &s, uint32_t iter)
{
    const uint32_t maxN = s.desc.max_fluid_neighborhood;
    const float bds = s.desc.fluid.boundary_density_scale;
    const float maxUnder = s.desc.fluid.max_under_density_ratio;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) { s.fluidNormalC[i] = f4{0, 0, 0, 0}; continue; }
        const f4 self = s.x[i];
        if (self.w <= kEps) { s.fluidNormalC[i] = f4{0, 0, 0, 0}; continue; }
        const f3 sdl = iter > 0 ? xyz(s.fluidDelta[i]) : f3{0, 0, 0};
        const f3 sp = xyz(self) + sdl;
        const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[i]];
        const float rho0 = std::max(fm.rest_density, 1.0f);
        const float scale = fm.density_constraint_scale;
        const float h = std::max(fm.smoothing_radius, 1.0e-4f);
        const float st = std::max(fm.surface_tension, 0.0f);
        float density = 0.0f;
        f3 normal{0, 0, 0};
        const uint32_t cnt = s.nbrCount[i];
        const uint32_t *lst = &s.nbrList[size_t(i) * maxN];
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t c = lst[k];
            const f3 nd = iter > 0 ? xyz(s.fluidDelta[c]) : f3{0, 0, 0};
            const f3 delta = sp - (xyz(s.x[c]) + nd);
            const float dist = length(delta);
            if (dist >= h) continue;
            density += SpikyW(dist, h);
            if (st > kEps) normal += SpikyGrad(delta, dist, h);
        }
        for (uint32_t c : s.boundaryCand[i]) {
            f3 ghost;
            if (!FluidGhostDelta(s, c, sp, h, ghost)) continue;
            const float dist = length(ghost);
            if (dist >= h) continue;
            density += SpikyW(dist, h) * bds;
        }
        const float C = std::max(density - rho0, -rho0 * std::max(maxUnder, 0.0f)) * scale;
        if (st > kEps) {
            normal = normal * st;
            s.fluidNormalC[i] = mk4(normal, C);
        } else {
            s.fluidNormalC[i] = f4{0, 0, 0, C};
        }
    }
}

// physics_fluid_compute_delta_positions.cs.hlsl:27-157
void fluidDeltaPositions(cno_solver &s, uint32_t iter, float dt)
{
    const uint32_t maxN = s.desc.max_fluid_neighborhood;
    const float coef = s.desc.fluid.constraint_relaxation;
    const float bdelta = s.desc.fluid.boundary_delta_scale;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) { s.fluidDx[i] = f4{0, 0, 0, 0}; continue; }
        const f4 self = s.x[i];
        if (self.w <= kEps) { s.fluidDx[i] = f4{0, 0, 0, 0}; continue; }
        const f3 sdl = iter > 0 ? xyz(s.fluidDelta[i]) : f3{0, 0, 0};
        const f3 sp = xyz(self) + sdl;
        const f4 snc = s.fluidNormalC[i];
        const float sC = snc.w;
        const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[i]];
        const float h = std::max(fm.smoothing_radius, 1.0e-4f);
        const float cohesion = dt * std::max(fm.cohesion, 0.0f);
        const float visc = dt * std::max(fm.viscosity, 0.0f);
        const float st = std::max(fm.surface_tension, 0.0f);
        const float cfl = std::max(fm.cfl_radius, 0.0f);
        f3 dp{0, 0, 0};
        float weight = 0.0f;
        const f3 sn = st > kEps ? xyz(snc) : f3{0, 0, 0};
        const uint32_t cnt = s.nbrCount[i];
        const uint32_t *lst = &s.nbrList[size_t(i) * maxN];
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t c = lst[k];
            const f4 np = s.x[c];
            if (np.w <= kEps) continue;
            const f3 nd = iter > 0 ? xyz(s.fluidDelta[c]) : f3{0, 0, 0};
            const f3 npos = xyz(np) + nd;
            const f3 delta = sp - npos;
            const float dist = length(delta);
            if (dist >= h || dist <= kEps) continue;
            const f4 nnc = s.fluidNormalC[c];
            const f3 nij = divv(delta, dist);
            const float dw = SpikyDW(dist, h);
            f3 pd = -0.5f * (sC + nnc.w) * dw * nij;
            if (s.fluidMatIdx[i] == s.fluidMatIdx[c]) {
                const f3 rel = sdl - nd;
                if (cohesion > kEps) pd -= nij * (cohesion * CohesionW(dist, h, fm.cohesion1, fm.cohesion2));
                if (visc > kEps) {
                    const float vs = 1.0f - (1.0f / (1.0f + visc * SpikyW(dist, h)));
                    pd -= vs * rel;
                }
                if (cfl > kEps) {
                    const float proj = dot(rel, nij);
                    if (proj < -cfl) pd -= nij * (proj + cfl) * 0.5f;
                }
                if (st > kEps) pd -= dt * (sn - xyz(nnc));
            }
            dp += pd;
            weight += 1.0f;
        }
        f3 bd{0, 0, 0};
        for (uint32_t c : s.boundaryCand[i]) {
            f3 ghost;
            if (!FluidGhostDelta(s, c, sp, h, ghost)) continue;
            const float dist = length(ghost);
            if (dist <= kEps || dist >= h) continue;
            const f3 nij = divv(ghost, dist);
            const float dw = SpikyDW(dist, h);
            bd += -std::max(sC, 0.0f) * dw * nij;
        }
        bd = bd * bdelta;
        const f3 packed = dp * coef + bd;
        s.fluidDx[i] = mk4(packed, weight);
    }
}

// physics_fluid_compute_vorticity.cs.hlsl:13-76 then physics_fluid_apply_vorticity_confinement.cs.hlsl:13-92,
// over the lists of the post-update rebuild: the curl of the velocity field from same-material
// neighbours, then the confinement force along the gradient of its magnitude, added to v.
bool anyVorticity(const cno_solver &s)
{
    for (const cn_fluid_material &m : s.fluidMaterials)
        if (std::max(m.vorticity_confinement, 0.0f) > kEps) return true;
    return false;
}
void fluidVorticity(cno_solver &s, float dt)
{
    const uint32_t maxN = s.desc.max_fluid_neighborhood;
    s.fluidVorticity.assign(s.N, f4{0, 0, 0, 0});
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[i]];
        if (std::max(fm.vorticity_confinement, 0.0f) <= kEps) continue;
        const f4 self = s.x[i];
        if (self.w <= kEps) continue;
        const f3 sp = xyz(self), sv = xyz(s.v[i]);
        const float h = std::max(fm.smoothing_radius, 1.0e-4f);
        f3 curl{0, 0, 0};
        const uint32_t *lst = &s.nbrList[size_t(i) * maxN];
        for (uint32_t k = 0; k < s.nbrCount[i]; ++k) {
            const uint32_t c = lst[k];
            if (s.fluidMatIdx[i] != s.fluidMatIdx[c]) continue;
            const f3 delta = sp - xyz(s.x[c]);
            const float dist = length(delta);
            if (dist <= kEps || dist >= h) continue;
            curl += cross(xyz(s.v[c]) - sv, SpikyGrad(delta, dist, h));
        }
        s.fluidVorticity[i] = mk4(curl, length(curl));
    }
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const cn_fluid_material &fm = s.fluidMaterials[s.fluidMatIdx[i]];
        const float conf = std::max(fm.vorticity_confinement, 0.0f);
        if (conf <= kEps) continue;
        const f4 self = s.x[i];
        if (self.w <= kEps) continue;
        const f4 sc = s.fluidVorticity[i];
        if (sc.w <= kEps) continue;
        const f3 sp = xyz(self);
        const float h = std::max(fm.smoothing_radius, 1.0e-4f);
        f3 grad{0, 0, 0};
        const uint32_t *lst = &s.nbrList[size_t(i) * maxN];
        for (uint32_t k = 0; k < s.nbrCount[i]; ++k) {
            const uint32_t c = lst[k];
            if (s.fluidMatIdx[i] != s.fluidMatIdx[c]) continue;
            const f3 delta = sp - xyz(s.x[c]);
            const float dist = length(delta);
            if (dist <= kEps || dist >= h) continue;
            grad += s.fluidVorticity[c].w * SpikyGrad(delta, dist, h);
        }
        const float gl = length(grad);
        if (gl <= kEps) continue;
        const f3 force = conf * cross(grad / gl, xyz(sc));
        s.v[i] = mk4(xyz(s.v[i]) + dt * force, 0.0f);
    }
}

// physics_fluid_apply_delta_positions.cs.hlsl:11-31 + physics_fluid_clamp_boundary.cs.hlsl:23-80
void fluidApplyAndClamp(cno_solver &s, uint32_t iter)
{
    const float relax = s.desc.fluid.position_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const f4 dw = s.fluidDx[i];
        const float weight = std::max(dw.w * relax, 1.0f);
        const f3 d = xyz(dw) / weight;
        const f3 prev = iter > 0 ? xyz(s.fluidDelta[i]) : f3{0, 0, 0};
        s.fluidDelta[i] = mk4(prev + d, 0.0f);
    }
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const f3 base = xyz(s.x[i]);
        const float pr = std::max(s.radii[i], 0.0f);
        f3 cur = base + xyz(s.fluidDelta[i]);
        for (uint32_t sweep = 0; sweep < 2u; ++sweep) {
            bool changed = false;
            for (uint32_t c : s.boundaryCand[i]) {
                float sd = 0.0f;
                f3 n{0, 1, 0};
                if (!FluidBoundaryContactInfo(s, c, cur, sd, n)) continue;
                if (sd >= pr) continue;
                cur += n * (pr - sd);
                changed = true;
            }
            if (!changed) break;
        }
        s.fluidDelta[i] = mk4(cur - base, 0.0f);
    }
}

// ---- XPBD families (Jacobi: solve writes per-constraint records, apply gathers) ----
// physics_soft_solve_edge_constraints.cs.hlsl:10-74
void solveEdgeOne(cno_solver &s, float dt, float relax, uint32_t e)
{
    const cn_soft_edge &ed = s.edges[e];
    f4 &cA = s.edgeCorr[2 * e], &cB = s.edgeCorr[2 * e + 1];
    cA = f4{0, 0, 0, 0}; cB = f4{0, 0, 0, 0};
    if (ed.enabled == 0u) return;
    const f4 a = s.x[ed.particle_a], b = s.x[ed.particle_b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    if (wSum <= kEps) return;
    const f3 delta = xyz(b) - xyz(a);
    const float l2 = dot(delta, delta);
    if (l2 <= kEps) return;
    const float len = std::sqrt(l2);
    const f3 gA = -delta / len;
    const f3 gB = -gA;
    const float compliance = std::max(ed.compliance, 0.0f);
    const float alpha = compliance / std::max(dt * dt, kEps);
    const float Cv = len - ed.rest_length;
    const float lambda = s.edgeLambda[e];
    const float den = wSum + alpha;
    if (den <= kEps) return;
    const float dl = -(Cv + alpha * lambda) / den;
    s.edgeLambda[e] = lambda + dl;
    cA = mk4(wA * dl * gA * relax, 0.0f);
    cB = mk4(wB * dl * gB * relax, 0.0f);
}
void solveEdges(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t ee = 0; ee < int64_t(s.edges.size()); ++ee) solveEdgeOne(s, dt, relax, uint32_t(ee));
}
// physics_soft_apply_edge_corrections.cs.hlsl:9-35 (and the strand distance apply, which
// indexes its correction records through the strand-segment incidence table,
// physics_strand_apply_distance_corrections.cs.hlsl:9-38)
void applyPairCorrections(cno_solver &s, const std::vector<Range> &ranges,
                          const std::vector<Incident> &inc, const std::vector<f4> &corr)
{
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f4 p = s.x[i];
        if (p.w <= kEps) continue;
        const Range r = ranges[i];
        f3 total{0, 0, 0};
        for (uint32_t k = 0; k < r.count; ++k) {
            const Incident &ref = inc[r.start + k];
            total += ref.slot == 0u ? xyz(corr[2 * ref.index]) : xyz(corr[2 * ref.index + 1]);
        }
        s.x[i] = mk4(xyz(p) + total, p.w);
    }
}
// physics_soft_apply_tet_corrections.cs.hlsl:9-50, physics_soft_apply_bend_corrections.cs.hlsl:9-51
void applyQuadCorrections(cno_solver &s, const std::vector<Range> &ranges,
                          const std::vector<Incident> &inc, const std::vector<f4> &corr)
{
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f4 p = s.x[i];
        if (p.w <= kEps) continue;
        const Range r = ranges[i];
        f3 total{0, 0, 0};
        for (uint32_t k = 0; k < r.count; ++k) {
            const Incident &ref = inc[r.start + k];
            const uint32_t slot = ref.slot > 3u ? 3u : ref.slot;
            total += xyz(corr[4 * ref.index + slot]);
        }
        s.x[i] = mk4(xyz(p) + total, p.w);
    }
}
// physics_soft_solve_tet_constraints.cs.hlsl:15-87
void solveTetOne(cno_solver &s, float dt, float relax, uint32_t t)
{
    const cn_soft_tet &tet = s.tets[t];
    const f4 q0 = s.x[tet.particle_indices[0]], q1 = s.x[tet.particle_indices[1]];
    const f4 q2 = s.x[tet.particle_indices[2]], q3 = s.x[tet.particle_indices[3]];
    const float w0 = q0.w, w1 = q1.w, w2 = q2.w, w3 = q3.w;
    if ((w0 + w1 + w2 + w3) <= kEps) return; // keeps the previous correction record
    const f3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2), p3 = xyz(q3);
    const float sv = dot(cross(p1 - p0, p2 - p0), p3 - p0) / 6.0f;
    const float vs = (sv >= 0.0f) ? 1.0f : -1.0f;
    const float vol = std::fabs(sv);
    const float rv = std::max(tet.rest_volume, 0.0f);
    const float Cv = vol - rv;
    const f3 g0 = cross(p3 - p1, p2 - p1) * (vs / 6.0f);
    const f3 g1 = cross(p2 - p0, p3 - p0) * (vs / 6.0f);
    const f3 g2 = cross(p3 - p0, p1 - p0) * (vs / 6.0f);
    const f3 g3 = cross(p1 - p0, p2 - p0) * (vs / 6.0f);
    const float sg = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2) + w3 * dot(g3, g3);
    const float compliance = std::max(tet.compliance, 0.0f);
    const float alpha = compliance / std::max(dt * dt, kEps);
    const float lambda = s.tetLambda[t];
    const float den = sg + alpha;
    if (den <= kEps) return;
    const float dl = -(Cv + alpha * lambda) / den;
    s.tetLambda[t] = lambda + dl;
    s.tetCorr[4 * t + 0] = mk4(w0 * dl * g0 * relax, 0.0f);
    s.tetCorr[4 * t + 1] = mk4(w1 * dl * g1 * relax, 0.0f);
    s.tetCorr[4 * t + 2] = mk4(w2 * dl * g2 * relax, 0.0f);
    s.tetCorr[4 * t + 3] = mk4(w3 * dl * g3 * relax, 0.0f);
}
void solveTets(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t tt = 0; tt < int64_t(s.tets.size()); ++tt) solveTetOne(s, dt, relax, uint32_t(tt));
}
// physics_soft_solve_bend_constraints.cs.hlsl:20-86
void solveBendOne(cno_solver &s, float dt, float relax, uint32_t b)
{
    const cn_soft_bend &bd = s.bends[b];
    f4 *out = &s.bendCorr[4 * b];
    out[0] = out[1] = out[2] = out[3] = f4{0, 0, 0, 0};
    const f4 q0 = s.x[bd.particle0], q1 = s.x[bd.particle1], q2 = s.x[bd.particle2];
    const float w0 = q0.w, w1 = q1.w, w2 = q2.w;
    if (w0 + w1 + w2 <= kEps) return;
    const f3 e0 = xyz(q0) - xyz(q1), e1 = xyz(q2) - xyz(q1);
    const float l0s = dot(e0, e0), l1s = dot(e1, e1);
    if (l0s <= kEps || l1s <= kEps) return;
    const float l0 = std::sqrt(l0s), l1 = std::sqrt(l1s);
    const f3 d0 = e0 / l0, d1 = e1 / l1;
    const float ct = std::min(std::max(dot(d0, d1), -1.0f + 1.0e-4f), 1.0f - 1.0e-4f);
    const float st2 = std::max(1.0f - ct * ct, 1.0e-8f);
    const float st = std::sqrt(st2);
    const float theta = std::acos(ct);
    const f3 g0 = -(d1 - ct * d0) / std::max(l0 * st, kEps);
    const f3 g2 = -(d0 - ct * d1) / std::max(l1 * st, kEps);
    const f3 g1 = -(g0 + g2);
    const float den = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2);
    const float alpha = std::max(bd.compliance, 0.0f) / std::max(dt * dt, kEps);
    if (den + alpha <= kEps) return;
    const float Cv = theta - bd.rest_angle;
    const float lambda = s.bendLambda[b];
    const float dl = -(Cv + alpha * lambda) / (den + alpha);
    s.bendLambda[b] = lambda + dl;
    out[0] = mk4(w0 * dl * g0 * relax, 0.0f);
    out[1] = mk4(w1 * dl * g1 * relax, 0.0f);
    out[2] = mk4(w2 * dl * g2 * relax, 0.0f);
}
void solveBends(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t bb = 0; bb < int64_t(s.bends.size()); ++bb) solveBendOne(s, dt, relax, uint32_t(bb));
}
// physics_cloth_solve_dihedral_constraints.cs.hlsl:20-95
void solveDihedralOne(cno_solver &s, float dt, float relax, uint32_t d)
{
    const uint32_t off = uint32_t(s.bends.size());
    const uint32_t ci = off + d;
    const cn_cloth_dihedral &h = s.dihedrals[d];
    f4 *out = &s.bendCorr[4 * ci];
    out[0] = out[1] = out[2] = out[3] = f4{0, 0, 0, 0};
    const f4 e0m = s.x[h.edge_particle0], e1m = s.x[h.edge_particle1];
    const f4 o0m = s.x[h.opposite_particle0], o1m = s.x[h.opposite_particle1];
    const f3 p0 = xyz(o0m), p1 = xyz(o1m), p2 = xyz(e0m), p3 = xyz(e1m);
    const f3 edge = p3 - p2;
    const float el2 = dot(edge, edge);
    const f3 rn0 = cross(p2 - p0, p3 - p0);
    const f3 rn1 = cross(p3 - p1, p2 - p1);
    const float n0s = dot(rn0, rn0), n1s = dot(rn1, rn1);
    if (el2 <= kEps || n0s <= kEps || n1s <= kEps) return;
    const float el = std::sqrt(el2);
    const float iel = 1.0f / el;
    const f3 sn0 = rn0 / n0s, sn1 = rn1 / n1s;
    const f3 dO0 = el * sn0, dO1 = el * sn1;
    const f3 dE0 = dot(p0 - p3, edge) * iel * sn0 + dot(p1 - p3, edge) * iel * sn1;
    const f3 dE1 = dot(p2 - p0, edge) * iel * sn0 + dot(p2 - p1, edge) * iel * sn1;
    const f3 g0 = -dE0, g1 = -dE1, g2 = -dO0, g3 = -dO1;
    const f3 n0 = rn0 / std::sqrt(n0s), n1 = rn1 / std::sqrt(n1s);
    const float theta = std::atan2(dot(edge * iel, cross(n0, n1)),
                                   std::min(std::max(dot(n0, n1), -1.0f), 1.0f));
    const float twoPi = 6.283185307179586f;
    float Cv = theta - h.rest_angle;
    Cv = Cv - twoPi * std::floor((Cv + 3.141592653589793f) / twoPi);
    const float w0 = e0m.w, w1 = e1m.w, w2 = o0m.w, w3 = o1m.w;
    const float den = w0 * dot(g0, g0) + w1 * dot(g1, g1) + w2 * dot(g2, g2) + w3 * dot(g3, g3);
    const float alpha = std::max(h.compliance, 0.0f) / std::max(dt * dt, kEps);
    if (den + alpha <= kEps) return;
    const float lambda = s.bendLambda[ci];
    const float dl = -(Cv + alpha * lambda) / (den + alpha);
    s.bendLambda[ci] = lambda + dl;
    out[0] = mk4(w0 * dl * g0 * relax, 0.0f);
    out[1] = mk4(w1 * dl * g1 * relax, 0.0f);
    out[2] = mk4(w2 * dl * g2 * relax, 0.0f);
    out[3] = mk4(w3 * dl * g3 * relax, 0.0f);
}
void solveDihedrals(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t dd = 0; dd < int64_t(s.dihedrals.size()); ++dd) solveDihedralOne(s, dt, relax, uint32_t(dd));
}

// 3x3 helpers of physics_strand_solve_{segment,joint}_constraints.cs.hlsl:12-64
struct m3 { float m[3][3]; };
inline m3 outer(f3 a, f3 b)
{
    return m3{{{a.x * b.x, a.x * b.y, a.x * b.z}, {a.y * b.x, a.y * b.y, a.y * b.z},
               {a.z * b.x, a.z * b.y, a.z * b.z}}};
}
inline void addScaled(m3 &acc, float s, const m3 &o)
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) acc.m[r][c] = acc.m[r][c] + s * o.m[r][c];
}
inline f3 mul3(const m3 &m, f3 v)
{
    return f3{dot(f3{m.m[0][0], m.m[0][1], m.m[0][2]}, v), dot(f3{m.m[1][0], m.m[1][1], m.m[1][2]}, v),
              dot(f3{m.m[2][0], m.m[2][1], m.m[2][2]}, v)};
}
inline m3 inverse3(const m3 &M)
{
    const float a00 = M.m[0][0], a01 = M.m[0][1], a02 = M.m[0][2];
    const float a10 = M.m[1][0], a11 = M.m[1][1], a12 = M.m[1][2];
    const float a20 = M.m[2][0], a21 = M.m[2][1], a22 = M.m[2][2];
    const float c00 = a11 * a22 - a12 * a21, c01 = a02 * a21 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const float c10 = a12 * a20 - a10 * a22, c11 = a00 * a22 - a02 * a20, c12 = a02 * a10 - a00 * a12;
    const float c20 = a10 * a21 - a11 * a20, c21 = a01 * a20 - a00 * a21, c22 = a00 * a11 - a01 * a10;
    const float det = a00 * c00 + a01 * c10 + a02 * c20;
    if (std::fabs(det) <= kEps) return m3{{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}};
    const float id = 1.0f / det;
    return m3{{{c00 * id, c01 * id, c02 * id}, {c10 * id, c11 * id, c12 * id},
               {c20 * id, c21 * id, c22 * id}}};
}
inline float StrandOrientationInvMass(float wA, float wB, float rl)
{
    const float ws = std::max(wA + wB, 0.0f);
    if (ws <= kEps || rl <= kEps) return 0.0f;
    const float avg = ws * 0.5f;
    return 12.0f * avg / std::max(rl * rl, kEps);
}
// physics_strand_solve_segment_constraints.cs.hlsl:66-147
void solveSegmentOne(cno_solver &s, float dt, float relax, uint32_t g)
{
    const cn_strand_segment &sg = s.segs[g];
    const f4 a = s.x[sg.particle_a], b = s.x[sg.particle_b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    f4 *out = &s.segCorr[3 * g];
    out[0] = out[1] = out[2] = f4{0, 0, 0, 0};
    if (wSum <= kEps) return;
    const f3 delta = xyz(b) - xyz(a);
    if (dot(delta, delta) <= kEps) return;
    const f4 q = QNormalize(s.segOrient[g]);
    const f3 axis = QRotate(q, f3{1, 0, 0});
    const float irl = 1.0f / std::max(sg.rest_length, kEps);
    const float oim = StrandOrientationInvMass(wA, wB, sg.rest_length);
    const f3 Cv = delta * irl - axis;
    const float alpha = std::max(sg.stretch_shear_compliance, 0.0f) / std::max(dt * dt, kEps);
    const f3 lambda = xyz(s.segLambda[g]);
    const f3 qv = xyz(q);
    const float qw = q.w;
    const f3 gQw = 2.0f * f3{qw, qv.z, -qv.y};
    const f3 gQx = 2.0f * f3{0.0f, qv.y, qv.z};
    const f3 gQy = 2.0f * f3{-qv.y, 0.0f, -qw};
    const f3 gQz = 2.0f * f3{-qv.z, qw, 0.0f};
    const float dg = wSum * irl * irl + alpha;
    m3 sys{{{dg, 0, 0}, {0, dg, 0}, {0, 0, dg}}};
    addScaled(sys, oim, outer(gQx, gQx));
    addScaled(sys, oim, outer(gQy, gQy));
    addScaled(sys, oim, outer(gQz, gQz));
    addScaled(sys, oim, outer(gQw, gQw));
    const f3 rhs = -(Cv + alpha * lambda);
    const f3 dl = mul3(inverse3(sys), rhs);
    if (dot(dl, dl) > 0.0f) {
        s.segLambda[g] = mk4(lambda + dl, 0.0f);
        out[0] = mk4(-wA * irl * dl * relax, 0.0f);
        out[1] = mk4(wB * irl * dl * relax, 0.0f);
        const f4 qg{-dot(gQx, dl), -dot(gQy, dl), -dot(gQz, dl), -dot(gQw, dl)};
        out[2] = qg * (oim * relax);
    }
}
void solveSegments(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t gg = 0; gg < int64_t(s.segs.size()); ++gg) solveSegmentOne(s, dt, relax, uint32_t(gg));
}
// physics_strand_apply_segment_corrections.cs.hlsl:11-43
void applySegments(cno_solver &s)
{
    const uint32_t n = std::max<uint32_t>(s.N, uint32_t(s.segs.size()));
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(n); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (i < s.N) {
            const f4 p = s.x[i];
            if (p.w > kEps) {
                const Range r = s.segRanges[i];
                f3 total{0, 0, 0};
                for (uint32_t k = 0; k < r.count; ++k) {
                    const Incident &ref = s.segInc[r.start + k];
                    total += ref.slot == 0u ? xyz(s.segCorr[3 * ref.index]) : xyz(s.segCorr[3 * ref.index + 1]);
                }
                s.x[i] = mk4(xyz(p) + total, p.w);
            }
        }
        if (i < s.segs.size()) s.segOrient[i] = QNormalize(s.segOrient[i] + s.segCorr[3 * i + 2]);
    }
}
// physics_strand_solve_joint_constraints.cs.hlsl:66-154
void solveJointOne(cno_solver &s, float dt, float relax, uint32_t j)
{
    const cn_strand_joint &jt = s.joints[j];
    const cn_strand_segment &sA = s.segs[jt.segment_a], &sB = s.segs[jt.segment_b];
    f4 *out = &s.jointCorr[5 * j];
    for (int k = 0; k < 5; ++k) out[k] = f4{0, 0, 0, 0};
    const f4 oA = QNormalize(s.segOrient[jt.segment_a]);
    const f4 oB = QNormalize(s.segOrient[jt.segment_b]);
    const float wA0 = s.x[sA.particle_a].w, wA1 = s.x[sA.particle_b].w;
    const float wB0 = s.x[sB.particle_a].w, wB1 = s.x[sB.particle_b].w;
    const float imA = StrandOrientationInvMass(wA0, wA1, sA.rest_length);
    const float imB = StrandOrientationInvMass(wB0, wB1, sB.rest_length);
    const f4 rel = QNormalize(QMul(QConj(oA), oB));
    f4 rr = QNormalize(f4{jt.rest_relative_orientation[0], jt.rest_relative_orientation[1],
                          jt.rest_relative_orientation[2], jt.rest_relative_orientation[3]});
    if (dot4(rel, rr) < 0.0f) rr = f4{-rr.x, -rr.y, -rr.z, -rr.w};
    const f3 Cv = xyz(rel) - xyz(rr);
    const f4 lambda = s.jointLambda[j];
    const float ba = std::max(jt.bend_compliance, 0.0f) / std::max(dt * dt, kEps);
    const float ta = std::max(jt.twist_compliance, 0.0f) / std::max(dt * dt, kEps);
    const f3 av{ta, ba, ba};
    m3 sys{{{av.x, 0, 0}, {0, av.y, 0}, {0, 0, av.z}}};
    const f3 va = xyz(oA), vb = xyz(oB);
    const float wa = oA.w, wb = oB.w;
    const f3 gAX{-wb, vb.z, -vb.y}, gAY{-vb.z, -wb, vb.x}, gAZ{vb.y, -vb.x, -wb}, gAW = vb;
    const f3 gBX{wa, -va.z, va.y}, gBY{va.z, wa, -va.x}, gBZ{-va.y, va.x, wa}, gBW = -va;
    addScaled(sys, imA, outer(gAX, gAX));
    addScaled(sys, imA, outer(gAY, gAY));
    addScaled(sys, imA, outer(gAZ, gAZ));
    addScaled(sys, imA, outer(gAW, gAW));
    addScaled(sys, imB, outer(gBX, gBX));
    addScaled(sys, imB, outer(gBY, gBY));
    addScaled(sys, imB, outer(gBZ, gBZ));
    addScaled(sys, imB, outer(gBW, gBW));
    const f3 rhs = -(Cv + av * xyz(lambda));
    const f3 dl = mul3(inverse3(sys), rhs);
    if (dot(dl, dl) > 0.0f) {
        s.jointLambda[j] = mk4(xyz(lambda) + dl, 0.0f);
        out[3] = f4{dot(gAX, dl), dot(gAY, dl), dot(gAZ, dl), dot(gAW, dl)} * (imA * relax);
        out[4] = f4{dot(gBX, dl), dot(gBY, dl), dot(gBZ, dl), dot(gBW, dl)} * (imB * relax);
    }
}
void solveJoints(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t jj = 0; jj < int64_t(s.joints.size()); ++jj) solveJointOne(s, dt, relax, uint32_t(jj));
}
// physics_strand_apply_joint_corrections.cs.hlsl
void applyJoints(cno_solver &s)
{
#pragma omp parallel for schedule(static)
    for (int64_t gg = 0; gg < int64_t(s.segs.size()); ++gg) {
        const uint32_t g = uint32_t(gg);
        const Range r = s.segJointRanges[g];
        f4 total{0, 0, 0, 0};
        for (uint32_t k = 0; k < r.count; ++k) {
            const Incident &ref = s.segJointInc[r.start + k];
            total = total + (ref.slot == 0u ? s.jointCorr[5 * ref.index + 3] : s.jointCorr[5 * ref.index + 4]);
        }
        s.segOrient[g] = QNormalize(s.segOrient[g] + total);
    }
}
// physics_strand_solve_distance_constraints.cs.hlsl:10-59
void solveDistanceOne(cno_solver &s, float dt, float relax, uint32_t c)
{
    const cn_strand_distance &dc = s.dists[c];
    f4 &cA = s.distCorr[2 * c], &cB = s.distCorr[2 * c + 1];
    cA = cB = f4{0, 0, 0, 0};
    const f4 a = s.x[dc.particle_a], b = s.x[dc.particle_b];
    const float wA = a.w, wB = b.w, wSum = wA + wB;
    if (wSum <= kEps) return;
    const f3 delta = xyz(b) - xyz(a);
    const float l2 = dot(delta, delta);
    if (l2 <= kEps) return;
    const float len = std::sqrt(l2);
    const f3 grad = delta / len;
    const float alpha = std::max(dc.distance_compliance, 0.0f) / std::max(dt * dt, kEps);
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
void solveDistances(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
#pragma omp parallel for schedule(static)
    for (int64_t cc = 0; cc < int64_t(s.dists.size()); ++cc) solveDistanceOne(s, dt, relax, uint32_t(cc));
}

// ---- coloured XPBD schedules (this build's opt-in; no reference counterpart) ----
// Greedy colouring: constraint c, in ascending order, takes the lowest colour that no earlier
// constraint sharing one of its elements holds.  Restated here with per-element colour lists.
template <class F>
void colourFamily(uint32_t n, uint32_t count, uint32_t per, F elementOf, std::vector<uint32_t> &order,
                  std::vector<uint32_t> &starts)
{
    order.clear();
    starts.clear();
    if (count == 0) return;
    std::vector<std::vector<uint32_t>> held(n);
    std::vector<uint32_t> colourOf(count);
    uint32_t colours = 0;
    for (uint32_t c = 0; c < count; ++c) {
        std::vector<uint32_t> taken;
        for (uint32_t k = 0; k < per; ++k) {
            const uint32_t e = elementOf(c, k);
            if (e < n) taken.insert(taken.end(), held[e].begin(), held[e].end());
        }
        std::sort(taken.begin(), taken.end());
        uint32_t colour = 0;
        for (uint32_t t : taken) {
            if (t == colour) ++colour;
            else if (t > colour) break;
        }
        for (uint32_t k = 0; k < per; ++k) {
            const uint32_t e = elementOf(c, k);
            if (e < n) held[e].push_back(colour);
        }
        colourOf[c] = colour;
        colours = std::max(colours, colour + 1);
    }
    starts.assign(colours + 1, 0);
    for (uint32_t c = 0; c < count; ++c) ++starts[colourOf[c] + 1];
    for (uint32_t k = 0; k < colours; ++k) starts[k + 1] += starts[k];
    order.resize(count);
    std::vector<uint32_t> fill(starts.begin(), starts.end() - 1);
    for (uint32_t c = 0; c < count; ++c) order[fill[colourOf[c]]++] = c;
}

void buildColourings(cno_solver &s)
{
    const uint32_t N = s.N, S = uint32_t(s.segs.size()), nb = uint32_t(s.bends.size());
    colourFamily(N, uint32_t(s.edges.size()), 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? s.edges[c].particle_a : s.edges[c].particle_b; }, s.colOrder[0], s.colStarts[0]);
    colourFamily(N, S, 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? s.segs[c].particle_a : s.segs[c].particle_b; }, s.colOrder[1], s.colStarts[1]);
    colourFamily(N, nb + uint32_t(s.dihedrals.size()), 4, [&](uint32_t c, uint32_t k) -> uint32_t {
        if (c < nb) {
            const cn_soft_bend &b = s.bends[c];
            return k == 0 ? b.particle0 : k == 1 ? b.particle1 : k == 2 ? b.particle2 : 0xffffffffu;
        }
        const cn_cloth_dihedral &h = s.dihedrals[c - nb];
        return k == 0 ? h.edge_particle0 : k == 1 ? h.edge_particle1 : k == 2 ? h.opposite_particle0
                                                                             : h.opposite_particle1;
    }, s.colOrder[2], s.colStarts[2]);
    colourFamily(S, uint32_t(s.joints.size()), 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? s.joints[c].segment_a : s.joints[c].segment_b; }, s.colOrder[3], s.colStarts[3]);
    colourFamily(N, uint32_t(s.dists.size()), 2, [&](uint32_t c, uint32_t k) {
        return k == 0 ? s.dists[c].particle_a : s.dists[c].particle_b; }, s.colOrder[4], s.colStarts[4]);
    colourFamily(N, uint32_t(s.tets.size()), 4, [&](uint32_t c, uint32_t k) {
        return s.tets[c].particle_indices[k]; }, s.colOrder[5], s.colStarts[5]);
    s.softAcc.assign(N, f4{0, 0, 0, 0});
    s.orientAcc.assign(S, f4{0, 0, 0, 0});
}

// A constraint's records into its particles (Gauss-Seidel: x += r where invMass > kEps) or into
// the family's per-particle sum (colour Jacobi).
inline void moveRecord(cno_solver &s, bool gs, uint32_t p, const f4 &r)
{
    if (p >= s.N) return;
    if (gs) {
        const f4 q = s.x[p];
        if (q.w > kEps) s.x[p] = mk4(xyz(q) + xyz(r), q.w);
    } else {
        s.softAcc[p] = mk4(xyz(s.softAcc[p]) + xyz(r), 0.0f);
    }
}
inline void moveOrientation(cno_solver &s, bool gs, uint32_t g, const f4 &r)
{
    if (g >= s.segs.size()) return;
    if (gs) s.segOrient[g] = QNormalize(s.segOrient[g] + r);
    else s.orientAcc[g] = s.orientAcc[g] + r;
}

void colourOne(cno_solver &s, uint32_t fam, float dt, float relax, bool gs, uint32_t c)
{
    const uint32_t nb = uint32_t(s.bends.size());
    switch (fam) {
    case 0: {
        solveEdgeOne(s, dt, relax, c);
        moveRecord(s, gs, s.edges[c].particle_a, s.edgeCorr[2 * c]);
        moveRecord(s, gs, s.edges[c].particle_b, s.edgeCorr[2 * c + 1]);
        break;
    }
    case 1: { // the segment's own orientation is read by it alone: applied in place
        solveSegmentOne(s, dt, relax, c);
        moveRecord(s, gs, s.segs[c].particle_a, s.segCorr[3 * c]);
        moveRecord(s, gs, s.segs[c].particle_b, s.segCorr[3 * c + 1]);
        s.segOrient[c] = QNormalize(s.segOrient[c] + s.segCorr[3 * c + 2]);
        break;
    }
    case 2: {
        const f4 *r = &s.bendCorr[4 * size_t(c)];
        if (c < nb) {
            solveBendOne(s, dt, relax, c);
            moveRecord(s, gs, s.bends[c].particle0, r[0]);
            moveRecord(s, gs, s.bends[c].particle1, r[1]);
            moveRecord(s, gs, s.bends[c].particle2, r[2]);
        } else {
            solveDihedralOne(s, dt, relax, c - nb);
            const cn_cloth_dihedral &h = s.dihedrals[c - nb];
            moveRecord(s, gs, h.edge_particle0, r[0]);
            moveRecord(s, gs, h.edge_particle1, r[1]);
            moveRecord(s, gs, h.opposite_particle0, r[2]);
            moveRecord(s, gs, h.opposite_particle1, r[3]);
        }
        break;
    }
    case 3: {
        solveJointOne(s, dt, relax, c);
        moveOrientation(s, gs, s.joints[c].segment_a, s.jointCorr[5 * c + 3]);
        moveOrientation(s, gs, s.joints[c].segment_b, s.jointCorr[5 * c + 4]);
        break;
    }
    case 4: {
        solveDistanceOne(s, dt, relax, c);
        moveRecord(s, gs, s.dists[c].particle_a, s.distCorr[2 * c]);
        moveRecord(s, gs, s.dists[c].particle_b, s.distCorr[2 * c + 1]);
        break;
    }
    default: {
        solveTetOne(s, dt, relax, c);
        for (uint32_t k = 0; k < 4; ++k) moveRecord(s, gs, s.tets[c].particle_indices[k], s.tetCorr[4 * c + k]);
        break;
    }
    }
}

// Particles [lo, hi) with records in a family's incidence (strand distances: the segments').
std::pair<uint32_t, uint32_t> familyWindow(const cno_solver &s, uint32_t fam)
{
    const std::vector<Range> &r = fam == 0 ? s.edgeRanges : fam == 2 ? s.bendRanges : fam == 5 ? s.tetRanges : s.segRanges;
    uint32_t lo = uint32_t(r.size()), hi = 0;
    for (uint32_t i = 0; i < r.size(); ++i)
        if (r[i].count) {
            lo = std::min(lo, i);
            hi = i + 1;
        }
    return lo < hi ? std::make_pair(lo, hi) : std::make_pair(0u, 0u);
}

// One soft iteration under a coloured schedule: each family in the gather order, colour by colour.
void colouredSoftIteration(cno_solver &s, float dt)
{
    const float relax = s.desc.soft.internal_relaxation;
    const bool gs = s.desc.soft.xpbd_schedule == CN_XPBD_COLOUR_GAUSS_SEIDEL;
    for (uint32_t fam = 0; fam < 6; ++fam) {
        const std::vector<uint32_t> &order = s.colOrder[fam], &starts = s.colStarts[fam];
        if (order.empty()) continue;
        for (size_t k = 0; k + 1 < starts.size(); ++k) {
#pragma omp parallel for schedule(static)
            for (int64_t j = int64_t(starts[k]); j < int64_t(starts[k + 1]); ++j)
                colourOne(s, fam, dt, relax, gs, order[size_t(j)]);
        }
        if (gs) continue;
        if (fam == 3) {
            for (size_t g = 0; g < s.segs.size(); ++g) {
                const f4 a = s.orientAcc[g];
                s.orientAcc[g] = f4{0, 0, 0, 0};
                s.segOrient[g] = QNormalize(s.segOrient[g] + a);
            }
            continue;
        }
        const auto win = familyWindow(s, fam);
        for (uint32_t i = win.first; i < win.second; ++i) {
            const f4 a = s.softAcc[i];
            s.softAcc[i] = f4{0, 0, 0, 0};
            const f4 p = s.x[i];
            if (p.w > kEps) s.x[i] = mk4(xyz(p) + xyz(a), p.w);
        }
    }
}

// physics_particle_generate_explicit_contacts.cs.hlsl (no suturing / proxies) +
// compact + physics_particle_solve_explicit_contacts.cs.hlsl (non-proxy branch).
void particleParticleContacts(cno_solver &s)
{
    const size_t P = s.particlePairs.size();
    s.particleContacts.assign(P, ParticleContact{});
#pragma omp parallel for schedule(static)
    for (int64_t pp = 0; pp < int64_t(P); ++pp) {
        ParticleContact out{};
        const uint32_t a = s.particlePairs[pp].first, b = s.particlePairs[pp].second;
        out.material = mk4(CombineContactMaterial(s.contactMaterials[s.matIdx[a]],
                                                  s.contactMaterials[s.matIdx[b]]), 0.0f);
        if (s.kinds[a] == CN_PARTICLE_FLUID && s.kinds[b] == CN_PARTICLE_FLUID) {
            s.particleContacts[pp] = out;
            continue;
        }
        const f3 pa = xyz(s.x[a]), pb = xyz(s.x[b]);
        const float cr = s.radii[a] + s.radii[b];
        const f3 delta = pb - pa;
        const float d2 = dot(delta, delta);
        if (d2 <= kEps) {
            out.a = a; out.b = b; out.active = 1;
            out.normalPenetration = f4{0, 1, 0, cr};
            s.particleContacts[pp] = out;
            continue;
        }
        const float dist = std::sqrt(d2);
        const float pen = cr - dist;
        if (pen > 0.0f) {
            out.a = a; out.b = b; out.active = 1;
            out.normalPenetration = mk4(delta / dist, pen);
        }
        s.particleContacts[pp] = out;
    }
    s.activeParticleContacts.clear();
    for (const ParticleContact &c : s.particleContacts)
        if (c.active) s.activeParticleContacts.push_back(c);
    const float relax = s.desc.contact.soft_relaxation;
    const float maxCorr = s.desc.contact.soft_max_correction_per_iteration;
    const float minFric = s.desc.contact.position_friction_min_distance;
    // physics_particle_solve_explicit_contacts.cs.hlsl:27-238 (float atomics in contact order);
    // a rigid proxy's share goes to its body
    for (const ParticleContact &c : s.activeParticleContacts) {
        const f4 A = s.x[c.a], Bp = s.x[c.b];
        const bool proxyA = c.a < s.nProxy, proxyB = c.b < s.nProxy;
        float iA = A.w, iB = Bp.w;
        f3 curA = xyz(A), curB = xyz(Bp), prevA = xyz(s.xprev[c.a]), prevB = xyz(s.xprev[c.b]);
        f3 rA{0, 0, 0}, rB{0, 0, 0}, inA{0, 0, 0}, inB{0, 0, 0};
        f4 qA{0, 0, 0, 1}, qB{0, 0, 0, 1};
        uint32_t bA = 0, bB = 0;
        auto proxySide = [&](uint32_t p, uint32_t &b, float &im, f3 &inv, f4 &q, f3 &cur, f3 &prev, f3 &r) {
            b = s.ownerIdx[p];
            const f4 bp = s.predBodyPos[b];
            q = QNormalize(s.predBodyRot[b]);
            const f4 pq = QNormalize(s.prevBodyRot[b]);
            im = s.bodyType[b] == CN_BODY_DYNAMIC ? bp.w : 0.0f;
            inv = im > kEps ? xyz(s.bodyInvInertia[b]) : f3{0, 0, 0};
            const f3 l = xyz(s.proxyLocal[p]);
            cur = xyz(bp) + QRotate(q, l);
            prev = xyz(s.prevBodyPos[b]) + QRotate(pq, l);
            r = cur - xyz(bp);
        };
        if (proxyA) proxySide(c.a, bA, iA, inA, qA, curA, prevA, rA);
        if (proxyB) proxySide(c.b, bB, iB, inB, qB, curB, prevB, rB);
        if (iA <= kEps && iB <= kEps) continue;
        const float pen = std::min(std::max(c.normalPenetration.w - s.slop(), 0.0f), maxCorr);
        if (pen <= 0.0f) continue;
        const f3 mat = xyz(c.material);
        const f3 n = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
        const f3 relDisp = (curB - prevB) - (curA - prevA);
        const float nmA = proxyA ? ContactEffectiveMass(iA, inA, qA, rA, n) : iA;
        const float nmB = proxyB ? ContactEffectiveMass(iB, inB, qB, rB, n) : iB;
        const float denom = nmA + nmB;
        if (denom <= kEps) continue;
        const float lambda = (pen / denom) * relax;
        f3 cA{0, 0, 0}, cB{0, 0, 0}, tA{0, 0, 0}, tB{0, 0, 0}, wA{0, 0, 0}, wB{0, 0, 0};
        if (proxyA) {
            tA = -n * (iA * lambda);
            wA = -MulWorldInvInertia(inA, qA, cross(rA, n)) * lambda;
        } else {
            cA = -n * (iA * lambda);
        }
        if (proxyB) {
            tB = n * (iB * lambda);
            wB = MulWorldInvInertia(inB, qB, cross(rB, n)) * lambda;
        } else {
            cB = n * (iB * lambda);
        }
        const f3 tdisp = ProjectOntoTangent(relDisp, n);
        // ComputePositionFrictionDelta (physics_rigid_solver_shared.hlsli:50-68)
        f3 fd{0, 0, 0};
        const float td = length(tdisp);
        if (!(td <= minFric || pen <= kEps)) {
            const float sl = saturate(mat.z) * pen;
            if (td <= sl) fd = tdisp;
            else fd = tdisp * std::min(saturate(mat.x) * pen / td, 1.0f);
        }
        const float fdist = length(fd);
        if (fdist > 0.0f) {
            const f3 t = fd / fdist;
            const float tmA = proxyA ? ContactEffectiveMass(iA, inA, qA, rA, t) : iA;
            const float tmB = proxyB ? ContactEffectiveMass(iB, inB, qB, rB, t) : iB;
            const float tden = tmA + tmB;
            if (tden > kEps) {
                const float tl = (fdist / tden) * relax;
                if (proxyA) {
                    tA += t * (iA * tl);
                    wA += MulWorldInvInertia(inA, qA, cross(rA, t)) * tl;
                } else {
                    cA += t * (iA * tl);
                }
                if (proxyB) {
                    tB -= t * (iB * tl);
                    wB -= MulWorldInvInertia(inB, qB, cross(rB, t)) * tl;
                } else {
                    cB -= t * (iB * tl);
                }
            }
        }
        if (!proxyA && iA > kEps) s.posCorr[c.a] = mk4(xyz(s.posCorr[c.a]) + cA, s.posCorr[c.a].w);
        if (!proxyB && iB > kEps) s.posCorr[c.b] = mk4(xyz(s.posCorr[c.b]) + cB, s.posCorr[c.b].w);
        if (proxyA && iA > kEps) {
            s.bodyTransCorr[bA] = s.bodyTransCorr[bA] + tA;
            s.bodyRotCorr[bA] = s.bodyRotCorr[bA] + wA;
        }
        if (proxyB && iB > kEps) {
            s.bodyTransCorr[bB] = s.bodyTransCorr[bB] + tB;
            s.bodyRotCorr[bB] = s.bodyRotCorr[bB] + wB;
        }
    }
}

// physics_particle_rigid_generate_contacts.cs.hlsl:29-210 + compact_active_rigid_contacts +
// physics_particle_rigid_solve_contacts.cs.hlsl:27-141 (static / kinematic bodies).
void particleRigidContacts(cno_solver &s)
{
    const size_t P = s.rigidPairs.size();
    s.rigidContacts.assign(P, RigidContact{});
#pragma omp parallel for schedule(static)
    for (int64_t pp = 0; pp < int64_t(P); ++pp) {
        RigidContact out{};
        const uint32_t i = s.rigidPairs[pp].first, b = s.rigidPairs[pp].second;
        if (s.ownerTypes[i] == CN_OWNER_RIGID_BODY) { s.rigidContacts[pp] = out; continue; }
        const f3 sp = xyz(s.x[i]);
        const float sr = s.radii[i];
        const uint32_t *m = &s.meta[4 * i];
        const f3 bpos = xyz(s.predBodyPos[b]);
        const f4 bq = QNormalize(s.predBodyRot[b]);
        const f4 bsc = s.bodyScale[b];
        const uint32_t co = s.bodyColRanges[2 * b], cc = s.bodyColRanges[2 * b + 1];
        float bestPen = 0.0f;
        uint32_t bestCol = 0;
        f3 bestN{0, 1, 0}, bestW{0, 0, 0};
        for (uint32_t k = 0; k < kColliderCap; ++k) {
            if (k >= cc) break;
            const uint32_t c = s.bodyColIdx[co + k];
            const cn_collider_broadphase &bp = s.colBp[c];
            if (bp.enabled_flag == 0u || bp.environment_index != m[0]) continue;
            if ((m[3] & bp.collision_layer) == 0u || (bp.collision_mask & m[2]) == 0u) continue;
            const cn_collider_geometry &cg = s.colGeo[c];
            const f3 clp{cg.local_position[0], cg.local_position[1], cg.local_position[2]};
            const f4 clq = QNormalize(f4{cg.local_orientation[0], cg.local_orientation[1],
                                         cg.local_orientation[2], cg.local_orientation[3]});
            const f3 cwp = bpos + QRotate(bq, clp);
            const f4 cwq = QNormalize(QMul(bq, clq));
            const f3 pl = QInvRotate(cwq, sp - cwp);
            f3 nl{0, 1, 0}, cw{0, 0, 0};
            float sd = 0.0f;
            const f4 sp4{cg.shape_params[0], cg.shape_params[1], cg.shape_params[2], cg.shape_params[3]};
            if (bp.shape_type == CN_COLLIDER_SPHERE) {
                const float r = SphereRadius(sp4, bsc);
                const float l = std::sqrt(dot(pl, pl));
                nl = l > kEps ? (pl / l) : f3{0, 1, 0};
                sd = l - r;
                cw = cwp + QRotate(cwq, nl * r);
            } else if (bp.shape_type == CN_COLLIDER_BOX) {
                const f3 he = BoxHalfExtents(sp4, bsc);
                const f3 cl = clamp3(pl, -he, he);
                const f3 d = pl - cl;
                const float dl = std::sqrt(dot(d, d));
                if (dl > kEps) {
                    nl = d / dl;
                    sd = dl;
                    cw = cwp + QRotate(cwq, cl);
                } else {
                    nl = ClosestFaceNormalLocal(pl, he);
                    const f3 ds = he - fabs3(pl);
                    sd = -std::min(ds.x, std::min(ds.y, ds.z));
                    f3 cs = pl;
                    if (std::fabs(nl.x) > 0.5f) cs.x = nl.x * he.x;
                    else if (std::fabs(nl.y) > 0.5f) cs.y = nl.y * he.y;
                    else cs.z = nl.z * he.z;
                    cw = cwp + QRotate(cwq, cs);
                }
            } else {
                f3 a, b2;
                float cr = 0.0f;
                CapsuleSegment(cwp, cwq, sp4, bsc, a, b2, cr);
                const f3 seg = b2 - a;
                const float l2 = dot(seg, seg);
                float t = 0.0f;
                if (l2 > kEps) t = saturate(dot(sp - a, seg) / l2);
                const f3 cl = lerp3(a, b2, t);
                const f3 d = sp - cl;
                const float l = std::sqrt(dot(d, d));
                const f3 wn = l > kEps ? (d / l) : f3{1, 0, 0};
                sd = l - cr;
                nl = QInvRotate(cwq, wn);
                cw = cl + wn * cr;
            }
            const float pen = sr - sd;
            if (pen <= 0.0f || pen <= bestPen) continue;
            bestPen = pen;
            bestCol = c;
            bestN = SafeNormalize(QRotate(cwq, nl), f3{0, 1, 0});
            bestW = cw;
        }
        if (bestPen > 0.0f) {
            out.particle = i; out.body = b; out.collider = bestCol; out.active = 1;
            out.normalPenetration = mk4(bestN, bestPen);
            out.rigidLocalPoint = mk4(QInvRotate(bq, bestW - bpos), 0.0f);
        }
        s.rigidContacts[pp] = out;
    }
    s.activeRigidContacts.clear();
    for (const RigidContact &c : s.rigidContacts)
        if (c.active) s.activeRigidContacts.push_back(c);
    const float relax = s.desc.contact.soft_relaxation;
    const float maxCorr = s.desc.contact.soft_max_correction_per_iteration;
    const float minFric = s.desc.contact.position_friction_min_distance;
    for (const RigidContact &c : s.activeRigidContacts) {
        const uint32_t i = c.particle, b = c.body;
        const f4 sp = s.x[i];
        const float iS = sp.w;
        const f3 prevS = xyz(s.xprev[i]);
        const f4 prevB = s.prevBodyPos[b], predB = s.predBodyPos[b];
        const f4 prevQ = QNormalize(s.prevBodyRot[b]), predQ = QNormalize(s.predBodyRot[b]);
        const float iR = s.bodyType[b] == CN_BODY_DYNAMIC ? predB.w : 0.0f;
        if (iS <= kEps && iR <= kEps) continue;
        const float pen = std::min(std::max(c.normalPenetration.w - s.slop(), 0.0f), maxCorr);
        if (pen <= 0.0f) continue;
        const f3 n = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
        f3 inI = xyz(s.bodyInvInertia[b]);
        const f3 mat = CombineContactMaterial(s.contactMaterials[s.matIdx[i]], s.colMat[c.collider]);
        if (iR <= kEps) inI = f3{0, 0, 0};
        const f3 prevCP = xyz(prevB) + QRotate(prevQ, xyz(c.rigidLocalPoint));
        const f3 cp = xyz(predB) + QRotate(predQ, xyz(c.rigidLocalPoint));
        const f3 rR = cp - xyz(predB);
        const float nmR = ContactEffectiveMass(iR, inI, predQ, rR, n);
        const float denom = iS + nmR;
        if (denom <= kEps) continue;
        const float lambda = (pen / denom) * relax;
        f3 corr = n * (iS * lambda);
        f3 rt = -n * (iR * lambda);
        f3 rr = -MulWorldInvInertia(inI, predQ, cross(rR, n)) * lambda;
        const f3 relDisp = (cp - prevCP) - (xyz(sp) - prevS);
        const f3 tdisp = ProjectOntoTangent(relDisp, n);
        f3 fd{0, 0, 0};
        const float td = length(tdisp);
        if (!(td <= minFric || pen <= kEps)) {
            const float sl = saturate(mat.z) * pen;
            if (td <= sl) fd = tdisp;
            else fd = tdisp * std::min(saturate(mat.x) * pen / td, 1.0f);
        }
        const float fdist = length(fd);
        if (fdist > 0.0f) {
            const f3 t = fd / fdist;
            const float tmR = ContactEffectiveMass(iR, inI, predQ, rR, t);
            const float tden = iS + tmR;
            if (tden > kEps) {
                const float tl = fdist / tden;
                corr += t * (tl * iS * relax);
                rt -= t * (tl * iR * relax);
                rr -= MulWorldInvInertia(inI, predQ, cross(rR, t)) * (tl * relax);
            }
        }
        if (iS > kEps) s.posCorr[i] = mk4(xyz(s.posCorr[i]) + corr, s.posCorr[i].w);
        if (iR > kEps) { // float atomics in the reference; summed here in pair order
            s.bodyTransCorr[b] += rt;
            s.bodyRotCorr[b] += rr;
        }
    }
}

// physics_rigid_apply_corrections.cs.hlsl:13-54
void applyRigidCorrections(cno_solver &s)
{
    for (uint32_t b = 0; b < s.B; ++b) {
        f4 p = s.predBodyPos[b];
        f4 q = QNormalize(s.predBodyRot[b]);
        f3 tc = s.bodyTransCorr[b], rc = s.bodyRotCorr[b];
        if (s.bodyType[b] == CN_BODY_DYNAMIC && p.w != 0.0f) {
            tc = ClampLength(tc, s.desc.rigid.max_translation_correction_per_iteration);
            rc = ClampLength(rc, s.desc.rigid.max_rotation_correction_per_iteration);
            p = mk4(xyz(p) + tc, p.w);
            q = QNormalize(QMul(QuaternionFromRotationVector(rc), q));
        }
        s.predBodyPos[b] = p;
        s.predBodyRot[b] = q;
        s.bodyTransCorr[b] = f3{0, 0, 0};
        s.bodyRotCorr[b] = f3{0, 0, 0};
    }
}

// physics_rigid_update_velocities.cs.hlsl:14-51
void updateRigidVelocities(cno_solver &s, float dt)
{
    for (uint32_t b = 0; b < s.B; ++b) {
        const f4 prevP = s.prevBodyPos[b];
        const f4 prevQ = QNormalize(s.prevBodyRot[b]);
        const f4 p = s.predBodyPos[b];
        const f4 q = QNormalize(s.predBodyRot[b]);
        if (s.bodyType[b] == CN_BODY_STATIC) {
            s.predBodyRot[b] = QNormalize(q);
            s.predBodyLin[b] = f4{0, 0, 0, 0};
            s.predBodyAng[b] = f4{0, 0, 0, 0};
            continue;
        }
        const f3 l = (xyz(p) - xyz(prevP)) / std::max(dt, kEps);
        const f3 a = AngularVelocityFromQuaternionDelta(prevQ, q, std::max(dt, kEps));
        s.predBodyRot[b] = q;
        s.predBodyLin[b] = mk4(l, 0.0f);
        s.predBodyAng[b] = mk4(a, 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Rigid-rigid contacts (scenes with dynamic bodies).
// ---------------------------------------------------------------------------
// ComputePositionFrictionDelta (physics_rigid_solver_shared.hlsli:50-68)
inline f3 PositionFrictionDelta(f3 td, float pen, float kin, float stat, float minDist)
{
    const float d = length(td);
    if (d <= minDist || pen <= kEps) return f3{0, 0, 0};
    const float sl = saturate(stat) * pen;
    if (d <= sl) return td;
    return td * std::min(saturate(kin) * pen / d, 1.0f);
}
inline f3 ClosestPointOnBox(f3 q, f3 c, f4 o, f3 h) { return c + QRotate(o, clamp3(QInvRotate(o, q - c), f3{-h.x, -h.y, -h.z}, h)); }
inline f3 BoxSupportPoint(f3 c, f4 o, f3 h, f3 dir)
{
    const f3 ld = QInvRotate(o, dir);
    return c + QRotate(o, f3{ld.x >= 0.0f ? h.x : -h.x, ld.y >= 0.0f ? h.y : -h.y, ld.z >= 0.0f ? h.z : -h.z});
}
inline float Comp(f3 v, uint32_t i) { return i == 0u ? v.x : (i == 1u ? v.y : v.z); }
inline float PenetrationFromPoints(f3 a, f3 b, f3 n) { return std::max(0.0f, -dot(b - a, n)); }

// physics_rigid_contact_primitives.hlsli:17-47
bool SphereSphere(f3 cA, float rA, f3 cB, float rB, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0, 0, 0};
    pen = 0.0f;
    const f3 d = cB - cA;
    const float d2 = dot(d, d);
    const float r = rA + rB;
    if (d2 > r * r) return false;
    const float dist = std::sqrt(std::max(d2, 0.0f));
    n = dist > kEps ? d / dist : f3{0, 1, 0};
    pA = cA + n * rA;
    pB = cB - n * rB;
    pen = PenetrationFromPoints(pA, pB, n);
    return pen > 0.0f;
}
// :50-99
bool SphereBox(f3 sc, float sr, f3 bc, f4 bq, f3 h, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0, 0, 0};
    pen = 0.0f;
    const f3 ls = QInvRotate(bq, sc - bc);
    const f3 cl = clamp3(ls, f3{-h.x, -h.y, -h.z}, h);
    const bool inside = ls.x >= -h.x && ls.y >= -h.y && ls.z >= -h.z && ls.x <= h.x && ls.y <= h.y && ls.z <= h.z;
    if (!inside) {
        const f3 bp = bc + QRotate(bq, cl);
        const f3 d = bp - sc;
        const float d2 = dot(d, d);
        if (d2 > sr * sr) return false;
        const float dist = std::sqrt(std::max(d2, 0.0f));
        n = dist > kEps ? d / dist : f3{0, 1, 0};
        pA = sc + n * sr;
        pB = bp;
        pen = PenetrationFromPoints(pA, pB, n);
        return pen > 0.0f;
    }
    const f3 lfn = ClosestFaceNormalLocal(ls, h);
    const float depth = std::min(h.x - std::fabs(ls.x), std::min(h.y - std::fabs(ls.y), h.z - std::fabs(ls.z)));
    n = -QRotate(bq, lfn);
    pB = bc + QRotate(bq, ls + lfn * depth);
    pA = sc + n * sr;
    pen = depth + sr;
    return pen > 0.0f;
}
// :101-119
bool SphereCapsule(f3 sc, float sr, f3 a, f3 b, float cr, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    const f3 seg = b - a;
    const float l2 = dot(seg, seg);
    float t = 0.0f;
    if (l2 > kEps) t = saturate(dot(sc - a, seg) / l2);
    return SphereSphere(sc, sr, a + seg * t, cr, n, pA, pB, pen);
}
// :272-331
void ClosestSegmentSegment(f3 a0, f3 a1, f3 b0, f3 b1, f3 &oa, f3 &ob)
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
            if (tn < 0.0f) { t = 0.0f; sv = saturate(-c / a); }
            else if (tn > e) { t = 1.0f; sv = saturate((b - c) / a); }
            else t = tn / e;
        }
    }
    oa = a0 + d1 * sv;
    ob = b0 + d2 * t;
}
// :121-270 (separating-axis test, the deepest axis' contact points)
bool BoxBox(f3 cA, f4 qA, f3 hA, f3 cB, f4 qB, f3 hB, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0, 0, 0};
    pen = 0.0f;
    const f3 axA[3] = {QRotate(qA, f3{1, 0, 0}), QRotate(qA, f3{0, 1, 0}), QRotate(qA, f3{0, 0, 1})};
    const f3 axB[3] = {QRotate(qB, f3{1, 0, 0}), QRotate(qB, f3{0, 1, 0}), QRotate(qB, f3{0, 0, 1})};
    const f3 cd = cB - cA;
    auto proj = [](f3 axis, const f3 *ax, f3 h) {
        return h.x * std::fabs(dot(axis, ax[0])) + h.y * std::fabs(dot(axis, ax[1])) + h.z * std::fabs(dot(axis, ax[2]));
    };
    float minPen = 3.402823466e+38f;
    f3 best{0, 1, 0};
    uint32_t bType = 0, bA = 0, bB = 0;
    auto test = [&](f3 axis, uint32_t type, uint32_t ia, uint32_t ib) {
        const float l2 = dot(axis, axis);
        if (l2 <= kEps) return true;
        const f3 nn = axis * (1.0f / std::sqrt(l2));
        const float dist = std::fabs(dot(cd, nn));
        const float ov = proj(nn, axA, hA) + proj(nn, axB, hB) - dist;
        if (ov < 0.0f) return false;
        if (ov < minPen) {
            minPen = ov;
            best = dot(cd, nn) >= 0.0f ? nn : -nn;
            bType = type; bA = ia; bB = ib;
        }
        return true;
    };
    for (uint32_t i = 0; i < 3; ++i) if (!test(axA[i], 0, i, 0)) return false;
    for (uint32_t i = 0; i < 3; ++i) if (!test(axB[i], 1, i, 0)) return false;
    for (uint32_t a = 0; a < 3; ++a)
        for (uint32_t b = 0; b < 3; ++b)
            if (!test(cross(axA[a], axB[b]), 2, a, b)) return false;
    n = best;
    auto edge = [](uint32_t axis, f3 c, const f3 *ax, f3 h, f3 dir, f3 &e0, f3 &e1) {
        const uint32_t oa = (axis + 1) % 3, ob = (axis + 2) % 3;
        const float sa = dot(ax[oa], dir) >= 0.0f ? 1.0f : -1.0f;
        const float sb = dot(ax[ob], dir) >= 0.0f ? 1.0f : -1.0f;
        const f3 ec = c + ax[oa] * (Comp(h, oa) * sa) + ax[ob] * (Comp(h, ob) * sb);
        const f3 eh = ax[axis] * Comp(h, axis);
        e0 = ec - eh;
        e1 = ec + eh;
    };
    if (bType == 2) {
        f3 ea0, ea1, eb0, eb1;
        edge(bA, cA, axA, hA, n, ea0, ea1);
        edge(bB, cB, axB, hB, -n, eb0, eb1);
        ClosestSegmentSegment(ea0, ea1, eb0, eb1, pA, pB);
    } else if (bType == 1) {
        pB = BoxSupportPoint(cB, qB, hB, -n);
        pA = ClosestPointOnBox(pB, cA, qA, hA);
    } else {
        pA = BoxSupportPoint(cA, qA, hA, n);
        pB = ClosestPointOnBox(pA, cB, qB, hB);
    }
    pen = minPen;
    return pen > 0.0f;
}
// :333-448
void ClosestSegmentBox(f3 sa, f3 sb, f3 bc, f4 bq, f3 h, f3 &outSeg, f3 &outBox, bool &inter)
{
    outSeg = sa;
    outBox = ClosestPointOnBox(sa, bc, bq, h);
    const f3 la = QInvRotate(bq, sa - bc), lb = QInvRotate(bq, sb - bc);
    const f3 d = lb - la;
    // SegmentIntersectsAabbLocal
    inter = true;
    float tMin = 0.0f, tMax = 1.0f;
    for (uint32_t ax = 0; ax < 3 && inter; ++ax) {
        const float o = Comp(la, ax), dl = Comp(d, ax), lo = -Comp(h, ax), hi = Comp(h, ax);
        if (std::fabs(dl) <= kEps) {
            if (o < lo || o > hi) inter = false;
            continue;
        }
        const float inv = 1.0f / dl;
        float t0 = (lo - o) * inv, t1 = (hi - o) * inv;
        if (t0 > t1) std::swap(t0, t1);
        tMin = std::max(tMin, t0);
        tMax = std::min(tMax, t1);
        if (tMin > tMax) inter = false;
    }
    if (inter) {
        outSeg = bc + QRotate(bq, la + d * tMin);
        outBox = outSeg;
        return;
    }
    float bestD2 = 3.402823466e+38f;
    const f3 nh{-h.x, -h.y, -h.z};
    f3 bestSeg = la, bestBox = clamp3(la, nh, h);
    auto cand = [&](float t) {
        if (t < 0.0f || t > 1.0f) return;
        const f3 sp = lerp3(la, lb, t);
        const f3 bp = clamp3(sp, nh, h);
        const float d2 = dot(sp - bp, sp - bp);
        if (d2 < bestD2) { bestD2 = d2; bestSeg = sp; bestBox = bp; }
    };
    cand(0.0f);
    cand(1.0f);
    for (uint32_t ax = 0; ax < 3; ++ax) {
        const float dl = Comp(d, ax);
        if (std::fabs(dl) > kEps) {
            cand((-Comp(h, ax) - Comp(la, ax)) / dl);
            cand((Comp(h, ax) - Comp(la, ax)) / dl);
        }
    }
    outSeg = bc + QRotate(bq, bestSeg);
    outBox = bc + QRotate(bq, bestBox);
}
// :467-518
bool BoxCapsule(f3 bc, f4 bq, f3 h, f3 ca, f3 cb, float cr, f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0, 0, 0};
    pen = 0.0f;
    f3 segP, boxP;
    bool inter = false;
    ClosestSegmentBox(ca, cb, bc, bq, h, segP, boxP, inter);
    if (!inter) {
        const f3 d = segP - boxP;
        const float d2 = dot(d, d);
        if (d2 > cr * cr) return false;
        const float dist = std::sqrt(std::max(d2, 0.0f));
        n = dist > kEps ? d / dist : f3{0, 1, 0};
        pA = boxP;
        pB = segP - n * cr;
        pen = PenetrationFromPoints(pA, pB, n);
        return pen > 0.0f;
    }
    const f3 ls = QInvRotate(bq, segP - bc);
    const f3 lfn = ClosestFaceNormalLocal(ls, h);
    n = QRotate(bq, lfn);
    const float depth = std::min(h.x - std::fabs(ls.x), std::min(h.y - std::fabs(ls.y), h.z - std::fabs(ls.z)));
    pA = bc + QRotate(bq, ls + lfn * depth);
    pB = segP - n * cr;
    pen = PenetrationFromPoints(pA, pB, n);
    return pen > 0.0f;
}
// GenerateRigidContact (:520-641)
bool RigidContactPoints(uint32_t tA, f3 cA, f4 qA, f4 prA, f4 sA, uint32_t tB, f3 cB, f4 qB, f4 prB, f4 sB,
                        f3 &n, f3 &pA, f3 &pB, float &pen)
{
    n = pA = pB = f3{0, 0, 0};
    pen = 0.0f;
    const uint32_t S = CN_COLLIDER_SPHERE, X = CN_COLLIDER_BOX, K = CN_COLLIDER_CAPSULE;
    if (tA == S && tB == S) return SphereSphere(cA, SphereRadius(prA, sA), cB, SphereRadius(prB, sB), n, pA, pB, pen);
    if (tA == S && tB == X) return SphereBox(cA, SphereRadius(prA, sA), cB, qB, BoxHalfExtents(prB, sB), n, pA, pB, pen);
    if (tA == X && tB == S) {
        f3 ns, ps, pb;
        const bool hit = SphereBox(cB, SphereRadius(prB, sB), cA, qA, BoxHalfExtents(prA, sA), ns, ps, pb, pen);
        n = -ns; pA = pb; pB = ps;
        pen = PenetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    if (tA == S && tB == K) {
        f3 b0, b1; float rB = 0.0f;
        CapsuleSegment(cB, qB, prB, sB, b0, b1, rB);
        return SphereCapsule(cA, SphereRadius(prA, sA), b0, b1, rB, n, pA, pB, pen);
    }
    if (tA == K && tB == S) {
        f3 a0, a1; float rA = 0.0f;
        CapsuleSegment(cA, qA, prA, sA, a0, a1, rA);
        f3 ns, ps, pc;
        const bool hit = SphereCapsule(cB, SphereRadius(prB, sB), a0, a1, rA, ns, ps, pc, pen);
        n = -ns; pA = pc; pB = ps;
        pen = PenetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    if (tA == X && tB == X) return BoxBox(cA, qA, BoxHalfExtents(prA, sA), cB, qB, BoxHalfExtents(prB, sB), n, pA, pB, pen);
    if (tA == K && tB == K) {
        f3 a0, a1, b0, b1, ca, cb; float rA = 0.0f, rB = 0.0f;
        CapsuleSegment(cA, qA, prA, sA, a0, a1, rA);
        CapsuleSegment(cB, qB, prB, sB, b0, b1, rB);
        ClosestSegmentSegment(a0, a1, b0, b1, ca, cb);
        return SphereSphere(ca, rA, cb, rB, n, pA, pB, pen);
    }
    if (tA == X && tB == K) {
        f3 b0, b1; float rB = 0.0f;
        CapsuleSegment(cB, qB, prB, sB, b0, b1, rB);
        return BoxCapsule(cA, qA, BoxHalfExtents(prA, sA), b0, b1, rB, n, pA, pB, pen);
    }
    if (tA == K && tB == X) {
        f3 a0, a1; float rA = 0.0f;
        CapsuleSegment(cA, qA, prA, sA, a0, a1, rA);
        f3 nb, pbx, pcap;
        const bool hit = BoxCapsule(cB, qB, BoxHalfExtents(prB, sB), a0, a1, rA, nb, pbx, pcap, pen);
        n = -nb; pA = pcap; pB = pbx;
        pen = PenetrationFromPoints(pA, pB, n);
        return hit && pen > 0.0f;
    }
    return false;
}

// physics_rigid_box_box_manifold.hlsli: face-preferring separating axis, incident face clipped
// against the reference face (or the edge pair, or corner recovery), reduced to <= 4 points.
struct BoxCand { f3 a, b; float pen; };
bool BoxBoxSat(f3 cA, const f3 *axA, f3 hA, f3 cB, const f3 *axB, f3 hB, f3 &nOut, float &penOut, uint32_t &type,
               uint32_t &ia, uint32_t &ib)
{
    nOut = f3{0, 0, 0}; penOut = 0.0f; type = 0; ia = ib = 0;
    const f3 cd = cB - cA;
    auto proj = [](f3 axis, const f3 *ax, f3 h) {
        return h.x * std::fabs(dot(axis, ax[0])) + h.y * std::fabs(dot(axis, ax[1])) + h.z * std::fabs(dot(axis, ax[2]));
    };
    float bestFace = 3.402823466e+38f, bestEdge = 3.402823466e+38f;
    f3 faceAxis{0, 1, 0}, edgeAxis{0, 1, 0};
    uint32_t faceType = 0, faceA = 0, edgeA = 0, edgeB = 0;
    bool hasEdge = false;
    for (uint32_t side = 0; side < 2; ++side)
        for (uint32_t i = 0; i < 3; ++i) {
            f3 n = side == 0 ? axA[i] : axB[i];
            const float ov = proj(n, axA, hA) + proj(n, axB, hB) - std::fabs(dot(cd, n));
            if (ov < 0.0f) return false;
            if (dot(cd, n) < 0.0f) n = -n;
            if (ov < bestFace - 5.0e-4f) { bestFace = ov; faceAxis = n; faceType = side; faceA = i; }
        }
    for (uint32_t a = 0; a < 3; ++a)
        for (uint32_t b = 0; b < 3; ++b) {
            const f3 axis = cross(axA[a], axB[b]);
            const float l2 = dot(axis, axis);
            if (l2 <= kEps) continue;
            hasEdge = true;
            f3 n = axis * (1.0f / std::sqrt(l2));
            const float ov = proj(n, axA, hA) + proj(n, axB, hB) - std::fabs(dot(cd, n));
            if (ov < 0.0f) return false;
            if (dot(cd, n) < 0.0f) n = -n;
            if (ov < bestEdge) { bestEdge = ov; edgeAxis = n; edgeA = a; edgeB = b; }
        }
    if (hasEdge && bestEdge < bestFace * 0.95f - 1.0e-3f) {
        nOut = edgeAxis; penOut = bestEdge; type = 2; ia = edgeA; ib = edgeB;
    } else {
        nOut = faceAxis; penOut = bestFace; type = faceType; ia = faceA; ib = 0;
    }
    return penOut > 0.0f;
}
void InsertBoxCand(f3 pa, f3 pb, float pen, float merge2, std::vector<BoxCand> &cand)
{
    if (pen <= kEps) return;
    const f3 mid = (pa + pb) * 0.5f;
    for (auto &c : cand) {
        const f3 d = (c.a + c.b) * 0.5f - mid;
        if (dot(d, d) <= merge2) {
            if (pen > c.pen) c = BoxCand{pa, pb, pen};
            return;
        }
    }
    if (cand.size() < 16) { cand.push_back(BoxCand{pa, pb, pen}); return; }
    size_t r = 0;
    for (size_t i = 1; i < cand.size(); ++i) if (cand[i].pen < cand[r].pen) r = i;
    if (pen > cand[r].pen) cand[r] = BoxCand{pa, pb, pen};
}
uint32_t ClipPlane(const f3 *in, uint32_t inCount, f3 origin, f3 normal, float offset, bool keepLess, f3 *out)
{
    if (inCount == 0) return 0;
    uint32_t oc = 0;
    f3 prev = in[inCount - 1];
    float prevC = dot(prev - origin, normal);
    bool prevIn = keepLess ? prevC <= offset : prevC >= offset;
    for (uint32_t i = 0; i < inCount && i < 8; ++i) {
        const f3 cur = in[i];
        const float curC = dot(cur - origin, normal);
        const bool curIn = keepLess ? curC <= offset : curC >= offset;
        if (curIn != prevIn) {
            const float den = curC - prevC;
            const float t = std::fabs(den) > kEps ? (offset - prevC) / den : 0.0f;
            if (oc < 8) out[oc++] = lerp3(prev, cur, saturate(t));
        }
        if (curIn && oc < 8) out[oc++] = cur;
        prev = cur; prevC = curC; prevIn = curIn;
    }
    return oc;
}
bool InsideBox(f3 p, f3 c, f4 q, f3 h)
{
    const f3 l = QInvRotate(q, p - c);
    return l.x >= -h.x && l.y >= -h.y && l.z >= -h.z && l.x <= h.x && l.y <= h.y && l.z <= h.z;
}
f3 ProjectInsideAlong(f3 p, f3 c, f4 q, f3 h, f3 dir)
{
    if (!InsideBox(p, c, q, h)) return ClosestPointOnBox(p, c, q, h);
    const f3 lp = QInvRotate(q, p - c);
    const f3 ld = QInvRotate(q, SafeNormalize(dir, f3{0, 1, 0}));
    float bestT = 3.402823466e+38f;
    for (uint32_t ax = 0; ax < 3; ++ax) {
        const float d = Comp(ld, ax);
        if (std::fabs(d) <= kEps) continue;
        const float face = d > 0.0f ? Comp(h, ax) : -Comp(h, ax);
        const float t = (face - Comp(lp, ax)) / d;
        if (t >= 0.0f && t < bestT) bestT = t;
    }
    f3 ls = lp;
    if (bestT < 3.402823466e+37f) ls = lp + ld * bestT;
    else ls = lp + ClosestFaceNormalLocal(lp, h) * std::min(h.x - std::fabs(lp.x), std::min(h.y - std::fabs(lp.y), h.z - std::fabs(lp.z)));
    return c + QRotate(q, ls);
}
uint32_t BoxBoxManifold(f3 cA, f4 qA, f3 hA, f3 cB, f4 qB, f3 hB, f3 nIn, float merge2, float slop, f3 &n,
                        f3 *ptsA, f3 *ptsB, float *pens)
{
    std::vector<BoxCand> cand;
    const f3 axA[3] = {QRotate(qA, f3{1, 0, 0}), QRotate(qA, f3{0, 1, 0}), QRotate(qA, f3{0, 0, 1})};
    const f3 axB[3] = {QRotate(qB, f3{1, 0, 0}), QRotate(qB, f3{0, 1, 0}), QRotate(qB, f3{0, 0, 1})};
    n = SafeNormalize(nIn, f3{0, 1, 0});
    f3 satN; float satPen = 0.0f; uint32_t type = 0, ia = 0, ib = 0;
    const bool sat = BoxBoxSat(cA, axA, hA, cB, axB, hB, satN, satPen, type, ia, ib);
    if (sat) n = SafeNormalize(satN, n);
    auto edge = [](uint32_t axis, f3 c, const f3 *ax, f3 h, f3 dir, f3 &e0, f3 &e1) {
        const uint32_t oa = (axis + 1) % 3, ob = (axis + 2) % 3;
        const float sa = dot(ax[oa], dir) >= 0.0f ? 1.0f : -1.0f;
        const float sb = dot(ax[ob], dir) >= 0.0f ? 1.0f : -1.0f;
        const f3 ec = c + ax[oa] * (Comp(h, oa) * sa) + ax[ob] * (Comp(h, ob) * sb);
        const f3 eh = ax[axis] * Comp(h, axis);
        e0 = ec - eh; e1 = ec + eh;
    };
    if (sat && type == 2) {
        f3 ea0, ea1, eb0, eb1, pa, pb;
        edge(ia, cA, axA, hA, n, ea0, ea1);
        edge(ib, cB, axB, hB, -n, eb0, eb1);
        ClosestSegmentSegment(ea0, ea1, eb0, eb1, pa, pb);
        InsertBoxCand(pa, pb, std::max(satPen, PenetrationFromPoints(pa, pb, n)), merge2, cand);
    }
    if (sat && type < 2) {
        const bool refA = type == 0;
        const f3 *rax = refA ? axA : axB;
        const f3 rc = refA ? cA : cB, rh = refA ? hA : hB;
        const float sign = dot(rax[ia], refA ? n : -n) >= 0.0f ? 1.0f : -1.0f;
        const uint32_t tu = (ia + 1) % 3, tv = (ia + 2) % 3;
        const f3 refN = rax[ia] * sign;
        const f3 refC = rc + refN * Comp(rh, ia);
        const f3 refU = rax[tu], refV = rax[tv];
        const float halfU = Comp(rh, tu), halfV = Comp(rh, tv);
        const f3 *iax = refA ? axB : axA;
        const f3 ic = refA ? cB : cA, ih = refA ? hB : hA;
        uint32_t ii = 0;
        float best = std::fabs(dot(iax[0], refN));
        for (uint32_t i = 1; i < 3; ++i) {
            const float al = std::fabs(dot(iax[i], refN));
            if (al > best) { best = al; ii = i; }
        }
        const float isign = dot(iax[ii], refN) >= 0.0f ? -1.0f : 1.0f;
        const uint32_t iu = (ii + 1) % 3, iv = (ii + 2) % 3;
        const f3 iN = iax[ii] * isign;
        const f3 iC = ic + iN * Comp(ih, ii);
        const f3 du = iax[iu] * Comp(ih, iu), dv = iax[iv] * Comp(ih, iv);
        f3 pA8[8] = {iC + du + dv, iC - du + dv, iC - du - dv, iC + du - dv}, pB8[8];
        uint32_t pc = 4;
        pc = ClipPlane(pA8, pc, refC, refU, halfU, true, pB8);
        pc = ClipPlane(pB8, pc, refC, refU, -halfU, false, pA8);
        pc = ClipPlane(pA8, pc, refC, refV, halfV, true, pB8);
        pc = ClipPlane(pB8, pc, refC, refV, -halfV, false, pA8);
        for (uint32_t i = 0; i < pc && i < 8; ++i) {
            const f3 ip = pA8[i];
            const float sep = dot(ip - refC, refN);
            if (sep > slop) continue;
            const f3 rp = ip - refN * sep;
            const float pen = std::max(0.0f, -sep);
            if (refA) InsertBoxCand(rp, ip, pen, merge2, cand);
            else InsertBoxCand(ip, rp, pen, merge2, cand);
        }
    }
    if (cand.empty()) {
        for (uint32_t k = 0; k < 8; ++k) {
            auto corner = [k](f3 c, f4 q, f3 h) {
                return c + QRotate(q, f3{(k & 1u) ? h.x : -h.x, (k & 2u) ? h.y : -h.y, (k & 4u) ? h.z : -h.z});
            };
            const f3 ca = corner(cA, qA, hA);
            f3 pbA = ClosestPointOnBox(ca, cB, qB, hB);
            if (InsideBox(ca, cB, qB, hB)) pbA = ProjectInsideAlong(ca, cB, qB, hB, -n);
            InsertBoxCand(ca, pbA, PenetrationFromPoints(ca, pbA, n), merge2, cand);
            const f3 cb = corner(cB, qB, hB);
            f3 paB = ClosestPointOnBox(cb, cA, qA, hA);
            if (InsideBox(cb, cA, qA, hA)) paB = ProjectInsideAlong(cb, cA, qA, hA, n);
            InsertBoxCand(paB, cb, PenetrationFromPoints(paB, cb, n), merge2, cand);
        }
    }
    if (cand.empty()) return 0;
    const f3 tx = SafeNormalize(cross(std::fabs(n.y) < 0.9f ? f3{0, 1, 0} : f3{1, 0, 0}, n), f3{1, 0, 0});
    const f3 ty = cross(n, tx);
    const size_t count = cand.size();
    std::vector<float> mu(count), mv(count);
    std::vector<bool> sel(count, false);
    for (size_t i = 0; i < count; ++i) {
        const f3 mid = (cand[i].a + cand[i].b) * 0.5f;
        mu[i] = dot(mid, tx);
        mv[i] = dot(mid, ty);
    }
    const uint32_t target = uint32_t(std::min<size_t>(count, 4));
    size_t deepest = 0;
    for (size_t i = 1; i < count; ++i) if (cand[i].pen > cand[deepest].pen) deepest = i;
    sel[deepest] = true;
    uint32_t out = 0;
    ptsA[out] = cand[deepest].a; ptsB[out] = cand[deepest].b; pens[out++] = cand[deepest].pen;
    while (out < target) {
        size_t bi = 0; float bs = -1.0f; bool found = false;
        for (size_t i = 0; i < count; ++i) {
            if (sel[i]) continue;
            float md = 3.402823466e+38f;
            for (size_t j = 0; j < count; ++j) {
                if (!sel[j]) continue;
                const float du2 = mu[i] - mu[j], dv2 = mv[i] - mv[j];
                md = std::min(md, du2 * du2 + dv2 * dv2);
            }
            const float score = md + cand[i].pen * 1.0e-4f;
            if (score > bs) { bs = score; bi = i; found = true; }
        }
        if (!found) break;
        sel[bi] = true;
        ptsA[out] = cand[bi].a; ptsB[out] = cand[bi].b; pens[out++] = cand[bi].pen;
    }
    return out;
}

// physics_rigid_count_pairs / emit_pairs + generate_contacts: every moving collider against the
// others (a moving partner once, at the higher collider index; a static one always), canonical
// (lower shape type first), then one contact per pair.
void rigidPairsAndContacts(cno_solver &s)
{
    s.rrPairs.clear();
    s.rrContacts.clear();
    const uint32_t C = s.C;
    const uint32_t cap = std::max<uint32_t>(64u, 32u * C); // rigid_body_common.cpp:35-47
    uint32_t required = 0;
    const std::vector<uint32_t> &order = s.colliderQueryOrder;
    for (uint32_t k = 0; k < s.activeMovingCount && order.size() >= 2; ++k) {
        const uint32_t cA = order[k];
        const cn_collider_broadphase &a = s.colBp[cA];
        for (uint32_t cB : order) {
            if (cB == cA) continue;
            const cn_collider_broadphase &b = s.colBp[cB];
            if (b.owner_body == a.owner_body) continue;
            if (s.bodyType[b.owner_body] != CN_BODY_STATIC && cB < cA) continue;
            if (a.environment_index != b.environment_index) continue;
            if ((a.collision_mask & b.collision_layer) == 0u || (b.collision_mask & a.collision_layer) == 0u) continue;
            if (!AabbOverlaps(s.colAabbMin[cA], s.colAabbMax[cA], s.colAabbMin[cB], s.colAabbMax[cB])) continue;
            if (required < cap) s.rrPairs.push_back(a.shape_type > b.shape_type ? std::make_pair(cB, cA) : std::make_pair(cA, cB));
            ++required;
        }
    }
    s.requiredRigidRigidPairs = required;
    s.rrContacts.assign(s.rrPairs.size() * 4, cno_solver::RigidPairContact{});
    const float merge = s.desc.contact.manifold_merge_slop_multiplier * s.slop();
    for (size_t p = 0; p < s.rrPairs.size(); ++p) {
        const auto &pr = s.rrPairs[p];
        cno_solver::RigidPairContact *slot = &s.rrContacts[4 * p];
        const cn_collider_broadphase &bpA = s.colBp[pr.first], &bpB = s.colBp[pr.second];
        const uint32_t bA = bpA.owner_body, bB = bpB.owner_body;
        if (bA >= s.B || bB >= s.B || bA == bB) continue;
        if (s.bodyType[bA] != CN_BODY_DYNAMIC && s.bodyType[bB] != CN_BODY_DYNAMIC) continue;
        const f4 posA = s.predBodyPos[bA], posB = s.predBodyPos[bB];
        const f4 qA = QNormalize(s.predBodyRot[bA]), qB = QNormalize(s.predBodyRot[bB]);
        const cn_collider_geometry &gA = s.colGeo[pr.first], &gB = s.colGeo[pr.second];
        const f4 prmA{gA.shape_params[0], gA.shape_params[1], gA.shape_params[2], gA.shape_params[3]};
        const f4 prmB{gB.shape_params[0], gB.shape_params[1], gB.shape_params[2], gB.shape_params[3]};
        const f4 scA = s.bodyScale[bA], scB = s.bodyScale[bB];
        const f3 mat = CombineContactMaterial(s.colMat[pr.first], s.colMat[pr.second]);
        const f3 cpA = xyz(posA) + QRotate(qA, f3{gA.local_position[0], gA.local_position[1], gA.local_position[2]} * xyz(scA));
        const f3 cpB = xyz(posB) + QRotate(qB, f3{gB.local_position[0], gB.local_position[1], gB.local_position[2]} * xyz(scB));
        const f4 cqA = QNormalize(QMul(qA, QNormalize(f4{gA.local_orientation[0], gA.local_orientation[1], gA.local_orientation[2], gA.local_orientation[3]})));
        const f4 cqB = QNormalize(QMul(qB, QNormalize(f4{gB.local_orientation[0], gB.local_orientation[1], gB.local_orientation[2], gB.local_orientation[3]})));
        f3 a0, a1, b0, b1;
        ComputeBodyAabb(bpA.shape_type, cpA, cqA, prmA, scA, a0, a1);
        ComputeBodyAabb(bpB.shape_type, cpB, cqB, prmB, scB, b0, b1);
        if (!AabbOverlaps(a0, a1, b0, b1)) continue;
        auto write = [&](uint32_t k, f3 n, float pen, f3 pa, f3 pb) {
            cno_solver::RigidPairContact c;
            c.bodyA = bA; c.bodyB = bB; c.active = true;
            c.normalPenetration = mk4(n, pen);
            c.material = mk4(mat, 0.0f);
            c.localA = mk4(QInvRotate(qA, pa - xyz(posA)), 1.0f);
            c.localB = mk4(QInvRotate(qB, pb - xyz(posB)), 1.0f);
            slot[k] = c;
        };
        if (bpA.shape_type == CN_COLLIDER_BOX && bpB.shape_type == CN_COLLIDER_BOX) {
            const f3 hA = BoxHalfExtents(prmA, scA), hB = BoxHalfExtents(prmB, scB);
            const f3 axA[3] = {QRotate(cqA, f3{1, 0, 0}), QRotate(cqA, f3{0, 1, 0}), QRotate(cqA, f3{0, 0, 1})};
            const f3 axB[3] = {QRotate(cqB, f3{1, 0, 0}), QRotate(cqB, f3{0, 1, 0}), QRotate(cqB, f3{0, 0, 1})};
            f3 satN; float satPen = 0.0f; uint32_t t0, t1, t2;
            if (!BoxBoxSat(cpA, axA, hA, cpB, axB, hB, satN, satPen, t0, t1, t2)) continue;
            f3 pa[4], pb[4], n; float pens[4];
            const uint32_t m = BoxBoxManifold(cpA, cqA, hA, cpB, cqB, hB, SafeNormalize(satN, f3{0, 1, 0}), merge * merge,
                                              s.slop(), n, pa, pb, pens);
            if (m > 0) {
                for (uint32_t k = 0; k < m; ++k) write(k, n, pens[k], pa[k], pb[k]);
                continue;
            }
        }
        f3 n, pa, pb;
        float pen = 0.0f;
        if (!RigidContactPoints(bpA.shape_type, cpA, cqA, prmA, scA, bpB.shape_type, cpB, cqB, prmB, scB, n, pa, pb, pen) ||
            pen <= 0.0f) continue;
        write(0, SafeNormalize(n, f3{0, 1, 0}), pen, pa, pb);
    }
}

// physics_rigid_generate_proxy_contacts.cs.hlsl:30-183: every candidate of a proxy particle
// (proxies lead the particle order, so their candidates open the list) gets a contact after the
// pair contacts -- the deepest between the proxy sphere of body A and the candidate body B's
// enabled colliders, framed without the body scale (ComposeColliderWorldPosition) -- or an
// inactive one; at most max(64, 8 x proxies) of them.
void proxyRigidContacts(cno_solver &s)
{
    uint32_t proxyCands = 0;
    while (proxyCands < s.rigidPairs.size() && s.rigidPairs[proxyCands].first < s.nProxy) ++proxyCands;
    const uint32_t cap = std::max<uint32_t>(
        64u, (s.desc.particle_rigid_pairs_per_particle ? s.desc.particle_rigid_pairs_per_particle : 8u) * s.nProxy);
    const uint32_t used = std::min(proxyCands, cap);
    s.requiredProxyContacts = proxyCands;
    s.proxyContactSlots = used;
    for (uint32_t k = 0; k < used; ++k) {
        cno_solver::RigidPairContact out;
        const uint32_t p = s.rigidPairs[k].first, bB = s.rigidPairs[k].second;
        const uint32_t bA = s.ownerIdx[p];
        const f4 posA = s.predBodyPos[bA], posB = s.predBodyPos[bB];
        if (bA == bB || (posA.w <= kEps && posB.w <= kEps)) {
            s.rrContacts.push_back(out);
            continue;
        }
        const f3 sc = xyz(s.x[p]);
        const float sr = s.radii[p];
        const f4 qA = QNormalize(s.predBodyRot[bA]), qB = QNormalize(s.predBodyRot[bB]);
        const f4 scB = s.bodyScale[bB];
        float best = 0.0f;
        f3 bestN{0, 1, 0}, bestA{0, 0, 0}, bestB{0, 0, 0}, bestMat{0, 0, 0};
        const uint32_t off = s.bodyColRanges[2 * bB], cnt = s.bodyColRanges[2 * bB + 1];
        for (uint32_t i = 0; i < kColliderCap && i < cnt; ++i) {
            const uint32_t c = s.bodyColIdx[off + i];
            const cn_collider_broadphase &bp = s.colBp[c];
            if (bp.enabled_flag == 0u) continue;
            const cn_collider_geometry &g = s.colGeo[c];
            const f3 cwp = xyz(posB) + QRotate(qB, f3{g.local_position[0], g.local_position[1], g.local_position[2]});
            const f4 cwq = QNormalize(QMul(qB, QNormalize(f4{g.local_orientation[0], g.local_orientation[1],
                                                             g.local_orientation[2], g.local_orientation[3]})));
            const f4 prm{g.shape_params[0], g.shape_params[1], g.shape_params[2], g.shape_params[3]};
            f3 n, pa, pb;
            float pen = 0.0f;
            bool hit;
            if (bp.shape_type == CN_COLLIDER_SPHERE) {
                hit = SphereSphere(sc, sr, cwp, SphereRadius(prm, scB), n, pa, pb, pen);
            } else if (bp.shape_type == CN_COLLIDER_BOX) {
                hit = SphereBox(sc, sr, cwp, cwq, BoxHalfExtents(prm, scB), n, pa, pb, pen);
            } else {
                f3 ca, cb;
                float capR = 0.0f;
                CapsuleSegment(cwp, cwq, prm, scB, ca, cb, capR);
                hit = SphereCapsule(sc, sr, ca, cb, capR, n, pa, pb, pen);
            }
            if (!hit || pen <= best) continue;
            best = pen;
            bestN = SafeNormalize(n, f3{0, 1, 0});
            bestA = pa;
            bestB = pb;
            bestMat = CombineContactMaterial(s.bodyProxyMat[bA], s.colMat[c]);
        }
        if (best > 0.0f) {
            out.bodyA = bA; out.bodyB = bB; out.active = true;
            out.normalPenetration = mk4(bestN, best);
            out.localA = mk4(QInvRotate(qA, bestA - xyz(posA)), 0.0f);
            out.localB = mk4(QInvRotate(qB, bestB - xyz(posB)), 0.0f);
            out.material = mk4(bestMat, 0.0f);
        }
        s.rrContacts.push_back(out);
    }
}

// physics_rigid_init_contact_velocities.cs.hlsl: canonical contacts grouped by body pair (pair
// order within a group, at most 16), each with its restitution target.
void rigidVelocityInit(cno_solver &s)
{
    s.rrGroups.clear();
    s.rrGroupBodies.clear();
    std::vector<std::pair<uint64_t, uint32_t>> keyed;
    for (uint32_t p = 0; p < s.rrContacts.size(); ++p) {
        const auto &c = s.rrContacts[p];
        if (!c.active) continue;
        keyed.push_back({uint64_t(std::min(c.bodyA, c.bodyB)) * s.B + std::max(c.bodyA, c.bodyB), p});
    }
    std::stable_sort(keyed.begin(), keyed.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
    const float thr = s.desc.contact.rigid_restitution_velocity_threshold;
    for (size_t j = 0; j < keyed.size(); ++j) {
        if (j == 0 || keyed[j].first != keyed[j - 1].first) {
            s.rrGroups.emplace_back();
            const auto &c = s.rrContacts[keyed[j].second];
            s.rrGroupBodies.push_back({std::min(c.bodyA, c.bodyB), std::max(c.bodyA, c.bodyB)});
        }
        if (s.rrGroups.back().size() >= 16u) continue;
        auto c = s.rrContacts[keyed[j].second];
        if (c.bodyA > c.bodyB) {
            std::swap(c.bodyA, c.bodyB);
            c.normalPenetration = mk4(-xyz(c.normalPenetration), c.normalPenetration.w);
            std::swap(c.localA, c.localB);
        }
        cno_solver::RigidSlot sl;
        const f3 nrm = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
        sl.normal = mk4(nrm, saturate(c.material.x));
        sl.localA = mk4(xyz(c.localA), saturate(c.material.z));
        sl.localB = c.localB;
        sl.state = f4{0, 0, 0, 0};
        const f4 pA = s.predBodyPos[c.bodyA], pB = s.predBodyPos[c.bodyB];
        const f4 oA = QNormalize(s.predBodyRot[c.bodyA]), oB = QNormalize(s.predBodyRot[c.bodyB]);
        const f3 rA = (xyz(pA) + QRotate(oA, xyz(c.localA))) - xyz(pA);
        const f3 rB = (xyz(pB) + QRotate(oB, xyz(c.localB))) - xyz(pB);
        const f3 vA = xyz(s.predBodyLin[c.bodyA]) + cross(xyz(s.predBodyAng[c.bodyA]), rA);
        const f3 vB = xyz(s.predBodyLin[c.bodyB]) + cross(xyz(s.predBodyAng[c.bodyB]), rB);
        const float nv = dot(vB - vA, nrm);
        if (nv < -thr) sl.state.y = -saturate(c.material.y) * nv;
        s.rrGroups.back().push_back(sl);
    }
}

// physics_rigid_depenetrate_contacts.cs.hlsl:22-137 (summed in pair order)
void rigidDepenetration(cno_solver &s)
{
    const float slop = s.slop(), baum = s.desc.rigid.depenetration_baumgarte;
    const float maxC = s.desc.rigid.depenetration_max_correction_per_iteration;
    const float relax = s.desc.rigid.depenetration_relaxation;
    const float minFric = s.desc.contact.position_friction_min_distance;
    for (const auto &c : s.rrContacts) {
        if (!c.active) continue;
        const uint32_t bA = c.bodyA, bB = c.bodyB;
        const f4 pA0 = s.predBodyPos[bA], pB0 = s.predBodyPos[bB];
        const bool dA = s.bodyType[bA] == CN_BODY_DYNAMIC, dB = s.bodyType[bB] == CN_BODY_DYNAMIC;
        const float iA = dA ? pA0.w : 0.0f, iB = dB ? pB0.w : 0.0f;
        if (iA == 0.0f && iB == 0.0f) continue;
        const f4 qA = QNormalize(s.predBodyRot[bA]), qB = QNormalize(s.predBodyRot[bB]);
        const f4 pqA = QNormalize(s.prevBodyRot[bA]), pqB = QNormalize(s.prevBodyRot[bB]);
        f3 inA = xyz(s.bodyInvInertia[bA]), inB = xyz(s.bodyInvInertia[bB]);
        if (iA == 0.0f) inA = f3{0, 0, 0};
        if (iB == 0.0f) inB = f3{0, 0, 0};
        const f3 ptA = xyz(pA0) + QRotate(qA, xyz(c.localA)), ptB = xyz(pB0) + QRotate(qB, xyz(c.localB));
        const f3 ppA = xyz(s.prevBodyPos[bA]) + QRotate(pqA, xyz(c.localA));
        const f3 ppB = xyz(s.prevBodyPos[bB]) + QRotate(pqB, xyz(c.localB));
        const f3 n = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
        const float raw = std::max(-dot(ptB - ptA, n) - slop, 0.0f);
        const float pen = std::min(raw * baum, maxC);
        if (pen <= 0.0f) continue;
        const f3 rA = ptA - xyz(pA0), rB = ptB - xyz(pB0);
        const float den = ContactEffectiveMass(iA, inA, qA, rA, n) + ContactEffectiveMass(iB, inB, qB, rB, n);
        if (den <= kEps) continue;
        const float lambda = (pen / den) * relax;
        f3 tA = -n * (iA * lambda);
        f3 rotA = -MulWorldInvInertia(inA, qA, cross(rA, n)) * lambda;
        f3 tB = n * (iB * lambda);
        f3 rotB = MulWorldInvInertia(inB, qB, cross(rB, n)) * lambda;
        const f3 rel = (ptB - ppB) - (ptA - ppA);
        const f3 fd = PositionFrictionDelta(ProjectOntoTangent(rel, n), pen, saturate(c.material.x), saturate(c.material.z), minFric);
        const float fdist = length(fd);
        if (fdist > 0.0f) {
            const f3 t = fd / fdist;
            const float tden = ContactEffectiveMass(iA, inA, qA, rA, t) + ContactEffectiveMass(iB, inB, qB, rB, t);
            if (tden > kEps) {
                const float tl = (fdist / tden) * relax;
                tA += t * (iA * tl);
                rotA += MulWorldInvInertia(inA, qA, cross(rA, t)) * tl;
                tB -= t * (iB * tl);
                rotB -= MulWorldInvInertia(inB, qB, cross(rB, t)) * tl;
            }
        }
        if (dA && iA != 0.0f) { s.bodyTransCorr[bA] += tA; s.bodyRotCorr[bA] += rotA; }
        if (dB && iB != 0.0f) { s.bodyTransCorr[bB] += tB; s.bodyRotCorr[bB] += rotB; }
    }
}

// physics_rigid_solve_contact_velocities.cs.hlsl (one group at a time, the velocity change of
// each group summed into the bodies' corrections)
void rigidSolveVelocities(cno_solver &s)
{
    const float slop = s.slop(), stiff = s.desc.rigid.velocity_penetration_stiffness;
    for (size_t g = 0; g < s.rrGroups.size(); ++g) {
        auto &slots = s.rrGroups[g];
        const uint32_t bA = s.rrGroupBodies[g].first, bB = s.rrGroupBodies[g].second;
        const f4 pA = s.predBodyPos[bA], pB = s.predBodyPos[bB];
        const float iA = s.bodyType[bA] == CN_BODY_DYNAMIC ? pA.w : 0.0f;
        const float iB = s.bodyType[bB] == CN_BODY_DYNAMIC ? pB.w : 0.0f;
        if (iA == 0.0f && iB == 0.0f) continue;
        const f4 oA = QNormalize(s.predBodyRot[bA]), oB = QNormalize(s.predBodyRot[bB]);
        f3 inA = xyz(s.bodyInvInertia[bA]), inB = xyz(s.bodyInvInertia[bB]);
        if (iA == 0.0f) inA = f3{0, 0, 0};
        if (iB == 0.0f) inB = f3{0, 0, 0};
        const f3 lA0 = xyz(s.predBodyLin[bA]), lB0 = xyz(s.predBodyLin[bB]);
        const f3 aA0 = xyz(s.predBodyAng[bA]), aB0 = xyz(s.predBodyAng[bB]);
        f3 lA = lA0, lB = lB0, aA = aA0, aB = aB0;
        for (uint32_t pass = 0; pass < 2; ++pass) {
            for (auto &sl : slots) {
                const bool hasRest = sl.state.y > 0.0f;
                if ((pass == 0 && hasRest) || (pass == 1 && !hasRest)) continue;
                const f3 n = SafeNormalize(xyz(sl.normal), f3{0, 1, 0});
                const f3 ptA = xyz(pA) + QRotate(oA, xyz(sl.localA)), ptB = xyz(pB) + QRotate(oB, xyz(sl.localB));
                const f3 rA = ptA - xyz(pA), rB = ptB - xyz(pB);
                const float nv = dot((lB + cross(aB, rB)) - (lA + cross(aA, rA)), n);
                const float pen = std::max(PenetrationFromPoints(ptA, ptB, n) - slop, 0.0f);
                const float nd = ContactEffectiveMass(iA, inA, oA, rA, n) + ContactEffectiveMass(iB, inB, oB, rB, n);
                if (nd <= kEps) continue;
                float vi = (sl.state.y - nv) / nd;
                if (vi < -sl.state.x) vi = -sl.state.x;
                const float pi = pen > 0.0f ? (stiff * pen) / nd : 0.0f;
                const float applied = vi + pi;
                sl.state.x = sl.state.x + applied;
                if (std::fabs(applied) > kEps) {
                    const f3 imp = n * applied;
                    if (iA > kEps) { lA += -imp * iA; aA += MulWorldInvInertia(inA, oA, cross(rA, -imp)); }
                    if (iB > kEps) { lB += imp * iB; aB += MulWorldInvInertia(inB, oB, cross(rB, imp)); }
                }
                const float kf = saturate(sl.normal.w), sf = saturate(sl.localA.w);
                const f3 tv = ProjectOntoTangent((lB + cross(aB, rB)) - (lA + cross(aA, rA)), n);
                const float ts = length(tv);
                if (ts > 1.0e-5f) {
                    const f3 t = tv / ts;
                    const float td = ContactEffectiveMass(iA, inA, oA, rA, t) + ContactEffectiveMass(iB, inB, oB, rB, t);
                    if (td > kEps) {
                        const float raw = -dot(tv, t) / td;
                        const float old = sl.state.z;
                        const float maxS = sf * sl.state.x, maxD = kf * sl.state.x;
                        const float un = old + raw;
                        float acc = un;
                        if (std::fabs(un) > maxS) acc = std::min(std::max(un, -maxD), maxD);
                        const float at = acc - old;
                        sl.state.z = acc;
                        if (std::fabs(at) > kEps) {
                            const f3 ti = t * at;
                            if (iA > kEps) { lA += -ti * iA; aA += MulWorldInvInertia(inA, oA, cross(rA, -ti)); }
                            if (iB > kEps) { lB += ti * iB; aB += MulWorldInvInertia(inB, oB, cross(rB, ti)); }
                        }
                    }
                }
            }
        }
        if (iA > kEps) { s.bodyLinVelCorr[bA] += lA - lA0; s.bodyAngVelCorr[bA] += aA - aA0; }
        if (iB > kEps) { s.bodyLinVelCorr[bB] += lB - lB0; s.bodyAngVelCorr[bB] += aB - aB0; }
    }
}

// physics_rigid_apply_contact_velocities.cs.hlsl:14-58
void applyRigidContactVelocities(cno_solver &s)
{
    for (uint32_t b = 0; b < s.B; ++b) {
        if (s.bodyType[b] == CN_BODY_DYNAMIC) {
            const f3 lc = ClampLength(s.bodyLinVelCorr[b], s.desc.rigid.max_linear_velocity_correction_per_iteration);
            const f3 ac = ClampLength(s.bodyAngVelCorr[b], s.desc.rigid.max_angular_velocity_correction_per_iteration);
            s.predBodyLin[b] = mk4(xyz(s.predBodyLin[b]) + lc, s.predBodyLin[b].w);
            s.predBodyAng[b] = mk4(xyz(s.predBodyAng[b]) + ac, s.predBodyAng[b].w);
        }
        s.bodyLinVelCorr[b] = f3{0, 0, 0};
        s.bodyAngVelCorr[b] = f3{0, 0, 0};
    }
}

// physics_particle_apply_position_corrections.cs.hlsl:8-30
void applyPositionCorrections(cno_solver &s)
{
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f3 c = xyz(s.posCorr[i]);
        s.posCorr[i] = f4{0, 0, 0, 0};
        const f4 p = s.x[i];
        if (p.w <= kEps) continue;
        s.x[i] = mk4(xyz(p) + c, p.w);
    }
}

// physics_particle_update_velocities.cs.hlsl:13-44
void updateVelocities(cno_solver &s, float dt)
{
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        const f4 p = s.x[i];
        if (p.w <= kEps || dt <= kEps) { s.v[i] = f4{0, 0, 0, 0}; continue; }
        const f3 pp = xyz(s.xprev[i]);
        f3 pos = xyz(p);
        if (s.kinds[i] == CN_PARTICLE_FLUID) {
            pos += xyz(s.fluidDelta[i]);
            s.x[i] = mk4(pos, p.w);
            s.fluidDelta[i] = f4{0, 0, 0, 0};
        }
        const float damping = std::max(s.contactMaterials[s.matIdx[i]].z, 0.0f);
        const float ds = std::max(1.0f - damping * dt, 0.0f);
        s.v[i] = mk4(((pos - pp) / dt) * ds, 0.0f);
    }
}

// physics_fluid_project_boundary_velocities.cs.hlsl:24-117
void projectFluidBoundaryVelocities(cno_solver &s, float dt)
{
    const float slop = s.slop();
    const float minFric = s.desc.contact.position_friction_min_distance;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(s.N); ++ii) {
        const uint32_t i = uint32_t(ii);
        if (s.kinds[i] != CN_PARTICLE_FLUID) continue;
        const f3 pos = xyz(s.x[i]);
        const float pr = std::max(s.radii[i], 0.0f);
        f3 vel = xyz(s.v[i]);
        const f4 pm = s.contactMaterials[s.matIdx[i]];
        const float pd = std::max(pm.z, 0.0f);
        float bestD = 3.402823466e+38f;
        f3 bestN{0, 1, 0}, bestMat{0, 0, 0};
        bool found = false;
        for (uint32_t c : s.boundaryCand[i]) {
            float sd = 0.0f;
            f3 n{0, 1, 0};
            if (!FluidBoundaryContactInfo(s, c, pos, sd, n)) continue;
            const float cd = pr + 2.0f * slop;
            if (sd > cd) continue;
            if (sd < bestD) {
                bestD = sd; bestN = n;
                bestMat = CombineContactMaterial(pm, s.colMat[c]);
                found = true;
            }
        }
        if (!found) continue;
        const float pen = std::max(pr - bestD, 0.0f);
        const float cd = std::max(pr + 2.0f * slop, 1.0e-5f);
        const float cw = saturate((cd - bestD) / cd);
        f3 rv = vel;
        const float nv = dot(rv, bestN);
        if (nv < 0.0f) rv -= bestN * nv;
        f3 tv = ProjectOntoTangent(rv, bestN);
        if (dt > kEps) {
            const f3 tdisp = tv * dt;
            const float p2 = std::max(pen, slop);
            f3 fd{0, 0, 0};
            const float td = length(tdisp);
            if (!(td <= minFric || p2 <= kEps)) {
                const float sl = saturate(bestMat.z) * p2;
                if (td <= sl) fd = tdisp;
                else fd = tdisp * std::min(saturate(bestMat.x) * p2 / td, 1.0f);
            }
            tv -= fd / dt;
        }
        const float tds = std::max(1.0f - pd * cw * dt, 0.0f);
        tv = tv * tds;
        rv = bestN * std::max(dot(rv, bestN), 0.0f) + tv;
        s.v[i] = mk4(rv, 0.0f);
    }
}

// physics_particle_rigid_solve_contact_velocities.cs.hlsl + apply_contact_velocities.cs.hlsl,
// repeated softContactIterations times (physics_pass_dispatcher.cpp:3338-3410).
void particleRigidContactVelocities(cno_solver &s, uint32_t iterations)
{
    const float rvt = s.desc.contact.restitution_velocity_threshold;
    const float rpt = s.desc.contact.restitution_penetration_slop_multiplier * s.slop();
    for (uint32_t it = 0; it < iterations; ++it) {
        for (const RigidContact &c : s.activeRigidContacts) {
            const uint32_t i = c.particle, b = c.body;
            const float iS = s.x[i].w;
            const f3 sv = xyz(s.v[i]);
            const f4 rp = s.predBodyPos[b];
            const float iR = s.bodyType[b] == CN_BODY_DYNAMIC ? rp.w : 0.0f;
            if (iS <= kEps && iR <= kEps) continue;
            const f4 rq = QNormalize(s.predBodyRot[b]);
            const f3 rl = xyz(s.predBodyLin[b]), ra = xyz(s.predBodyAng[b]);
            const f3 inI = xyz(s.bodyInvInertia[b]);
            const f3 n = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
            const f3 cp = xyz(rp) + QRotate(rq, xyz(c.rigidLocalPoint));
            const f3 rR = cp - xyz(rp);
            const f3 rcv = rl + cross(ra, rR);
            const f3 rel = sv - rcv;
            const float nv = dot(rel, n);
            if (nv >= 0.0f) continue;
            const float rnd = ContactEffectiveMass(iR, inI, rq, rR, n);
            const float nd = iS + rnd;
            if (nd <= kEps) continue;
            const f3 mat = CombineContactMaterial(s.contactMaterials[s.matIdx[i]], s.colMat[c.collider]);
            const bool er = (-nv > rvt) && (c.normalPenetration.w <= rpt);
            const float rest = er ? saturate(mat.y) : 0.0f;
            const float dnv = er ? (-rest * nv) : 0.0f;
            const float imp = std::max(0.0f, (dnv - nv) / nd);
            const f3 ti = n * imp;
            if (iS > kEps) s.velCorr[i] = mk4(xyz(s.velCorr[i]) + ti * iS, s.velCorr[i].w);
            if (iR > kEps) { // float atomics in the reference; summed here in contact order
                s.bodyLinVelCorr[b] += -ti * iR;
                s.bodyAngVelCorr[b] += MulWorldInvInertia(inI, rq, cross(rR, -ti));
            }
        }
        for (uint32_t i = 0; i < s.N; ++i) {
            f4 vel = s.v[i];
            const float im = s.x[i].w;
            const f3 c = xyz(s.velCorr[i]);
            if (im > kEps) vel = mk4(xyz(vel) + c, vel.w);
            s.v[i] = vel;
            s.velCorr[i] = f4{0, 0, 0, 0};
        }
        if (s.hasDynamic) applyRigidContactVelocities(s);
    }
}

// physics_particle_solve_contact_velocities.cs.hlsl (non-proxy branch) +
// apply_contact_velocities.cs.hlsl, repeated softContactIterations times
// (physics_pass_dispatcher.cpp:3201-3273).
void particleContactVelocities(cno_solver &s, uint32_t iterations)
{
    const float rvt = s.desc.contact.restitution_velocity_threshold;
    const float rpt = s.desc.contact.restitution_penetration_slop_multiplier * s.slop();
    for (uint32_t it = 0; it < iterations; ++it) {
        for (const ParticleContact &c : s.activeParticleContacts) {
            float iA = s.x[c.a].w, iB = s.x[c.b].w;
            f3 vA = xyz(s.v[c.a]), vB = xyz(s.v[c.b]);
            const bool proxyA = c.a < s.nProxy, proxyB = c.b < s.nProxy;
            f3 rA{0, 0, 0}, rB{0, 0, 0}, inA{0, 0, 0}, inB{0, 0, 0};
            f4 qA{0, 0, 0, 1}, qB{0, 0, 0, 1};
            uint32_t bA = 0, bB = 0;
            // a proxy moves with its body (ComputeContactPointVelocity at the proxy's lever arm)
            auto proxySide = [&](uint32_t p, uint32_t &b, float &im, f3 &inv, f4 &q, f3 &vel, f3 &r) {
                b = s.ownerIdx[p];
                const f4 bp = s.predBodyPos[b];
                q = QNormalize(s.predBodyRot[b]);
                im = s.bodyType[b] == CN_BODY_DYNAMIC ? bp.w : 0.0f;
                inv = im > kEps ? xyz(s.bodyInvInertia[b]) : f3{0, 0, 0};
                r = QRotate(q, xyz(s.proxyLocal[p]));
                vel = xyz(s.predBodyLin[b]) + cross(xyz(s.predBodyAng[b]), r);
            };
            if (proxyA) proxySide(c.a, bA, iA, inA, qA, vA, rA);
            if (proxyB) proxySide(c.b, bB, iB, inB, qB, vB, rB);
            if (iA <= kEps && iB <= kEps) continue;
            const f3 n = SafeNormalize(xyz(c.normalPenetration), f3{0, 1, 0});
            const f3 rel = vB - vA;
            const float nv = dot(rel, n);
            if (nv >= 0.0f) continue;
            const float nmA = proxyA ? ContactEffectiveMass(iA, inA, qA, rA, n) : iA;
            const float nmB = proxyB ? ContactEffectiveMass(iB, inB, qB, rB, n) : iB;
            const float denom = nmA + nmB;
            if (denom <= kEps) continue;
            const f3 mat = xyz(c.material);
            const bool er = (-nv > rvt) && (c.normalPenetration.w <= rpt);
            const float rest = er ? saturate(mat.y) : 0.0f;
            const float dnv = er ? (-rest * nv) : 0.0f;
            const float imp = std::max(0.0f, (dnv - nv) / denom);
            const f3 ti = n * imp;
            if (!proxyA && iA > kEps) s.velCorr[c.a] = mk4(xyz(s.velCorr[c.a]) + (-ti * iA), s.velCorr[c.a].w);
            if (!proxyB && iB > kEps) s.velCorr[c.b] = mk4(xyz(s.velCorr[c.b]) + ti * iB, s.velCorr[c.b].w);
            if (proxyA && iA > kEps) {
                s.bodyLinVelCorr[bA] = s.bodyLinVelCorr[bA] + (-ti * iA);
                s.bodyAngVelCorr[bA] = s.bodyAngVelCorr[bA] + MulWorldInvInertia(inA, qA, cross(rA, -ti));
            }
            if (proxyB && iB > kEps) {
                s.bodyLinVelCorr[bB] = s.bodyLinVelCorr[bB] + ti * iB;
                s.bodyAngVelCorr[bB] = s.bodyAngVelCorr[bB] + MulWorldInvInertia(inB, qB, cross(rB, ti));
            }
        }
        for (uint32_t i = 0; i < s.N; ++i) {
            f4 vel = s.v[i];
            const float im = s.x[i].w;
            const f3 c = xyz(s.velCorr[i]);
            if (im > kEps) vel = mk4(xyz(vel) + c, vel.w);
            s.v[i] = vel;
            s.velCorr[i] = f4{0, 0, 0, 0};
        }
        // the bodies' sums after every iteration (solveParticleContactVelocities,
        // physics_pass_dispatcher.cpp:3255-3270); only proxies of dynamic bodies add to them
        if (s.hasDynamic && s.nProxy) applyRigidContactVelocities(s);
    }
}

uint32_t resolveIter(uint32_t o, uint32_t d) { return o > 0u ? o : d; }

void stepFrame(cno_solver &s, float frameDt)
{
    const cn_solver_desc &d = s.desc;
    const uint32_t substeps = std::max<uint32_t>(d.substeps, 1u);
    const uint32_t defIt = std::max<uint32_t>(d.default_iterations, 1u);
    const uint32_t fluidIt = resolveIter(d.fluid_iterations, defIt);
    const uint32_t softIt = resolveIter(d.soft_internal_iterations, defIt);
    const uint32_t contactIt = resolveIter(d.soft_contact_iterations, defIt);
    const uint32_t jointIt = resolveIter(d.rigid_joint_iterations, defIt);
    const uint32_t rrIt = resolveIter(d.rigid_rigid_contact_iterations, defIt);
    const uint32_t maxIt = std::max(std::max(std::max(fluidIt, softIt), contactIt), std::max(jointIt, rrIt));
    const float dt = frameDt / float(substeps);
    uint32_t fluidCount = 0;
    for (uint32_t k : s.kinds) fluidCount += k == CN_PARTICLE_FLUID ? 1u : 0u;
    const uint32_t N = s.N;

    for (uint32_t sub = 0; sub < substeps; ++sub) {
        // physics_solver.cpp:472-496 gating flags
        const bool hasFluidWork = fluidCount > 0 && N > 0;
        const bool hasSoftInternal = N > 0 && (!s.edges.empty() || !s.bends.empty() ||
                                               !s.dihedrals.empty() || !s.tets.empty() ||
                                               !s.segs.empty() || !s.joints.empty() || !s.dists.empty());
        const bool hasSoftSoftContact = contactIt > 0 && N > 1;
        const bool hasRigidCand = N > 0 && s.C > 0;
        const bool hasSoftRigidContact = contactIt > 0 && hasRigidCand;
        const bool hasBroadphase = hasSoftSoftContact || hasFluidWork || hasRigidCand;

        predictRigid(s, dt);
        // useInitialRigidContactSolve (physics_solver.cpp:512-514) where a body can move
        const bool rigidRigid = s.hasDynamic && rrIt > 0 &&
                                ((s.colliderQueryOrder.size() >= 2 && s.activeMovingCount > 0) || (s.nProxy > 0 && s.C > 0));
        if (rigidRigid) rigidPairsAndContacts(s);
        predictSoft(s, dt);
        syncRigidProxies(s);
        if (hasBroadphase) broadphase(s);
        s.particlePairs.clear();
        s.rigidPairs.clear();
        s.requiredParticlePairs = s.requiredRigidPairs = 0;
        if (N > 0) {
            if (hasSoftSoftContact) buildParticleParticleCandidates(s);
            if (hasRigidCand) buildParticleRigidCandidates(s);
            if (hasFluidWork && s.C > 0) buildFluidBoundaryCandidates(s);
        }
        if (rigidRigid && s.nProxy > 0 && hasRigidCand) proxyRigidContacts(s);
        if (rigidRigid) rigidVelocityInit(s);
        // clearSoftConstraintState (physics_clear_soft_constraint_state.cs.hlsl:14-54)
        std::fill(s.posCorr.begin(), s.posCorr.end(), f4{0, 0, 0, 0});
        std::fill(s.velCorr.begin(), s.velCorr.end(), f4{0, 0, 0, 0});
        std::fill(s.edgeLambda.begin(), s.edgeLambda.end(), 0.0f);
        std::fill(s.bendLambda.begin(), s.bendLambda.end(), 0.0f);
        std::fill(s.tetLambda.begin(), s.tetLambda.end(), 0.0f);
        std::fill(s.distLambda.begin(), s.distLambda.end(), 0.0f);
        std::fill(s.segLambda.begin(), s.segLambda.end(), f4{0, 0, 0, 0});
        std::fill(s.jointLambda.begin(), s.jointLambda.end(), f4{0, 0, 0, 0});
        // clearRigidCorrections (physics_rigid_clear_corrections.cs.hlsl)
        std::fill(s.bodyTransCorr.begin(), s.bodyTransCorr.end(), f3{0, 0, 0});
        std::fill(s.bodyRotCorr.begin(), s.bodyRotCorr.end(), f3{0, 0, 0});
        std::fill(s.bodyLinVelCorr.begin(), s.bodyLinVelCorr.end(), f3{0, 0, 0});
        std::fill(s.bodyAngVelCorr.begin(), s.bodyAngVelCorr.end(), f3{0, 0, 0});

        for (uint32_t it = 0; it < maxIt; ++it) {
            const bool runSoft = hasSoftInternal && it < softIt;
            const bool runContacts = hasSoftSoftContact && it < contactIt;
            const bool runRigid = hasSoftRigidContact && it < contactIt;
            const bool runFluid = hasFluidWork && it < fluidIt;
            if (runFluid) {
                buildFluidNeighbors(s, it);
                fluidDensity(s, it);
                fluidDeltaPositions(s, it, dt);
                fluidApplyAndClamp(s, it);
            }
            if (runSoft && s.desc.soft.xpbd_schedule != CN_XPBD_GATHER) {
                colouredSoftIteration(s, dt);
            } else if (runSoft) {
                solveEdges(s, dt);
                applyPairCorrections(s, s.edgeRanges, s.edgeInc, s.edgeCorr);
                solveSegments(s, dt);
                applySegments(s);
                solveBends(s, dt);
                solveDihedrals(s, dt);
                applyQuadCorrections(s, s.bendRanges, s.bendInc, s.bendCorr);
                solveJoints(s, dt);
                applyJoints(s);
                solveDistances(s, dt);
                applyPairCorrections(s, s.segRanges, s.segInc, s.distCorr);
                solveTets(s, dt);
                applyQuadCorrections(s, s.tetRanges, s.tetInc, s.tetCorr);
            }
            if (runContacts) particleParticleContacts(s);
            if (runRigid) particleRigidContacts(s);
            if (runContacts || runRigid) applyPositionCorrections(s);
            const bool runRigidRigid = rigidRigid && it < rrIt;
            if (runRigidRigid) rigidDepenetration(s);
            // applyRigidCorrections (physics_solver.cpp:1170-1177); zero sums without dynamic bodies
            if ((runRigid || runRigidRigid) && s.hasDynamic) {
                applyRigidCorrections(s);
                syncRigidProxies(s);   // physics_solver.cpp:1178-1186
            }
        }
        // updateRigidVelocities (physics_solver.cpp:1241-1246); restates the predict without
        // dynamic bodies
        if (s.hasDynamic) updateRigidVelocities(s, dt);
        updateVelocities(s, dt);
        if (hasFluidWork) projectFluidBoundaryVelocities(s, dt);
        const bool vorticity = hasFluidWork && anyVorticity(s);
        if (hasFluidWork && (s.postUpdateNeighbors || vorticity)) {
            // post-update neighbour rebuild (physics_solver.cpp:1262-1268); its lists feed
            // vorticity confinement (physics_solver.cpp:1269-1285) and render anisotropy.
            buildFluidNeighbors(s, maxIt > 0 ? maxIt - 1 : 0);
        }
        if (vorticity) fluidVorticity(s, dt);
        if (hasSoftSoftContact && contactIt > 0) particleContactVelocities(s, contactIt);
        if (hasSoftRigidContact && contactIt > 0) particleRigidContactVelocities(s, contactIt);
        skinSurfaceVertices(s);
        updateSurfaceTriangleNormals(s);
        updateSurfaceVertexNormals(s);
        updateSurfaceBounds(s);
        // solveRigidContactVelocities (physics_solver.cpp:1345-1354)
        if (rigidRigid)
            for (uint32_t it = 0; it < std::max(rrIt, jointIt); ++it) {
                if (it < rrIt) rigidSolveVelocities(s);
                applyRigidContactVelocities(s);
            }
        // copyPredictedRigidBodiesToPersistentState
        for (uint32_t b = 0; b < s.B; ++b) {
            s.bodyPos[b] = s.predBodyPos[b];
            s.bodyRot[b] = s.predBodyRot[b];
            s.bodyLin[b] = s.predBodyLin[b];
            s.bodyAng[b] = s.predBodyAng[b];
        }
    }
}

thread_local std::string g_err;

} // namespace

extern "C" {

CN_API const char *cno_last_error(void) { return g_err.c_str(); }

CN_API int cno_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

CN_API cno_solver *cno_create(const cn_solver_desc *desc, const cn_world_soa *world)
{
    if (!desc || !world) { g_err = "null argument"; return nullptr; }
    cno_solver *s = new cno_solver();
    s->desc = *desc;
    setupWorld(*s, *world);
    if (desc->soft.xpbd_schedule != CN_XPBD_GATHER) buildColourings(*s);
    return s;
}

CN_API void cno_destroy(cno_solver *s) { delete s; }

// Switches the reference's post-update neighbour rebuild off (lists then hold the last
// iteration's build), for comparisons with a GPU schedule that skips it.
CN_API void cno_set_post_update_neighbors(cno_solver *s, int enable) { s->postUpdateNeighbors = enable != 0; }

CN_API int cno_step(cno_solver *s, float frame_dt)
{
    if (!s) return CN_ERR_INVALID_ARGUMENT;
    stepFrame(*s, frame_dt);
    return CN_OK;
}

CN_API int cno_set_kinematic_target(cno_solver *s, uint32_t body, const float *pos, const float *rot)
{
    if (!s || body >= s->B) return CN_ERR_INVALID_ARGUMENT;
    s->bodyKinPos[body] = f4{pos[0], pos[1], pos[2], 0.0f};
    s->bodyKinRot[body] = f4{rot[0], rot[1], rot[2], rot[3]};
    s->bodyKinFlags[body] |= 1u;
    return CN_OK;
}

CN_API int cno_read_particles(cno_solver *s, float *x, float *v, float *xprev)
{
    if (!s) return CN_ERR_INVALID_ARGUMENT;
    if (x) std::memcpy(x, s->x.data(), s->x.size() * sizeof(f4));
    if (v) std::memcpy(v, s->v.data(), s->v.size() * sizeof(f4));
    if (xprev) std::memcpy(xprev, s->xprev.data(), s->xprev.size() * sizeof(f4));
    return CN_OK;
}

CN_API int cno_read_rigid_bodies(cno_solver *s, float *pos, float *rot, float *lin, float *ang)
{
    if (!s) return CN_ERR_INVALID_ARGUMENT;
    const size_t bytes = size_t(s->B) * sizeof(f4);
    if (pos) std::memcpy(pos, s->bodyPos.data(), bytes);
    if (rot) std::memcpy(rot, s->bodyRot.data(), bytes);
    if (lin) std::memcpy(lin, s->bodyLin.data(), bytes);
    if (ang) std::memcpy(ang, s->bodyAng.data(), bytes);
    return CN_OK;
}

CN_API int cno_read_surface_render(cno_solver *s, float *positions, float *normals, float *world_aabbs,
                                   float *triangle_normals)
{
    if (!s) return CN_ERR_INVALID_ARGUMENT;
    if (positions) std::memcpy(positions, s->surfPos.data(), s->surfPos.size() * sizeof(f4));
    if (normals) std::memcpy(normals, s->surfNrm.data(), s->surfNrm.size() * sizeof(f4));
    if (world_aabbs) std::memcpy(world_aabbs, s->surfWorldAabb.data(), s->surfWorldAabb.size() * sizeof(f4));
    if (triangle_normals) std::memcpy(triangle_normals, s->surfTriN.data(), s->surfTriN.size() * sizeof(f4));
    return CN_OK;
}

CN_API int cno_read_strand_orientations(cno_solver *s, float *q)
{
    if (!s) return CN_ERR_INVALID_ARGUMENT;
    std::memcpy(q, s->segOrient.data(), s->segOrient.size() * sizeof(f4));
    return CN_OK;
}

// Same buffer ids and layouts as cn_solver_debug_read.
CN_API size_t cno_debug_read(cno_solver *s, int which, void *dst, size_t cap)
{
    if (!s) return 0;
    std::vector<uint8_t> buf;
    auto put = [&](const void *p, size_t n) { buf.assign((const uint8_t *)p, (const uint8_t *)p + n); };
    switch (which) {
    case CN_DEBUG_CELL_ENTRIES: put(s->entries.data(), s->entries.size() * 4); break;
    case CN_DEBUG_SORTED_KEYS: {
        std::vector<uint32_t> kv(size_t(s->N) * 2);
        for (uint32_t i = 0; i < s->N; ++i) { kv[2 * i] = s->sortedKey[i]; kv[2 * i + 1] = s->sortedIdx[i]; }
        put(kv.data(), kv.size() * 4);
        break;
    }
    case CN_DEBUG_CELL_RANGES: put(s->cellRanges.data(), s->cellRanges.size() * sizeof(CellRange)); break;
    case CN_DEBUG_FLUID_NEIGHBOR_COUNTS: put(s->nbrCount.data(), s->nbrCount.size() * 4); break;
    case CN_DEBUG_FLUID_NEIGHBORS: put(s->nbrList.data(), s->nbrList.size() * 4); break;
    case CN_DEBUG_FLUID_CONSTRAINTS: put(s->fluidNormalC.data(), s->fluidNormalC.size() * 16); break;
    case CN_DEBUG_FLUID_DELTA: put(s->fluidDx.data(), s->fluidDx.size() * 16); break;
    case CN_DEBUG_RIGID_CONTACTS: put(s->activeRigidContacts.data(), s->activeRigidContacts.size() * sizeof(RigidContact)); break;
    default: return 0;
    }
    if (dst) std::memcpy(dst, buf.data(), std::min(cap, buf.size()));
    return buf.size();
}

CN_API uint32_t cno_meta(cno_solver *s, uint32_t *out, uint32_t n)
{
    // (required rigid pairs, rigid pair count, required particle pairs, particle pair count,
    //  active rigid contacts, active particle contacts, neighbour-list truncations)
    //  required rigid-rigid collider pairs, rigid-rigid pairs kept)
    //  required proxy contact slots, proxy contact slots kept)
    const uint32_t vals[11] = {s->requiredRigidPairs, uint32_t(s->rigidPairs.size()),
                               s->requiredParticlePairs, uint32_t(s->particlePairs.size()),
                               uint32_t(s->activeRigidContacts.size()),
                               uint32_t(s->activeParticleContacts.size()), s->truncations,
                               s->requiredRigidRigidPairs, uint32_t(s->rrPairs.size()),
                               s->requiredProxyContacts, s->proxyContactSlots};
    for (uint32_t i = 0; i < n && i < 11; ++i) out[i] = vals[i];
    return 11;
}

// Host derivations restated for cross-checking the product's authoring code:
// toFluidSolverMaterial / calculateFluidSolveScales (physics_world.cpp:150-262).
CN_API void cno_fluid_material(float particle_radius, float viscosity, float cohesion,
                               float surface_tension, float vorticity, float gravity_scale,
                               float cfl, cn_fluid_material *out)
{
    const float pi = 3.14159265358979323846f;
    const float restDist = std::max(2.0f * particle_radius, 1.0e-4f);
    const float h = std::max((2.0f / 0.6f) * particle_radius, restDist);
    // tightPack3D (physics_world.cpp:150-182)
    const int dim = int(std::ceil(h / restDist));
    const float rowScale = std::sqrt(0.75f) * restDist;
    float rho = 0.0f, scale = 0.0f, a = 0.0f, b = 0.0f;
    uint32_t count = 0;
    for (int z = -dim; z <= dim && count < 2048; ++z)
        for (int y = -dim; y <= dim && count < 2048; ++y)
            for (int x = -dim; x <= dim && count < 2048; ++x) {
                const float xp = x * restDist + (((y + z) & 1) != 0 ? restDist * 0.5f : 0.0f);
                const f3 smp{xp, y * rowScale, z * rowScale};
                const float m2 = smp.x * smp.x + smp.y * smp.y + smp.z * smp.z;
                if (m2 == 0.0f) continue;
                if (std::sqrt(m2) <= h) {
                    ++count;
                    const float dist = std::sqrt(smp.x * smp.x + smp.y * smp.y + smp.z * smp.z);
                    const float om = 1.0f - dist / h;
                    const float k = 15.0f / (pi * h * h * h);
                    rho += k * om * om;
                    const float dw = -k * 2.0f * om / h;
                    scale += dw * dw;
                    if (smp.y <= 0.0f && dist > 0.0f) {
                        const float ct = smp.y / dist;
                        a += dw * ct;
                        b -= dist * ct;
                    }
                }
            }
    if (rho <= 1.0e-6f) rho = 1.0f;
    if (scale <= 1.0e-6f) scale = 1.0f;
    const float surf = (std::fabs(b) > 1.0e-6f && std::fabs(a) > 1.0e-6f) ? std::fabs(a / b) : 1.0f;
    const float inv = 1.0f / rho;
    const float rr = std::min(std::max(restDist / h, 1.0e-3f), 0.999f);
    const float rr2 = rr * rr;
    out->rest_density = rho;
    out->inv_rest_density = inv;
    out->smoothing_radius = h;
    out->density_constraint_scale = 1.0f / std::max(scale, 1.0e-6f);
    out->viscosity = viscosity * inv;
    out->cohesion = cohesion * h;
    out->cohesion1 = -(1.0f + rr) / rr2;
    out->cohesion2 = (rr2 + rr + 1.0f) / rr2;
    out->surface_tension = (surface_tension * inv) / surf;
    out->vorticity_confinement = vorticity * inv * h;
    out->gravity_scale = gravity_scale;
    out->cfl_radius = cfl * h;
}

} // extern "C"
