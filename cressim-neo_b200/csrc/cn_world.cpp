// cn_world.cpp -- host authoring: the part of PhysicsWorld that derives the particle/constraint
// SoA the solver uploads (reference: src/physics/physics_world.cpp, soft_body_authoring.cpp,
// cloth_authoring.cpp).  Packing order follows PhysicsWorld::Impl::rebuildDerivedState
// (physics_world.cpp:4919-5400): soft bodies, then cloth, then strands, then fluids; phase
// groups are assigned in the same bases.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/cn_physics.h"
#include "cn_internal.h"

namespace {

struct v3 { float x, y, z; };
inline v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
struct quat { float x, y, z, w; };

v3 rotate(const quat &q, v3 v)
{
    const v3 qv{q.x, q.y, q.z};
    const v3 t = 2.0f * cross(qv, v);
    return v + q.w * t + cross(qv, t);
}
quat qmul(const quat &a, const quat &b)
{
    return quat{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
quat qnormalize(quat q)
{
    const float l2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (l2 <= 1.0e-12f) return quat{0, 0, 0, 1};
    const float inv = 1.0f / std::sqrt(l2);
    return quat{q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
// common::runtime_math::applyTransform: scale, rotate, translate.
v3 applyTransform(const cn_transform &t, v3 p)
{
    const v3 scaled{p.x * t.scale[0], p.y * t.scale[1], p.z * t.scale[2]};
    const quat q{t.rotation[0], t.rotation[1], t.rotation[2], t.rotation[3]};
    const v3 r = rotate(q, scaled);
    return v3{r.x + t.position[0], r.y + t.position[1], r.z + t.position[2]};
}

// physics_world.cpp:271-278
cn_contact_material_desc normalizeContact(cn_contact_material_desc m)
{
    m.friction = std::max(m.friction, 0.0f);
    m.static_friction = m.static_friction < 0.0f ? m.friction : std::max(m.static_friction, 0.0f);
    m.restitution = std::min(std::max(m.restitution, 0.0f), 1.0f);
    m.damping = std::max(m.damping, 0.0f);
    return m;
}

// physics_world.cpp:97-262: tightPack3D + calculateFluidSolveScales + toFluidSolverMaterial
cn_fluid_material fluidSolverMaterial(const cn_fluid_grid_desc &d)
{
    const float pi = 3.14159265358979323846f;
    const float r = d.particle_radius;
    const float restDist = std::max(2.0f * r, 1.0e-4f);
    const float h = std::max((2.0f / 0.6f) * r, restDist);
    const int dim = int(std::ceil(h / restDist));
    const float rowScale = std::sqrt(0.75f) * restDist;
    float rho = 0.0f, scale = 0.0f, a = 0.0f, b = 0.0f;
    uint32_t count = 0;
    for (int z = -dim; z <= dim && count < 2048; ++z)
        for (int y = -dim; y <= dim && count < 2048; ++y)
            for (int x = -dim; x <= dim && count < 2048; ++x) {
                const float xp = x * restDist + (((y + z) & 1) != 0 ? restDist * 0.5f : 0.0f);
                const v3 smp{xp, y * rowScale, z * rowScale};
                const float m2 = smp.x * smp.x + smp.y * smp.y + smp.z * smp.z;
                if (m2 == 0.0f) continue;
                if (std::sqrt(m2) > h) continue;
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
    if (rho <= 1.0e-6f) rho = 1.0f;
    if (scale <= 1.0e-6f) scale = 1.0f;
    const float surf = (std::fabs(b) > 1.0e-6f && std::fabs(a) > 1.0e-6f) ? std::fabs(a / b) : 1.0f;
    const float inv = 1.0f / rho;
    const float rr = std::min(std::max(restDist / h, 1.0e-3f), 0.999f);
    const float rr2 = rr * rr;
    cn_fluid_material m{};
    m.rest_density = rho;
    m.inv_rest_density = inv;
    m.smoothing_radius = h;
    m.density_constraint_scale = 1.0f / std::max(scale, 1.0e-6f);
    m.viscosity = std::max(d.viscosity, 0.0f) * inv;
    m.cohesion = std::max(d.cohesion, 0.0f) * h;
    m.cohesion1 = -(1.0f + rr) / rr2;
    m.cohesion2 = (rr2 + rr + 1.0f) / rr2;
    m.surface_tension = (std::max(d.surface_tension, 0.0f) * inv) / surf;
    m.vorticity_confinement = std::max(d.vorticity_confinement, 0.0f) * inv * h;
    m.gravity_scale = d.gravity_scale;
    m.cfl_radius = std::max(d.cfl_coefficient, 0.0f) * h;
    return m;
}

uint32_t packPhase(uint32_t group, bool selfCollide)
{
    return (group & CN_PHASE_GROUP_MASK) | (selfCollide ? CN_PHASE_SELF_COLLIDE : 0u);
}

enum class SoftSource { RegularGrid, TetMesh, Meshfree };
struct SoftBody {
    cn_soft_body_grid_desc desc;
    SoftSource source = SoftSource::RegularGrid;
    std::vector<v3> srcPositions;     // object space (TetMesh / TetGen / meshfree sources)
    std::vector<uint32_t> srcTets;    // 4 indices per tetrahedron (TetMesh / TetGen sources)
    uint32_t neighbourCount = 0;      // meshfree k-nearest graph
    std::vector<uint32_t> staticIdx;
    std::vector<v3> rest;
    std::vector<v3> local;            // rest positions in the object (source) frame
    std::vector<std::array<uint32_t, 4>> tets;
    std::vector<std::array<uint32_t, 2>> edges;
    std::vector<std::vector<uint32_t>> adjacency;
};
struct Fluid {
    cn_fluid_grid_desc desc;
    std::vector<v3> rest;
};
struct Cloth {
    cn_cloth_grid_desc desc;
    std::vector<uint32_t> staticIdx;
    std::vector<v3> rest;
    std::vector<v3> local;            // rest positions in the cloth's own frame
    std::vector<std::array<uint32_t, 2>> structural;
    std::vector<float> structuralRest;
    struct Hinge { uint32_t e0, e1, o0, o1; float angle; };
    std::vector<Hinge> hinges;
    std::vector<std::vector<uint32_t>> adjacency;
};
struct RigidProxies {
    cn_rigid_proxy_desc desc;
    std::vector<v3> local;            // body frame, before the body scale
};
struct Strand {
    cn_strand_desc desc;
    std::vector<uint32_t> staticIdx;
    std::vector<v3> rest;
    std::vector<float> segLen;
    std::vector<quat> segRot;
    std::vector<quat> jointRel;
};

} // namespace

struct cn_world {
    std::vector<SoftBody> softBodies;
    std::vector<Cloth> cloths;
    std::vector<Strand> strands;
    std::vector<Fluid> fluids;
    std::vector<cn_rigid_body_desc> bodies;
    std::vector<cn_collider_desc> colliders;
    std::vector<RigidProxies> proxies;  // at most one set per body
    // packed SoA storage
    std::vector<float> x, v, radii, contactMaterials, bodyPos, bodyRot, bodyLin, bodyAng, bodyScale,
        bodyInvI, bodyKinPos, bodyKinRot, colMat, segOrient, proxyLocal, bodyProxyMat;
    std::vector<uint32_t> kinds, meta, matIdx, fluidMatIdx, ownerTypes, ownerIdx, adjOff, adjCnt, adjIdx,
        bodyTypes, bodyKinFlags, bodyColRanges, bodyColIdx;
    std::vector<cn_fluid_material> fluidMaterials;
    std::vector<cn_soft_edge> edges;
    std::vector<cn_soft_tet> tets;
    std::vector<cn_cloth_dihedral> dihedrals;
    std::vector<cn_strand_segment> segs;
    std::vector<cn_strand_joint> joints;
    std::vector<cn_strand_distance> dists;
    std::vector<cn_collider_geometry> colGeo;
    std::vector<cn_collider_broadphase> colBp;
    // ParticleLayoutMapping views (filled by pack)
    struct OwnerRanges { std::vector<uint64_t> ids; std::vector<uint32_t> env, off, cnt; };
    std::vector<uint32_t> lmEnv, lmPhase, lmLayer, lmMask, lmStrandId, lmStrandOrder, lmStrandRole, lmOwningSoft;
    OwnerRanges lmSoft, lmCloth, lmFluid, lmStrand;
    uint64_t layoutRevision = 0;
    // surface render data: meshes bound by cn_world_add_surface_mesh (owner-relative particle
    // indices), or a caller's copy from cn_world_set_surface_render; packed arrays below
    struct SurfaceMesh {
        uint32_t ownerKind = 0, ownerIndex = 0;
        std::vector<cn_surface_vertex_binding> bindings;
        std::vector<float> fallback;                   // float4 per vertex
        std::vector<std::array<uint32_t, 3>> triangles; // particle indices (owner-relative)
        std::vector<std::array<uint32_t, 3>> triVerts;  // render vertices of each kept triangle
    };
    std::vector<SurfaceMesh> surfaceMeshes;
    bool customSurface = false;
    std::vector<cn_surface_vertex_binding> sBind;
    std::vector<float> sFallback;
    std::vector<cn_surface_triangle_range> sRanges;
    std::vector<uint32_t> sIdx, sTri, sSurf;
    cn_surface_render_data sData{};
    float cellSize = 1.0e-4f;
    // The packed SoA is rebuilt only after an authoring change, so edits a caller makes through
    // the SoA's arrays (state, per-constraint parameters) survive later cn_world_get_soa calls.
    bool packed = false;
};

namespace {

// soft_body_authoring.cpp:81-176 (buildRegularGridSource): object-space lattice and 5-tet split.
void regularGridSource(const cn_soft_body_grid_desc &d, std::vector<v3> &pos, std::vector<uint32_t> &idx)
{
    const float kMinExtent = 1.0e-4f, kMinSpacing = 1.0e-4f;
    const v3 size{std::max(d.size[0], kMinExtent), std::max(d.size[1], kMinExtent), std::max(d.size[2], kMinExtent)};
    const float spacing = std::max(d.target_particle_spacing, kMinSpacing);
    auto res = [spacing](float extent) {
        return std::max<uint32_t>(2u, uint32_t(std::ceil(extent / spacing)) + 1u);
    };
    const uint32_t rx = res(size.x), ry = res(size.y), rz = res(size.z);
    auto flat = [&](uint32_t x, uint32_t y, uint32_t z) { return x * ry * rz + y * rz + z; };
    pos.clear();
    idx.clear();
    for (uint32_t x = 0; x < rx; ++x) {
        const float tx = rx > 1u ? float(x) / float(rx - 1u) : 0.0f;
        for (uint32_t y = 0; y < ry; ++y) {
            const float ty = ry > 1u ? float(y) / float(ry - 1u) : 0.0f;
            for (uint32_t z = 0; z < rz; ++z) {
                const float tz = rz > 1u ? float(z) / float(rz - 1u) : 0.0f;
                pos.push_back(v3{(tx - 0.5f) * size.x, (ty - 0.5f) * size.y, (tz - 0.5f) * size.z});
            }
        }
    }
    for (uint32_t x = 0; x + 1u < rx; ++x)
        for (uint32_t y = 0; y + 1u < ry; ++y)
            for (uint32_t z = 0; z + 1u < rz; ++z) {
                const uint32_t p0 = flat(x, y, z), p1 = flat(x, y, z + 1), p3 = flat(x + 1, y, z),
                               p2 = flat(x + 1, y, z + 1), p7 = flat(x + 1, y + 1, z),
                               p6 = flat(x + 1, y + 1, z + 1), p4 = flat(x, y + 1, z), p5 = flat(x, y + 1, z + 1);
                const uint32_t odd[5][4] = {{p2, p1, p6, p3}, {p6, p3, p4, p7}, {p4, p1, p6, p5}, {p3, p1, p4, p0}, {p6, p1, p4, p3}};
                const uint32_t even[5][4] = {{p0, p2, p5, p1}, {p7, p2, p0, p3}, {p5, p2, p7, p6}, {p7, p0, p5, p4}, {p0, p2, p7, p5}};
                const auto &split = (((x + y + z) & 1u) != 0u) ? odd : even;
                for (int t = 0; t < 5; ++t) idx.insert(idx.end(), split[t], split[t] + 4);
            }
}

// soft_body_authoring.cpp:179-226 (buildMeshfreeKNearestGraph): each particle links to its k
// nearest others (ties by index); edges are unique (min, max) pairs in discovery order.
void meshfreeGraph(SoftBody &sb, uint32_t k)
{
    const uint32_t n = uint32_t(sb.rest.size());
    if (n < 2u) return;
    k = std::min(k, n - 1u);
    std::set<uint64_t> unique;
    std::vector<std::pair<float, uint32_t>> nearest;
    nearest.reserve(n - 1u);
    for (uint32_t i = 0; i < n; ++i) {
        nearest.clear();
        for (uint32_t c = 0; c < n; ++c) {
            if (c == i) continue;
            const v3 d = sb.rest[c] - sb.rest[i];
            nearest.emplace_back(dot(d, d), c);
        }
        std::sort(nearest.begin(), nearest.end(), [](const auto &a, const auto &b) {
            return a.first != b.first ? a.first < b.first : a.second < b.second;
        });
        for (uint32_t slot = 0; slot < k; ++slot) {
            const uint32_t j = nearest[slot].second;
            sb.adjacency[i].push_back(j);
            sb.adjacency[j].push_back(i);
            const uint32_t lo = std::min(i, j), hi = std::max(i, j);
            if (unique.insert((uint64_t(lo) << 32) | hi).second) sb.edges.push_back({lo, hi});
        }
    }
}

// soft_body_authoring.cpp:235-434 (resolveSoftBodyTopology): rest positions through the rest
// transform, then per tetrahedron the range / repeated-vertex / degenerate-volume checks, the
// tetrahedron itself, its 6 edges (unique, in discovery order) and adjacency; static indices are
// sorted, deduplicated and range-checked.  Returns an error text, empty on success.
std::string buildSoftBody(SoftBody &sb)
{
    const cn_soft_body_grid_desc &d = sb.desc;
    const float kMinRestVolume = 1.0e-8f;
    std::vector<v3> src;
    std::vector<uint32_t> idx;
    if (sb.source == SoftSource::RegularGrid) {
        regularGridSource(d, src, idx);
    } else {
        src = sb.srcPositions;
        idx = sb.srcTets;
    }
    if (src.empty()) return "Soft body source does not contain any rest positions.";
    const bool meshfree = sb.source == SoftSource::Meshfree;
    if (!meshfree && idx.empty()) return "Soft body source does not contain any tetrahedra.";
    if (!meshfree && (idx.size() % 4u) != 0u) return "Soft body tetrahedron index buffer size must be divisible by 4.";
    sb.rest.clear();
    for (const v3 &p : src) sb.rest.push_back(applyTransform(d.rest_transform, p));
    sb.local = src;
    const uint32_t n = uint32_t(sb.rest.size());
    sb.adjacency.assign(n, {});
    sb.tets.clear();
    sb.edges.clear();
    if (meshfree) {
        meshfreeGraph(sb, sb.neighbourCount);
    } else {
        std::set<uint64_t> unique;
        for (size_t b = 0; b < idx.size(); b += 4) {
            const std::array<uint32_t, 4> t{idx[b], idx[b + 1], idx[b + 2], idx[b + 3]};
            for (uint32_t v : t)
                if (v >= n)
                    return "Tet vertex index " + std::to_string(v) + " is out of range for " + std::to_string(n) +
                           " particles.";
            if (t[0] == t[1] || t[0] == t[2] || t[0] == t[3] || t[1] == t[2] || t[1] == t[3] || t[2] == t[3])
                return "Soft body tetrahedra must not repeat a vertex index.";
            const v3 a0 = sb.rest[t[0]], a1 = sb.rest[t[1]], a2 = sb.rest[t[2]], a3 = sb.rest[t[3]];
            const float vol = std::fabs(dot(cross(a1 - a0, a2 - a0), a3 - a0) / 6.0f);
            if (vol <= kMinRestVolume) return "Soft body source contains a degenerate tetrahedron.";
            sb.tets.push_back(t);
            const uint32_t pairs[6][2] = {{t[0], t[1]}, {t[0], t[2]}, {t[0], t[3]}, {t[1], t[2]}, {t[1], t[3]}, {t[2], t[3]}};
            for (const auto &e : pairs) {
                sb.adjacency[e[0]].push_back(e[1]);
                sb.adjacency[e[1]].push_back(e[0]);
                const uint32_t lo = std::min(e[0], e[1]), hi = std::max(e[0], e[1]);
                if (unique.insert((uint64_t(lo) << 32) | hi).second) sb.edges.push_back({lo, hi});
            }
        }
    }
    for (auto &a : sb.adjacency) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    for (uint32_t st : sb.staticIdx)
        if (st >= n)
            return "Static particle index " + std::to_string(st) + " is out of range for " + std::to_string(n) +
                   " particles.";
    return std::string();
}

// tetgen_loader.cpp:68-215 (loadTetGenFiles).  '#' starts a comment, blank lines are skipped.
// .node: "count 3 attributes markers" then "id x y z" rows (ids unique); .ele: "count 4 attributes"
// then "id i0 i1 i2 i3" rows whose indices must be ids of the .node table -- dense 0- or
// 1-based renumberings that do not match the ids are rejected rather than guessed.
bool nextMeaningfulLine(std::istream &in, std::string &line)
{
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        const size_t b = line.find_first_not_of(" \t\r\n");
        if (b == std::string::npos) continue;
        const size_t e = line.find_last_not_of(" \t\r\n");
        line = line.substr(b, e - b + 1);
        return true;
    }
    return false;
}

std::string loadTetGen(const char *nodeFile, const char *eleFile, std::vector<v3> &pos, std::vector<uint32_t> &idx)
{
    pos.clear();
    idx.clear();
    const std::string nf = nodeFile ? nodeFile : "", ef = eleFile ? eleFile : "";
    std::ifstream ns(nf);
    if (!ns.is_open()) return "Unable to open TetGen node file '" + nf + "'.";
    std::ifstream es(ef);
    if (!es.is_open()) return "Unable to open TetGen ele file '" + ef + "'.";
    std::string line;
    if (!nextMeaningfulLine(ns, line)) return "TetGen node file '" + nf + "' is empty.";
    uint32_t nodeCount = 0;
    int dim = 0, attrs = 0, markers = 0;
    {
        std::istringstream h(line);
        if (!(h >> nodeCount >> dim >> attrs >> markers)) return "TetGen node file '" + nf + "' has an invalid header.";
    }
    if (dim != 3) return "TetGen node file '" + nf + "' must describe 3D vertices.";
    std::unordered_map<int64_t, uint32_t> idToDense;
    pos.resize(nodeCount);
    for (uint32_t i = 0; i < nodeCount; ++i) {
        if (!nextMeaningfulLine(ns, line))
            return "TetGen node file '" + nf + "' ended before all declared vertices were read.";
        std::istringstream r(line);
        int64_t id = 0;
        v3 p{};
        if (!(r >> id >> p.x >> p.y >> p.z)) return "TetGen node file '" + nf + "' contains an invalid vertex row.";
        if (!idToDense.emplace(id, i).second) return "TetGen node file '" + nf + "' contains duplicate node ids.";
        pos[i] = p;
    }
    if (!nextMeaningfulLine(es, line)) return "TetGen ele file '" + ef + "' is empty.";
    uint32_t tetCount = 0;
    int perTet = 0, eattrs = 0;
    {
        std::istringstream h(line);
        if (!(h >> tetCount >> perTet >> eattrs)) return "TetGen ele file '" + ef + "' has an invalid header.";
    }
    if (perTet != 4) return "TetGen ele file '" + ef + "' must contain tetrahedra with exactly 4 vertices.";
    std::vector<int64_t> raw;
    raw.reserve(size_t(tetCount) * 4u);
    for (uint32_t i = 0; i < tetCount; ++i) {
        if (!nextMeaningfulLine(es, line))
            return "TetGen ele file '" + ef + "' ended before all declared tetrahedra were read.";
        std::istringstream r(line);
        int64_t id = 0, a = 0, b = 0, c = 0, dd = 0;
        if (!(r >> id >> a >> b >> c >> dd)) return "TetGen ele file '" + ef + "' contains an invalid tetrahedron row.";
        raw.insert(raw.end(), {a, b, c, dd});
    }
    idx.reserve(raw.size());
    for (int64_t v : raw) {
        const auto it = idToDense.find(v);
        if (it == idToDense.end()) {
            pos.clear();
            idx.clear();
            return "TetGen ele file '" + ef + "' references node ids missing from '" + nf +
                   "' (dense re-indexed element files are rejected).";
        }
        idx.push_back(it->second);
    }
    return std::string();
}

// physics_world.cpp:6857-6891
void buildFluid(Fluid &f)
{
    const cn_fluid_grid_desc &d = f.desc;
    const float sp = d.target_particle_spacing;
    const uint32_t nx = std::max<uint32_t>(1u, uint32_t(std::floor(d.size[0] / sp + 0.5f)));
    const uint32_t ny = std::max<uint32_t>(1u, uint32_t(std::floor(d.size[1] / sp + 0.5f)));
    const uint32_t nz = std::max<uint32_t>(1u, uint32_t(std::floor(d.size[2] / sp + 0.5f)));
    f.rest.clear();
    f.rest.reserve(size_t(nx) * ny * nz);
    for (uint32_t z = 0; z < nz; ++z)
        for (uint32_t y = 0; y < ny; ++y)
            for (uint32_t x = 0; x < nx; ++x)
                f.rest.push_back(applyTransform(d.rest_transform, v3{-d.size[0] * 0.5f + (float(x) + 0.5f) * sp,
                                                                     -d.size[1] * 0.5f + (float(y) + 0.5f) * sp,
                                                                     -d.size[2] * 0.5f + (float(z) + 0.5f) * sp}));
}

v3 safeNormalize(v3 v, v3 fb)
{
    const float l2 = dot(v, v);
    if (l2 <= 1.0e-8f) return fb;
    return v * (1.0f / std::sqrt(l2));
}

// cloth_authoring.cpp:58-191 for a rectangular grid triangulated as (v00, v10, v11), (v00, v11, v01).
cn_status buildCloth(Cloth &c)
{
    const cn_cloth_grid_desc &d = c.desc;
    const uint32_t nx = std::max<uint32_t>(d.resolution[0], 2u), ny = std::max<uint32_t>(d.resolution[1], 2u);
    c.rest.clear();
    c.local.clear();
    for (uint32_t j = 0; j < ny; ++j)
        for (uint32_t i = 0; i < nx; ++i) {
            const v3 lp{(float(i) / float(nx - 1) - 0.5f) * d.size[0], 0.0f, (float(j) / float(ny - 1) - 0.5f) * d.size[1]};
            c.local.push_back(lp);
            c.rest.push_back(applyTransform(d.rest_transform, lp));
        }
    struct Inc { uint32_t a, b; std::vector<uint32_t> opp; };
    std::map<uint64_t, Inc> edges;
    auto addTri = [&](uint32_t a, uint32_t b, uint32_t cc) {
        const uint32_t rec[3][3] = {{a, b, cc}, {b, cc, a}, {cc, a, b}};
        for (auto r : rec) {
            uint32_t e0 = r[0], e1 = r[1];
            if (e0 > e1) std::swap(e0, e1);
            auto it = edges.try_emplace((uint64_t(e0) << 32) | e1, Inc{e0, e1, {}}).first;
            it->second.opp.push_back(r[2]);
        }
    };
    for (uint32_t j = 0; j + 1 < ny; ++j)
        for (uint32_t i = 0; i + 1 < nx; ++i) {
            const uint32_t v00 = j * nx + i, v10 = v00 + 1, v01 = v00 + nx, v11 = v01 + 1;
            addTri(v00, v10, v11);
            addTri(v00, v11, v01);
        }
    c.adjacency.assign(c.rest.size(), {});
    c.structural.clear(); c.structuralRest.clear(); c.hinges.clear();
    for (auto &kv : edges) {
        Inc &e = kv.second;
        const v3 delta = c.rest[e.b] - c.rest[e.a];
        c.structural.push_back({e.a, e.b});
        c.structuralRest.push_back(std::sqrt(dot(delta, delta)));
        c.adjacency[e.a].push_back(e.b);
        c.adjacency[e.b].push_back(e.a);
        if (e.opp.size() == 2u) {
            std::sort(e.opp.begin(), e.opp.end());
            const v3 x0 = c.rest[e.a], x1 = c.rest[e.b], x2 = c.rest[e.opp[0]], x3 = c.rest[e.opp[1]];
            const v3 edge = safeNormalize(x1 - x0, v3{1, 0, 0});
            const v3 n0 = safeNormalize(cross(edge, x2 - x0), v3{0, 1, 0});
            const v3 n1 = safeNormalize(cross(x3 - x0, edge), v3{0, 1, 0});
            const float angle = std::atan2(dot(edge, cross(n0, n1)), dot(n0, n1));
            c.hinges.push_back({e.a, e.b, e.opp[0], e.opp[1], angle});
            c.adjacency[e.opp[0]].push_back(e.opp[1]);
            c.adjacency[e.opp[1]].push_back(e.opp[0]);
        }
    }
    for (auto &a : c.adjacency) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    for (uint32_t s : c.staticIdx)
        if (s >= c.rest.size()) return CN_ERR_INVALID_ARGUMENT;
    return CN_OK;
}

// physics_world.cpp:426-473 frame helpers + quaternionFromBasis (:374-424)
v3 defaultRootNormal(v3 dir0, v3 authored)
{
    const v3 dir = safeNormalize(dir0, v3{1, 0, 0});
    v3 n = authored;
    if (dot(n, n) <= 1.0e-8f) n = v3{0, 1, 0};
    n = n - dir * dot(n, dir);
    if (dot(n, n) <= 1.0e-8f) {
        v3 fb{0, 1, 0};
        if (std::fabs(dot(dir, fb)) > 0.9f) fb = v3{1, 0, 0};
        n = fb - dir * dot(fb, dir);
    }
    return safeNormalize(n, v3{0, 1, 0});
}
v3 parallelTransport(v3 prevT, v3 nextT, v3 prevN)
{
    v3 t = prevN - nextT * dot(prevN, nextT);
    if (dot(t, t) <= 1.0e-8f) t = defaultRootNormal(nextT, prevN);
    return safeNormalize(t, defaultRootNormal(nextT, prevN));
}
quat fromBasis(v3 xa, v3 ya, v3 za)
{
    const float m00 = xa.x, m01 = ya.x, m02 = za.x, m10 = xa.y, m11 = ya.y, m12 = za.y, m20 = xa.z, m21 = ya.z, m22 = za.z;
    const float tr = m00 + m11 + m22;
    quat r{};
    if (tr > 0.0f) {
        const float s = std::sqrt(tr + 1.0f) * 2.0f;
        r = quat{(m21 - m12) / s, (m02 - m20) / s, (m10 - m01) / s, 0.25f * s};
    } else if (m00 > m11 && m00 > m22) {
        const float s = std::sqrt(1.0f + m00 - m11 - m22) * 2.0f;
        r = quat{0.25f * s, (m01 + m10) / s, (m02 + m20) / s, (m21 - m12) / s};
    } else if (m11 > m22) {
        const float s = std::sqrt(1.0f + m11 - m00 - m22) * 2.0f;
        r = quat{(m01 + m10) / s, 0.25f * s, (m12 + m21) / s, (m02 - m20) / s};
    } else {
        const float s = std::sqrt(1.0f + m22 - m00 - m11) * 2.0f;
        r = quat{(m02 + m20) / s, (m12 + m21) / s, 0.25f * s, (m10 - m01) / s};
    }
    return qnormalize(r);
}

// physics_world.cpp:6893-6969 (prepareStrandStateForInsert)
cn_status buildStrand(Strand &st)
{
    const uint32_t n = uint32_t(st.rest.size());
    if (n < 2u) return CN_ERR_INVALID_ARGUMENT;
    st.segLen.clear(); st.segRot.clear(); st.jointRel.clear();
    v3 prevN{0, 1, 0}, prevT{1, 0, 0};
    for (uint32_t i = 0; i + 1 < n; ++i) {
        const v3 delta = st.rest[i + 1] - st.rest[i];
        const float len = std::sqrt(dot(delta, delta));
        if (len <= 1.0e-6f) return CN_ERR_INVALID_ARGUMENT;
        const v3 t = safeNormalize(delta, v3{1, 0, 0});
        v3 mn = i == 0 ? defaultRootNormal(t, v3{0, 1, 0}) : parallelTransport(prevT, t, prevN);
        mn = safeNormalize(mn, v3{0, 1, 0});
        const v3 xa = safeNormalize(t, v3{1, 0, 0});
        const v3 ya = safeNormalize(mn - xa * dot(mn, xa), defaultRootNormal(xa, mn));
        const v3 za = safeNormalize(cross(xa, ya), v3{0, 0, 1});
        st.segLen.push_back(len);
        st.segRot.push_back(fromBasis(xa, ya, za));
        prevN = mn;
        prevT = t;
    }
    for (uint32_t i = 0; i + 1 < st.segRot.size(); ++i) {
        const quat a = st.segRot[i];
        st.jointRel.push_back(qmul(quat{-a.x, -a.y, -a.z, a.w}, st.segRot[i + 1]));
    }
    for (uint32_t s : st.staticIdx)
        if (s >= n) return CN_ERR_INVALID_ARGUMENT;
    return CN_OK;
}

uint32_t findOrAppendContact(std::vector<float> &table, const cn_contact_material_desc &m)
{
    const float rec[4] = {m.friction, m.restitution, m.damping, m.static_friction};
    for (size_t i = 0; i + 4 <= table.size(); i += 4)
        if (std::memcmp(&table[i], rec, sizeof(rec)) == 0) return uint32_t(i / 4);
    table.insert(table.end(), rec, rec + 4);
    return uint32_t(table.size() / 4 - 1);
}
uint32_t findOrAppendFluid(std::vector<cn_fluid_material> &table, const cn_fluid_material &m)
{
    for (size_t i = 0; i < table.size(); ++i)
        if (std::memcmp(&table[i], &m, sizeof(m)) == 0) return uint32_t(i);
    table.push_back(m);
    return uint32_t(table.size() - 1);
}

void pushParticle(cn_world &w, v3 p, float invMass, float radius, uint32_t kind, uint32_t env, uint32_t phase,
                  uint32_t layer, uint32_t mask, uint32_t mat, uint32_t fmat, uint32_t ownerType, uint32_t owner)
{
    w.x.insert(w.x.end(), {p.x, p.y, p.z, invMass});
    w.v.insert(w.v.end(), {0.f, 0.f, 0.f, 0.f});
    w.radii.push_back(radius);
    w.kinds.push_back(kind);
    w.meta.insert(w.meta.end(), {env, phase, layer, mask});
    w.matIdx.push_back(mat);
    w.fluidMatIdx.push_back(fmat);
    w.ownerTypes.push_back(ownerType);
    w.ownerIdx.push_back(owner);
}

// ---------------------------------------------------------------------------- surface meshes
// Render-vertex bindings as the engine's World builds them (world.cpp:180-395, 3255-3554).

// quantizePoint (world.cpp:180-188): nearest integer lattice point at spacing epsilon
std::array<int64_t, 3> quantizePoint(v3 p, float eps)
{
    const double inv = 1.0 / double(std::max(eps, 1.0e-8f));
    return {std::llround(double(p.x) * inv), std::llround(double(p.y) * inv), std::llround(double(p.z) * inv)};
}

struct QuantKeyHash {
    size_t operator()(const std::array<int64_t, 3> &k) const
    {
        uint64_t h = 1469598103934665603ull;
        for (int64_t v : k) h = (h ^ uint64_t(v)) * 1099511628211ull;
        return size_t(h);
    }
};

// makeExactSurfaceDeformableVertexBinding (world.cpp:268-276)
cn_surface_vertex_binding exactBinding(uint32_t particle)
{
    cn_surface_vertex_binding b{};
    for (int k = 0; k < 4; ++k) b.particle_indices[k] = particle;
    b.weights[0] = 1.0f;
    return b;
}

// makeNearestParticleSkinBinding (world.cpp:278-366): the 4 nearest rest particles (strictly
// closer ones first, ties keep the earlier particle), weights 1 / (distance + 1e-6) normalised
cn_surface_vertex_binding nearestBinding(v3 vtx, const std::vector<v3> &rest)
{
    struct Cand { float d2; uint32_t idx; bool valid; };
    std::array<Cand, 4> nearest{};
    for (auto &c : nearest) c = Cand{std::numeric_limits<float>::max(), 0u, false};
    for (uint32_t p = 0; p < rest.size(); ++p) {
        const v3 dlt = rest[p] - vtx;
        const float d2 = dot(dlt, dlt);
        for (size_t slot = 0; slot < nearest.size(); ++slot) {
            if (nearest[slot].valid && d2 >= nearest[slot].d2) continue;
            for (size_t m = nearest.size() - 1; m > slot; --m) nearest[m] = nearest[m - 1];
            nearest[slot] = Cand{d2, p, true};
            break;
        }
    }
    cn_surface_vertex_binding b = exactBinding(nearest[0].valid ? nearest[0].idx : 0u);
    if (!nearest[0].valid) return b;
    float raw[4] = {0.f, 0.f, 0.f, 0.f}, sum = 0.0f;
    for (size_t slot = 0; slot < 4; ++slot) {
        if (!nearest[slot].valid) continue;
        const float dist = std::sqrt(std::max(nearest[slot].d2, 0.0f));
        raw[slot] = 1.0f / (dist + 1.0e-6f);
        sum += raw[slot];
        b.particle_indices[slot] = nearest[slot].idx;
    }
    if (sum <= 0.0f) return b;
    for (int k = 0; k < 4; ++k) b.weights[k] = raw[k] / sum;
    return b;
}

// dominantParticleIndex (world.cpp:367-388): the first particle of largest weight
uint32_t dominantParticle(const cn_surface_vertex_binding &b)
{
    uint32_t idx = b.particle_indices[0];
    float wt = b.weights[0];
    for (int k = 1; k < 4; ++k)
        if (b.weights[k] > wt) {
            idx = b.particle_indices[k];
            wt = b.weights[k];
        }
    return idx;
}

// transformNormal (world.cpp:213-228) with the identity transform
void fallbackNormal(const float *n, float *out)
{
    v3 v = n ? v3{n[0], n[1], n[2]} : v3{0.f, 0.f, 0.f};
    const float l2 = dot(v, v);
    if (l2 <= 1.0e-12f) v = v3{0.f, 1.f, 0.f};
    else v = v * (1.0f / std::sqrt(l2));
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = 0.0f;
}

std::string bindSurfaceMesh(const cn_world &w, const cn_surface_mesh_desc &d, cn_world::SurfaceMesh &m)
{
    const bool cloth = d.owner_kind == CN_SURFACE_OWNER_CLOTH;
    if (d.owner_kind > CN_SURFACE_OWNER_CLOTH) return "surface mesh: unknown owner kind";
    if (cloth ? d.owner_index >= w.cloths.size() : d.owner_index >= w.softBodies.size())
        return "surface mesh: owner index out of range";
    if (d.vertex_count == 0 || !d.positions) return "surface mesh: missing visual mesh";
    if (d.index_count && !d.indices) return "surface mesh: missing index buffer";
    const std::vector<v3> &rest = cloth ? w.cloths[d.owner_index].local : w.softBodies[d.owner_index].local;
    if (rest.empty()) return "surface mesh: owner has no rest positions";
    const float eps = d.match_epsilon > 0.0f ? d.match_epsilon : 1.0e-3f;
    const float eps2 = eps * eps;
    const uint32_t V = d.vertex_count;
    auto vtx = [&](uint32_t i) { return v3{d.positions[3 * i], d.positions[3 * i + 1], d.positions[3 * i + 2]}; };
    m.ownerKind = d.owner_kind;
    m.ownerIndex = d.owner_index;
    m.bindings.clear();
    m.fallback.assign(size_t(V) * 4, 0.0f);
    for (uint32_t i = 0; i < V; ++i) fallbackNormal(d.normals ? d.normals + 3 * i : nullptr, &m.fallback[4 * size_t(i)]);
    std::vector<uint32_t> mapping(V, 0u);
    if (cloth) {
        // identity when every vertex sits on the particle of its index, else one unique match each
        bool identity = rest.size() == V;
        for (uint32_t i = 0; identity && i < V; ++i) {
            const v3 dl = vtx(i) - rest[i];
            identity = dot(dl, dl) <= eps2;
            mapping[i] = i;
        }
        if (!identity)
            for (uint32_t i = 0; i < V; ++i) {
                uint32_t match = 0, matches = 0;
                for (uint32_t p = 0; p < rest.size(); ++p) {
                    const v3 dl = vtx(i) - rest[p];
                    if (dot(dl, dl) <= eps2) {
                        match = p;
                        ++matches;
                    }
                }
                if (matches != 1u)
                    return "Cloth render binding build failed: mapping is missing, ambiguous, mismatched, or "
                           "collapses a triangle.";
                mapping[i] = match;
            }
        for (uint32_t t = 0; t + 2u < d.index_count; t += 3u) {
            const uint32_t a = d.indices[t], b = d.indices[t + 1], c = d.indices[t + 2];
            if (a >= V || b >= V || c >= V || mapping[a] == mapping[b] || mapping[b] == mapping[c] ||
                mapping[c] == mapping[a])
                return "Cloth render binding build failed: mapping is missing, ambiguous, mismatched, or "
                       "collapses a triangle.";
        }
        for (uint32_t i = 0; i < V; ++i) m.bindings.push_back(exactBinding(mapping[i]));
    } else if (w.softBodies[d.owner_index].source == SoftSource::Meshfree) {
        for (uint32_t i = 0; i < V; ++i) m.bindings.push_back(nearestBinding(vtx(i), rest));
    } else {
        std::unordered_map<std::array<int64_t, 3>, uint32_t, QuantKeyHash> byKey;
        byKey.reserve(rest.size());
        for (uint32_t p = 0; p < rest.size(); ++p) byKey.try_emplace(quantizePoint(rest[p], eps), p);
        for (uint32_t i = 0; i < V; ++i) {
            const v3 q = vtx(i);
            const auto it = byKey.find(quantizePoint(q, eps));
            bool found = it != byKey.end();
            uint32_t best = found ? it->second : 0u;
            if (!found) { // findMatchingRestVertexLocal's scan: closest within epsilon, later ties win
                float bestD2 = eps2;
                for (uint32_t p = 0; p < rest.size(); ++p) {
                    const v3 dl = rest[p] - q;
                    const float d2 = dot(dl, dl);
                    if (d2 > bestD2) continue;
                    bestD2 = d2;
                    best = p;
                    found = true;
                }
            }
            if (!found)
                return "Soft-body render binding build failed: visual mesh vertices must match tet rest vertices "
                       "exactly.";
            m.bindings.push_back(exactBinding(best));
        }
    }
    m.triangles.clear();
    m.triVerts.clear();
    for (uint32_t t = 0; t + 2u < d.index_count; t += 3u) {
        const uint32_t a = d.indices[t], b = d.indices[t + 1], c = d.indices[t + 2];
        if (a >= V || b >= V || c >= V) continue;
        if (cloth)
            m.triangles.push_back({mapping[a], mapping[b], mapping[c]});
        else
            m.triangles.push_back({dominantParticle(m.bindings[a]), dominantParticle(m.bindings[b]),
                                   dominantParticle(m.bindings[c])});
        m.triVerts.push_back({a, b, c});
    }
    return {};
}

// Packs the surface render arrays once the particle offsets of the owners are known.
void packSurfaces(cn_world &w, const std::vector<uint32_t> &softOff, const std::vector<uint32_t> &clothOff)
{
    if (w.customSurface) return;
    w.sBind.clear(); w.sFallback.clear(); w.sRanges.clear(); w.sIdx.clear(); w.sTri.clear(); w.sSurf.clear();
    for (uint32_t si = 0; si < w.softBodies.size(); ++si) {
        w.sSurf.push_back(softOff[si]);
        w.sSurf.push_back(uint32_t(w.softBodies[si].rest.size()));
    }
    for (uint32_t ci = 0; ci < w.cloths.size(); ++ci) {
        w.sSurf.push_back(clothOff[ci]);
        w.sSurf.push_back(uint32_t(w.cloths[ci].rest.size()));
    }
    for (const cn_world::SurfaceMesh &m : w.surfaceMeshes) {
        const uint32_t off = m.ownerKind == CN_SURFACE_OWNER_CLOTH ? clothOff[m.ownerIndex] : softOff[m.ownerIndex];
        const uint32_t vBase = uint32_t(w.sBind.size()), tBase = uint32_t(w.sTri.size() / 4);
        for (cn_surface_vertex_binding b : m.bindings) {
            for (uint32_t &p : b.particle_indices) p += off;
            w.sBind.push_back(b);
        }
        w.sFallback.insert(w.sFallback.end(), m.fallback.begin(), m.fallback.end());
        std::vector<std::vector<uint32_t>> incident(m.bindings.size());
        for (uint32_t t = 0; t < m.triangles.size(); ++t) {
            for (uint32_t k = 0; k < 3; ++k) w.sTri.push_back(m.triangles[t][k] + off);
            w.sTri.push_back(0u);
            for (uint32_t k = 0; k < 3; ++k) incident[m.triVerts[t][k]].push_back(tBase + t);
        }
        for (uint32_t v = 0; v < incident.size(); ++v) {
            w.sRanges.push_back(cn_surface_triangle_range{uint32_t(w.sIdx.size()), uint32_t(incident[v].size()), 0u, 0u});
            w.sIdx.insert(w.sIdx.end(), incident[v].begin(), incident[v].end());
        }
        (void)vBase;
    }
}

// The ParticleLayoutMapping views of the packed particles (physics_world.cpp:4919-5400 fill the
// same per-particle arrays: strand ids / orders for strand particles, 0xffffffff elsewhere; the
// owning soft body for soft-body particles, 0xffffffff elsewhere; no strand roles without
// suturing) and each owner's contiguous slot range.
void packLayoutMapping(cn_world &w)
{
    const size_t N = w.radii.size();
    w.lmEnv.resize(N); w.lmPhase.resize(N); w.lmLayer.resize(N); w.lmMask.resize(N);
    w.lmStrandId.assign(N, 0xffffffffu); w.lmStrandOrder.assign(N, 0xffffffffu);
    w.lmStrandRole.assign(N, 0u); w.lmOwningSoft.assign(N, 0xffffffffu);
    cn_world::OwnerRanges *byType[6] = {nullptr, &w.lmSoft, &w.lmFluid, &w.lmStrand, nullptr, &w.lmCloth};
    const size_t owners[6] = {0, w.softBodies.size(), w.fluids.size(), w.strands.size(), 0, w.cloths.size()};
    for (int t = 0; t < 6; ++t) {
        if (!byType[t]) continue;
        cn_world::OwnerRanges &r = *byType[t];
        r.ids.resize(owners[t]);
        r.env.assign(owners[t], 0u);
        r.off.assign(owners[t], 0u);
        r.cnt.assign(owners[t], 0u);
        for (size_t k = 0; k < owners[t]; ++k) r.ids[k] = k;
    }
    for (size_t i = 0; i < N; ++i) {
        w.lmEnv[i] = w.meta[4 * i];
        w.lmPhase[i] = w.meta[4 * i + 1];
        w.lmLayer[i] = w.meta[4 * i + 2];
        w.lmMask[i] = w.meta[4 * i + 3];
        const uint32_t type = w.ownerTypes[i], owner = w.ownerIdx[i];
        if (type < 6 && byType[type] && owner < owners[type]) {
            cn_world::OwnerRanges &r = *byType[type];
            if (r.cnt[owner] == 0u) {
                r.off[owner] = uint32_t(i);
                r.env[owner] = w.meta[4 * i];
            }
            if (type == CN_OWNER_STRAND) {
                w.lmStrandId[i] = owner;
                w.lmStrandOrder[i] = r.cnt[owner];
            }
            ++r.cnt[owner];
        }
        if (type == CN_OWNER_SOFT_BODY) w.lmOwningSoft[i] = owner;
    }
    ++w.layoutRevision;
}

cn_status pack(cn_world &w)
{
    w.x.clear(); w.v.clear(); w.radii.clear(); w.kinds.clear(); w.meta.clear(); w.matIdx.clear();
    w.fluidMatIdx.clear(); w.ownerTypes.clear(); w.ownerIdx.clear(); w.contactMaterials.clear();
    w.fluidMaterials.clear(); w.edges.clear(); w.tets.clear(); w.dihedrals.clear(); w.segs.clear();
    w.segOrient.clear(); w.joints.clear(); w.dists.clear();
    std::vector<std::vector<uint32_t>> adjacency;
    const uint32_t clothBase = uint32_t(w.softBodies.size());
    const uint32_t strandBase = clothBase + uint32_t(w.cloths.size());
    const uint32_t fluidBase = strandBase + uint32_t(w.strands.size());
    const uint32_t proxyBase = fluidBase + uint32_t(w.fluids.size());

    // Rigid proxy particles first, bodies in index order (physics_world.cpp:4931-5023): inverse
    // mass 0, a phase group of their own per body (no self collision), the scaled local position
    // kept for the per-substep sync; the body's packed proxy material (zero without proxies).
    w.proxyLocal.clear();
    w.bodyProxyMat.assign(w.bodies.size() * 4, 0.0f);
    for (uint32_t b = 0; b < w.bodies.size(); ++b) {
        const RigidProxies *rp = nullptr;
        for (const RigidProxies &r : w.proxies)
            if (r.desc.body == b) rp = &r;
        if (!rp || rp->local.empty() || rp->desc.radius <= 0.0f) continue;
        const cn_rigid_body_desc &bd = w.bodies[b];
        const cn_contact_material_desc m = normalizeContact(rp->desc.material);
        const uint32_t mat = findOrAppendContact(w.contactMaterials, m);
        const float packed[4] = {m.friction, m.restitution, m.damping, m.static_friction};
        std::memcpy(&w.bodyProxyMat[4 * b], packed, sizeof(packed));
        const quat q{bd.orientation[0], bd.orientation[1], bd.orientation[2], bd.orientation[3]};
        const v3 pos{bd.position[0], bd.position[1], bd.position[2]};
        const uint32_t layer = rp->desc.collision_layer == 0u ? 1u : rp->desc.collision_layer;
        for (const v3 &l : rp->local) {
            const v3 scaled{l.x * bd.scale[0], l.y * bd.scale[1], l.z * bd.scale[2]};
            pushParticle(w, rotate(q, scaled) + pos, 0.0f, rp->desc.radius, CN_PARTICLE_SOLID, rp->desc.environment_index,
                         packPhase(proxyBase + b, false), layer, rp->desc.collision_mask, mat, 0xffffffffu,
                         CN_OWNER_RIGID_BODY, b);
            adjacency.emplace_back();
            w.proxyLocal.insert(w.proxyLocal.end(), {scaled.x, scaled.y, scaled.z, 0.0f});
        }
    }
    const bool anyProxy = !w.proxyLocal.empty();

    std::vector<uint32_t> softOff, clothOff;
    for (uint32_t si = 0; si < w.softBodies.size(); ++si) {
        SoftBody &sb = w.softBodies[si];
        const cn_soft_body_grid_desc &d = sb.desc;
        const uint32_t mat = findOrAppendContact(w.contactMaterials, normalizeContact(d.material));
        const uint32_t off = uint32_t(w.radii.size());
        softOff.push_back(off);
        const float inv = d.particle_mass > 0.0f ? 1.0f / d.particle_mass : 0.0f;
        std::unordered_set<uint32_t> fixed(sb.staticIdx.begin(), sb.staticIdx.end());
        const uint32_t layer = d.collision_layer == 0u ? 1u : d.collision_layer;
        for (uint32_t k = 0; k < sb.rest.size(); ++k) {
            pushParticle(w, sb.rest[k], fixed.count(k) ? 0.0f : inv, d.particle_radius, CN_PARTICLE_SOLID,
                         d.environment_index, packPhase(si, d.self_collision_enabled != 0u), layer,
                         d.collision_mask, mat, 0xffffffffu, CN_OWNER_SOFT_BODY, si);
            adjacency.emplace_back();
        }
        for (uint32_t k = 0; k < sb.adjacency.size(); ++k)
            for (uint32_t nb : sb.adjacency[k]) adjacency[off + k].push_back(off + nb);
        for (const auto &e : sb.edges) {
            const v3 delta = sb.rest[e[1]] - sb.rest[e[0]];
            cn_soft_edge ed{};
            ed.particle_a = off + e[0];
            ed.particle_b = off + e[1];
            ed.rest_length = std::sqrt(dot(delta, delta));
            ed.compliance = d.edge_compliance;
            ed.enabled = 1u;
            w.edges.push_back(ed);
        }
        for (const auto &t : sb.tets) {
            const v3 p0 = sb.rest[t[0]], p1 = sb.rest[t[1]], p2 = sb.rest[t[2]], p3 = sb.rest[t[3]];
            cn_soft_tet tt{};
            for (int k = 0; k < 4; ++k) tt.particle_indices[k] = off + t[k];
            tt.rest_volume = std::fabs(dot(cross(p1 - p0, p2 - p0), p3 - p0)) / 6.0f;
            tt.compliance = d.volume_compliance;
            w.tets.push_back(tt);
        }
    }
    for (uint32_t ci = 0; ci < w.cloths.size(); ++ci) {
        Cloth &c = w.cloths[ci];
        const cn_cloth_grid_desc &d = c.desc;
        const uint32_t mat = findOrAppendContact(w.contactMaterials, normalizeContact(d.material));
        const uint32_t off = uint32_t(w.radii.size());
        clothOff.push_back(off);
        const float inv = d.particle_mass > 0.0f ? 1.0f / d.particle_mass : 0.0f;
        std::unordered_set<uint32_t> fixed(c.staticIdx.begin(), c.staticIdx.end());
        const uint32_t layer = d.collision_layer == 0u ? 1u : d.collision_layer;
        for (uint32_t k = 0; k < c.rest.size(); ++k) {
            pushParticle(w, c.rest[k], fixed.count(k) ? 0.0f : inv, d.particle_radius, CN_PARTICLE_SOLID,
                         d.environment_index, packPhase(clothBase + ci, d.self_collision_enabled != 0u), layer,
                         d.collision_mask, mat, 0xffffffffu, CN_OWNER_CLOTH, ci);
            adjacency.emplace_back();
        }
        for (uint32_t k = 0; k < c.adjacency.size(); ++k)
            for (uint32_t nb : c.adjacency[k]) adjacency[off + k].push_back(off + nb);
        for (size_t k = 0; k < c.structural.size(); ++k) {
            cn_soft_edge ed{};
            ed.particle_a = off + c.structural[k][0];
            ed.particle_b = off + c.structural[k][1];
            ed.rest_length = c.structuralRest[k];
            ed.compliance = d.structural_compliance;
            ed.enabled = 1u;
            w.edges.push_back(ed);
        }
        for (const auto &h : c.hinges) {
            cn_cloth_dihedral dh{};
            dh.edge_particle0 = off + h.e0;
            dh.edge_particle1 = off + h.e1;
            dh.opposite_particle0 = off + h.o0;
            dh.opposite_particle1 = off + h.o1;
            dh.rest_angle = h.angle;
            dh.compliance = d.bend_compliance;
            w.dihedrals.push_back(dh);
        }
    }
    for (uint32_t si = 0; si < w.strands.size(); ++si) {
        Strand &st = w.strands[si];
        const cn_strand_desc &d = st.desc;
        const uint32_t mat = findOrAppendContact(w.contactMaterials, normalizeContact(d.material));
        const uint32_t off = uint32_t(w.radii.size());
        const uint32_t segOff = uint32_t(w.segs.size());
        const float inv = d.particle_mass > 0.0f ? 1.0f / d.particle_mass : 0.0f;
        std::unordered_set<uint32_t> fixed(st.staticIdx.begin(), st.staticIdx.end());
        const uint32_t layer = d.collision_layer == 0u ? 1u : d.collision_layer;
        for (uint32_t k = 0; k < st.rest.size(); ++k) {
            pushParticle(w, st.rest[k], fixed.count(k) ? 0.0f : inv, d.particle_radius, CN_PARTICLE_SOLID,
                         d.environment_index, packPhase(strandBase + si, d.self_collision_enabled != 0u), layer,
                         d.collision_mask, mat, 0xffffffffu, CN_OWNER_STRAND, si);
            adjacency.emplace_back();
        }
        for (uint32_t k = 0; k + 1 < st.rest.size(); ++k) {
            adjacency[off + k].push_back(off + k + 1);
            adjacency[off + k + 1].push_back(off + k);
        }
        for (uint32_t g = 0; g < st.segLen.size(); ++g) {
            cn_strand_segment sg{};
            sg.particle_a = off + g;
            sg.particle_b = off + g + 1;
            sg.rest_length = st.segLen[g];
            sg.stretch_shear_compliance = d.stretch_shear_compliance;
            const quat q = st.segRot[g];
            sg.rest_orientation[0] = q.x; sg.rest_orientation[1] = q.y;
            sg.rest_orientation[2] = q.z; sg.rest_orientation[3] = q.w;
            w.segs.push_back(sg);
            w.segOrient.insert(w.segOrient.end(), {q.x, q.y, q.z, q.w});
            w.dists.push_back(cn_strand_distance{sg.particle_a, sg.particle_b, sg.rest_length, d.distance_compliance});
        }
        for (uint32_t j = 0; j < st.jointRel.size(); ++j) {
            cn_strand_joint jt{};
            jt.segment_a = segOff + j;
            jt.segment_b = segOff + j + 1;
            jt.bend_compliance = d.bend_compliance;
            jt.twist_compliance = d.twist_compliance;
            const quat q = st.jointRel[j];
            jt.rest_relative_orientation[0] = q.x; jt.rest_relative_orientation[1] = q.y;
            jt.rest_relative_orientation[2] = q.z; jt.rest_relative_orientation[3] = q.w;
            w.joints.push_back(jt);
        }
    }
    for (uint32_t fi = 0; fi < w.fluids.size(); ++fi) {
        Fluid &f = w.fluids[fi];
        const cn_fluid_grid_desc &d = f.desc;
        const uint32_t mat = findOrAppendContact(w.contactMaterials, normalizeContact(d.material));
        const uint32_t fmat = findOrAppendFluid(w.fluidMaterials, fluidSolverMaterial(d));
        const float inv = d.particle_mass > 0.0f ? 1.0f / d.particle_mass : 0.0f;
        const uint32_t layer = d.collision_layer == 0u ? 1u : d.collision_layer;
        for (const v3 &p : f.rest) {
            pushParticle(w, p, inv, d.particle_radius, CN_PARTICLE_FLUID, d.environment_index,
                         packPhase(fluidBase + fi, true), layer, d.collision_mask, mat, fmat, CN_OWNER_FLUID, fi);
            adjacency.emplace_back();
        }
    }
    if (anyProxy) w.proxyLocal.resize(w.radii.size() * 4, 0.0f); // zero for every other particle
    else w.bodyProxyMat.clear();
    // adjacency CSR
    w.adjOff.assign(adjacency.size(), 0);
    w.adjCnt.assign(adjacency.size(), 0);
    w.adjIdx.clear();
    for (size_t i = 0; i < adjacency.size(); ++i) {
        w.adjOff[i] = uint32_t(w.adjIdx.size());
        w.adjCnt[i] = uint32_t(adjacency[i].size());
        w.adjIdx.insert(w.adjIdx.end(), adjacency[i].begin(), adjacency[i].end());
    }
    // recomputeParticleGridCellSize (physics_world.cpp:6829-6846)
    float cell = 0.0f;
    for (size_t i = 0; i < w.radii.size(); ++i) {
        cell = std::max(cell, w.radii[i] * 2.0f);
        if (w.fluidMatIdx[i] != 0xffffffffu && w.fluidMatIdx[i] < w.fluidMaterials.size())
            cell = std::max(cell, w.fluidMaterials[w.fluidMatIdx[i]].smoothing_radius);
    }
    w.cellSize = std::max(cell, 1.0e-4f);

    // rigid bodies and colliders
    const uint32_t B = uint32_t(w.bodies.size());
    w.bodyPos.clear(); w.bodyRot.clear(); w.bodyLin.clear(); w.bodyAng.clear(); w.bodyScale.clear();
    w.bodyInvI.clear(); w.bodyTypes.clear(); w.bodyKinPos.clear(); w.bodyKinRot.clear(); w.bodyKinFlags.clear();
    for (const cn_rigid_body_desc &b : w.bodies) {
        const float inv = (b.body_type == CN_BODY_DYNAMIC && b.mass > 0.0f) ? 1.0f / b.mass : 0.0f;
        w.bodyPos.insert(w.bodyPos.end(), {b.position[0], b.position[1], b.position[2], inv});
        w.bodyRot.insert(w.bodyRot.end(), {b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]});
        w.bodyLin.insert(w.bodyLin.end(), {0.f, 0.f, 0.f, 0.f});
        w.bodyAng.insert(w.bodyAng.end(), {0.f, 0.f, 0.f, 0.f});
        w.bodyScale.insert(w.bodyScale.end(), {b.scale[0], b.scale[1], b.scale[2], 0.f});
        w.bodyInvI.insert(w.bodyInvI.end(), {b.inverse_inertia_local[0], b.inverse_inertia_local[1],
                                             b.inverse_inertia_local[2], 0.f});
        w.bodyTypes.push_back(b.body_type);
        w.bodyKinPos.insert(w.bodyKinPos.end(), {b.position[0], b.position[1], b.position[2], 0.f});
        w.bodyKinRot.insert(w.bodyKinRot.end(), {b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]});
        w.bodyKinFlags.push_back(0u);
    }
    std::vector<std::vector<uint32_t>> bodyCols(B);
    w.colGeo.clear(); w.colBp.clear(); w.colMat.clear();
    for (uint32_t c = 0; c < w.colliders.size(); ++c) {
        const cn_collider_desc &d = w.colliders[c];
        if (d.body >= B) return CN_ERR_INVALID_ARGUMENT;
        bodyCols[d.body].push_back(c);
        cn_collider_geometry g{};
        std::memcpy(g.shape_params, d.shape_params, sizeof(g.shape_params));
        g.local_position[0] = d.local_position[0]; g.local_position[1] = d.local_position[1];
        g.local_position[2] = d.local_position[2];
        std::memcpy(g.local_orientation, d.local_orientation, sizeof(g.local_orientation));
        w.colGeo.push_back(g);
        cn_collider_broadphase bp{};
        bp.owner_body = d.body;
        bp.shape_type = d.shape_type;
        bp.environment_index = d.environment_index;
        bp.collision_layer = d.collision_layer == 0u ? 1u : d.collision_layer;
        bp.collision_mask = d.collision_mask;
        bp.enabled_flag = d.enabled ? 1u : 0u;
        w.colBp.push_back(bp);
        // normalizeColliderState (physics_world.cpp:3998-4007) + toColliderMaterial (:86-89)
        const float fr = std::max(d.friction, 0.0f);
        const float sf = d.static_friction < 0.0f ? fr : std::max(d.static_friction, 0.0f);
        const float rs = std::min(std::max(d.restitution, 0.0f), 1.0f);
        w.colMat.insert(w.colMat.end(), {fr, rs, 0.0f, sf});
    }
    w.bodyColRanges.assign(size_t(B) * 2, 0u);
    w.bodyColIdx.clear();
    for (uint32_t b = 0; b < B; ++b) {
        w.bodyColRanges[2 * b] = uint32_t(w.bodyColIdx.size());
        w.bodyColRanges[2 * b + 1] = uint32_t(bodyCols[b].size());
        w.bodyColIdx.insert(w.bodyColIdx.end(), bodyCols[b].begin(), bodyCols[b].end());
    }
    packSurfaces(w, softOff, clothOff);
    packLayoutMapping(w);
    return CN_OK;
}

template <class T> T *ptr(std::vector<T> &v) { return v.empty() ? nullptr : v.data(); }

} // namespace

extern "C" {

CN_API void cn_soft_body_grid_desc_defaults(cn_soft_body_grid_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->size[0] = d->size[1] = d->size[2] = 1.0f;
    d->target_particle_spacing = 0.25f;
    d->rest_transform.rotation[3] = 1.0f;
    d->rest_transform.scale[0] = d->rest_transform.scale[1] = d->rest_transform.scale[2] = 1.0f;
    d->particle_mass = 1.0f;
    d->particle_radius = 0.125f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
    d->material.static_friction = -1.0f;
}

CN_API void cn_fluid_grid_desc_defaults(cn_fluid_grid_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->size[0] = d->size[1] = d->size[2] = 1.0f;
    d->target_particle_spacing = 0.1f;
    d->rest_transform.rotation[3] = 1.0f;
    d->rest_transform.scale[0] = d->rest_transform.scale[1] = d->rest_transform.scale[2] = 1.0f;
    d->particle_mass = 1.0f;
    d->particle_radius = 0.05f;
    d->viscosity = 0.01f;
    d->gravity_scale = 1.0f;
    d->cfl_coefficient = 1.0f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
    d->material.static_friction = -1.0f;
}

CN_API void cn_cloth_grid_desc_defaults(cn_cloth_grid_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->resolution[0] = d->resolution[1] = 8;
    d->size[0] = d->size[1] = 1.0f;
    d->rest_transform.rotation[3] = 1.0f;
    d->rest_transform.scale[0] = d->rest_transform.scale[1] = d->rest_transform.scale[2] = 1.0f;
    d->particle_mass = 1.0f;
    d->particle_radius = 0.02f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
    d->material.static_friction = -1.0f;
}

CN_API void cn_strand_desc_defaults(cn_strand_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->particle_mass = 1.0f;
    d->particle_radius = 0.01f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
    d->material.static_friction = -1.0f;
}

CN_API void cn_rigid_body_desc_defaults(cn_rigid_body_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->orientation[3] = 1.0f;
    d->scale[0] = d->scale[1] = d->scale[2] = 1.0f;
    d->mass = 1.0f;
}

CN_API void cn_collider_desc_defaults(cn_collider_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->shape_params[0] = 0.5f;
    d->local_orientation[3] = 1.0f;
    d->enabled = 1u;
    d->friction = 0.5f;
    d->static_friction = -1.0f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
}

CN_API cn_status cn_world_create(cn_world **out)
{
    if (!out) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_create: null output");
    *out = new cn_world();
    return CN_OK;
}

CN_API void cn_world_destroy(cn_world *w) { delete w; }

namespace {
cn_status addSoftBody(cn_world *w, SoftBody &&sb, const cn_soft_body_grid_desc *d, uint32_t *out, const char *what)
{
    if (d->static_particle_indices && d->static_particle_count)
        sb.staticIdx.assign(d->static_particle_indices, d->static_particle_indices + d->static_particle_count);
    std::sort(sb.staticIdx.begin(), sb.staticIdx.end());
    sb.staticIdx.erase(std::unique(sb.staticIdx.begin(), sb.staticIdx.end()), sb.staticIdx.end());
    sb.desc.static_particle_indices = nullptr;
    const std::string err = buildSoftBody(sb);
    if (!err.empty()) return cn::setError(CN_ERR_INVALID_ARGUMENT, std::string(what) + ": " + err);
    if (out) *out = uint32_t(w->softBodies.size());
    w->softBodies.push_back(std::move(sb));
    return CN_OK;
}
} // namespace

CN_API cn_status cn_world_add_soft_body_grid(cn_world *w, const cn_soft_body_grid_desc *d, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_soft_body_grid: null argument");
    w->packed = false;
    SoftBody sb;
    sb.desc = *d;
    sb.source = SoftSource::RegularGrid;
    return addSoftBody(w, std::move(sb), d, out, "cn_world_add_soft_body_grid");
}

CN_API cn_status cn_world_add_soft_body_tet_mesh(cn_world *w, const cn_soft_body_grid_desc *d, const float *positions,
                                                 uint32_t vertex_count, const uint32_t *tet_indices,
                                                 uint32_t tet_count, uint32_t *out)
{
    if (!w || !d || (vertex_count && !positions) || (tet_count && !tet_indices))
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_soft_body_tet_mesh: null argument");
    w->packed = false;
    SoftBody sb;
    sb.desc = *d;
    sb.source = SoftSource::TetMesh;
    for (uint32_t i = 0; i < vertex_count; ++i)
        sb.srcPositions.push_back(v3{positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]});
    sb.srcTets.assign(tet_indices, tet_indices + size_t(tet_count) * 4u);
    return addSoftBody(w, std::move(sb), d, out, "cn_world_add_soft_body_tet_mesh");
}

CN_API cn_status cn_world_add_soft_body_tetgen(cn_world *w, const cn_soft_body_grid_desc *d, const char *node_file,
                                               const char *ele_file, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_soft_body_tetgen: null argument");
    w->packed = false;
    SoftBody sb;
    sb.desc = *d;
    sb.source = SoftSource::TetMesh;
    const std::string err = loadTetGen(node_file, ele_file, sb.srcPositions, sb.srcTets);
    if (!err.empty()) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_soft_body_tetgen: " + err);
    return addSoftBody(w, std::move(sb), d, out, "cn_world_add_soft_body_tetgen");
}

CN_API cn_status cn_world_add_soft_body_meshfree(cn_world *w, const cn_soft_body_grid_desc *d, const float *positions,
                                                 uint32_t particle_count, uint32_t neighbour_count, uint32_t *out)
{
    if (!w || !d || (particle_count && !positions))
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_soft_body_meshfree: null argument");
    w->packed = false;
    SoftBody sb;
    sb.desc = *d;
    sb.source = SoftSource::Meshfree;
    sb.neighbourCount = neighbour_count;
    for (uint32_t i = 0; i < particle_count; ++i)
        sb.srcPositions.push_back(v3{positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]});
    return addSoftBody(w, std::move(sb), d, out, "cn_world_add_soft_body_meshfree");
}

CN_API cn_status cn_world_add_fluid_grid(cn_world *w, const cn_fluid_grid_desc *d, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_fluid_grid: null argument");
    w->packed = false;
    if (!(d->target_particle_spacing > 0.0f)) return cn::setError(CN_ERR_INVALID_ARGUMENT, "fluid: spacing must be > 0");
    Fluid f;
    f.desc = *d;
    buildFluid(f);
    if (out) *out = uint32_t(w->fluids.size());
    w->fluids.push_back(std::move(f));
    return CN_OK;
}

CN_API cn_status cn_world_add_cloth_grid(cn_world *w, const cn_cloth_grid_desc *d, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_cloth_grid: null argument");
    w->packed = false;
    Cloth c;
    c.desc = *d;
    if (d->static_particle_indices && d->static_particle_count)
        c.staticIdx.assign(d->static_particle_indices, d->static_particle_indices + d->static_particle_count);
    c.desc.static_particle_indices = nullptr;
    if (buildCloth(c) != CN_OK) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cloth: static index out of range");
    if (out) *out = uint32_t(w->cloths.size());
    w->cloths.push_back(std::move(c));
    return CN_OK;
}

CN_API cn_status cn_world_add_strand(cn_world *w, const cn_strand_desc *d, uint32_t *out)
{
    if (!w || !d || !d->rest_positions)
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_strand: null argument");
    w->packed = false;
    Strand st;
    st.desc = *d;
    for (uint32_t i = 0; i < d->rest_position_count; ++i)
        st.rest.push_back(v3{d->rest_positions[3 * i], d->rest_positions[3 * i + 1], d->rest_positions[3 * i + 2]});
    if (d->static_particle_indices && d->static_particle_count)
        st.staticIdx.assign(d->static_particle_indices, d->static_particle_indices + d->static_particle_count);
    st.desc.rest_positions = nullptr;
    st.desc.static_particle_indices = nullptr;
    if (buildStrand(st) != CN_OK)
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "strand: needs >= 2 distinct rest positions");
    if (out) *out = uint32_t(w->strands.size());
    w->strands.push_back(std::move(st));
    return CN_OK;
}

CN_API cn_status cn_world_add_rigid_body(cn_world *w, const cn_rigid_body_desc *d, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_rigid_body: null argument");
    w->packed = false;
    if (d->body_type > CN_BODY_DYNAMIC) return cn::setError(CN_ERR_INVALID_ARGUMENT, "rigid body: unknown body type");
    if (out) *out = uint32_t(w->bodies.size());
    w->bodies.push_back(*d);
    return CN_OK;
}

CN_API cn_status cn_world_add_collider(cn_world *w, const cn_collider_desc *d, uint32_t *out)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_collider: null argument");
    w->packed = false;
    if (d->body >= w->bodies.size()) return cn::setError(CN_ERR_INVALID_ARGUMENT, "collider: body index out of range");
    if (d->shape_type > CN_COLLIDER_CAPSULE) return cn::setError(CN_ERR_INVALID_ARGUMENT, "collider: unknown shape");
    if (out) *out = uint32_t(w->colliders.size());
    w->colliders.push_back(*d);
    return CN_OK;
}

CN_API void cn_rigid_proxy_desc_defaults(cn_rigid_proxy_desc *d)
{
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->material.static_friction = -1.0f;
    d->collision_layer = 1u;
    d->collision_mask = 0xffffffffu;
}

CN_API cn_status cn_world_set_rigid_proxy_particles(cn_world *w, const cn_rigid_proxy_desc *d)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_set_rigid_proxy_particles: null argument");
    if (d->body >= w->bodies.size()) return cn::setError(CN_ERR_INVALID_ARGUMENT, "rigid proxies: body index out of range");
    if (d->count && !d->local_positions) return cn::setError(CN_ERR_INVALID_ARGUMENT, "rigid proxies: null positions");
    w->packed = false;
    RigidProxies rp;
    rp.desc = *d;
    rp.desc.local_positions = nullptr;
    rp.desc.radius = std::max(d->radius, 0.0f);
    for (uint32_t i = 0; i < d->count; ++i)
        rp.local.push_back(v3{d->local_positions[3 * i], d->local_positions[3 * i + 1], d->local_positions[3 * i + 2]});
    for (RigidProxies &r : w->proxies)
        if (r.desc.body == d->body) {
            r = std::move(rp);
            return CN_OK;
        }
    w->proxies.push_back(std::move(rp));
    return CN_OK;
}

CN_API cn_status cn_world_particle_layout_mapping(cn_world *w, cn_particle_layout_mapping *o)
{
    if (!w || !o) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_particle_layout_mapping: null argument");
    if (!w->packed) {
        const cn_status st = pack(*w);
        if (st != CN_OK) return cn::setError(st, "cn_world_particle_layout_mapping: invalid world");
        w->packed = true;
    }
    std::memset(o, 0, sizeof(*o));
    o->particle_count = uint32_t(w->radii.size());
    o->soft_body_count = uint32_t(w->softBodies.size());
    o->cloth_count = uint32_t(w->cloths.size());
    o->fluid_count = uint32_t(w->fluids.size());
    o->strand_count = uint32_t(w->strands.size());
    o->layout_revision = w->layoutRevision;
    o->environment_indices = ptr(w->lmEnv);
    o->particle_kinds = ptr(w->kinds);
    o->owner_types = ptr(w->ownerTypes);
    o->owner_indices = ptr(w->ownerIdx);
    o->strand_ids = ptr(w->lmStrandId);
    o->strand_orders = ptr(w->lmStrandOrder);
    o->strand_roles = ptr(w->lmStrandRole);
    o->owning_soft_body_indices = ptr(w->lmOwningSoft);
    o->particle_material_indices = ptr(w->matIdx);
    o->fluid_material_indices = ptr(w->fluidMatIdx);
    o->phases = ptr(w->lmPhase);
    o->collision_layers = ptr(w->lmLayer);
    o->collision_masks = ptr(w->lmMask);
    o->adjacency_offsets = ptr(w->adjOff);
    o->adjacency_counts = ptr(w->adjCnt);
    auto ranges = [](cn_world::OwnerRanges &r) {
        cn_particle_owner_ranges out{};
        out.count = uint32_t(r.ids.size());
        out.ids = ptr(r.ids);
        out.environment_indices = ptr(r.env);
        out.particle_offsets = ptr(r.off);
        out.particle_counts = ptr(r.cnt);
        return out;
    };
    o->soft_bodies = ranges(w->lmSoft);
    o->cloths = ranges(w->lmCloth);
    o->fluids = ranges(w->lmFluid);
    o->strands = ranges(w->lmStrand);
    return CN_OK;
}

CN_API cn_status cn_world_get_soa(cn_world *w, cn_world_soa *o)
{
    if (!w || !o) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_get_soa: null argument");
    if (!w->packed) {
        const cn_status st = pack(*w);
        if (st != CN_OK) return cn::setError(st, "cn_world_get_soa: invalid world");
        w->packed = true;
    }
    std::memset(o, 0, sizeof(*o));
    o->particle_count = uint32_t(w->radii.size());
    o->positions_inv_mass = ptr(w->x);
    o->velocities = ptr(w->v);
    o->radii = ptr(w->radii);
    o->kinds = ptr(w->kinds);
    o->metadata = ptr(w->meta);
    o->material_indices = ptr(w->matIdx);
    o->fluid_material_indices = ptr(w->fluidMatIdx);
    o->owner_types = ptr(w->ownerTypes);
    o->owner_indices = ptr(w->ownerIdx);
    o->adjacency_offsets = ptr(w->adjOff);
    o->adjacency_counts = ptr(w->adjCnt);
    o->adjacency_indices = ptr(w->adjIdx);
    o->adjacency_index_count = uint32_t(w->adjIdx.size());
    o->particle_grid_cell_size = w->cellSize;
    o->contact_material_count = uint32_t(w->contactMaterials.size() / 4);
    o->contact_materials = ptr(w->contactMaterials);
    o->fluid_material_count = uint32_t(w->fluidMaterials.size());
    o->fluid_materials = ptr(w->fluidMaterials);
    o->edge_count = uint32_t(w->edges.size()); o->edges = ptr(w->edges);
    o->dihedral_count = uint32_t(w->dihedrals.size()); o->dihedrals = ptr(w->dihedrals);
    o->tet_count = uint32_t(w->tets.size()); o->tets = ptr(w->tets);
    o->strand_segment_count = uint32_t(w->segs.size()); o->strand_segments = ptr(w->segs);
    o->strand_segment_orientations = ptr(w->segOrient);
    o->strand_joint_count = uint32_t(w->joints.size()); o->strand_joints = ptr(w->joints);
    o->strand_distance_count = uint32_t(w->dists.size()); o->strand_distances = ptr(w->dists);
    o->rigid_body_count = uint32_t(w->bodies.size());
    o->body_positions_inv_mass = ptr(w->bodyPos);
    o->body_orientations = ptr(w->bodyRot);
    o->body_linear_velocities = ptr(w->bodyLin);
    o->body_angular_velocities = ptr(w->bodyAng);
    o->body_scales = ptr(w->bodyScale);
    o->body_inverse_inertia = ptr(w->bodyInvI);
    o->body_types = ptr(w->bodyTypes);
    o->body_kinematic_target_positions = ptr(w->bodyKinPos);
    o->body_kinematic_target_orientations = ptr(w->bodyKinRot);
    o->body_kinematic_target_flags = ptr(w->bodyKinFlags);
    o->body_collider_ranges = ptr(w->bodyColRanges);
    o->body_collider_indices = ptr(w->bodyColIdx);
    o->body_collider_index_count = uint32_t(w->bodyColIdx.size());
    o->collider_count = uint32_t(w->colliders.size());
    o->collider_geometry = ptr(w->colGeo);
    o->collider_broadphase = ptr(w->colBp);
    o->collider_materials = ptr(w->colMat);
    cn_surface_render_data &sd = w->sData;
    sd = cn_surface_render_data{};
    sd.vertex_count = uint32_t(w->sBind.size());
    sd.vertex_bindings = ptr(w->sBind);
    sd.fallback_normals = ptr(w->sFallback);
    sd.vertex_triangle_ranges = ptr(w->sRanges);
    sd.vertex_triangle_index_count = uint32_t(w->sIdx.size());
    sd.vertex_triangle_indices = ptr(w->sIdx);
    sd.triangle_count = uint32_t(w->sTri.size() / 4);
    sd.triangle_particle_indices = ptr(w->sTri);
    sd.surface_count = uint32_t(w->sSurf.size() / 2);
    sd.surface_particle_ranges = ptr(w->sSurf);
    o->surface_render = (sd.vertex_count || sd.surface_count) ? &sd : nullptr;
    o->rigid_proxy_local_positions = w->proxyLocal.empty() ? nullptr : w->proxyLocal.data();
    o->body_proxy_contact_materials = w->bodyProxyMat.empty() ? nullptr : w->bodyProxyMat.data();
    return CN_OK;
}

CN_API void cn_surface_mesh_desc_defaults(cn_surface_mesh_desc *d)
{
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->match_epsilon = 1.0e-3f; // kSoftBodyVertexMatchEpsilon (world.cpp:17)
}

CN_API cn_status cn_world_add_surface_mesh(cn_world *w, const cn_surface_mesh_desc *d, uint32_t *out_first_vertex)
{
    if (!w || !d) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_add_surface_mesh: null argument");
    cn_world::SurfaceMesh m;
    const std::string err = bindSurfaceMesh(*w, *d, m);
    if (!err.empty()) return cn::setError(CN_ERR_INVALID_ARGUMENT, err);
    uint32_t first = 0;
    for (const auto &e : w->surfaceMeshes) first += uint32_t(e.bindings.size());
    if (out_first_vertex) *out_first_vertex = first;
    w->surfaceMeshes.push_back(std::move(m));
    w->customSurface = false;
    w->packed = false;
    return CN_OK;
}

CN_API cn_status cn_world_set_surface_render(cn_world *w, const cn_surface_render_data *d)
{
    if (!w) return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_set_surface_render: null world");
    w->packed = false;
    if (!d) {
        w->customSurface = false;
        return CN_OK;
    }
    auto need = [](uint32_t n, const void *p) { return n == 0u || p != nullptr; };
    if (!need(d->vertex_count, d->vertex_bindings) || !need(d->vertex_count, d->fallback_normals) ||
        !need(d->vertex_count, d->vertex_triangle_ranges) ||
        !need(d->vertex_triangle_index_count, d->vertex_triangle_indices) ||
        !need(d->triangle_count, d->triangle_particle_indices) || !need(d->surface_count, d->surface_particle_ranges))
        return cn::setError(CN_ERR_INVALID_ARGUMENT, "cn_world_set_surface_render: missing array");
    w->customSurface = true;
    w->sBind.assign(d->vertex_bindings, d->vertex_bindings + d->vertex_count);
    w->sFallback.assign(d->fallback_normals, d->fallback_normals + size_t(d->vertex_count) * 4);
    w->sRanges.assign(d->vertex_triangle_ranges, d->vertex_triangle_ranges + d->vertex_count);
    w->sIdx.assign(d->vertex_triangle_indices, d->vertex_triangle_indices + d->vertex_triangle_index_count);
    w->sTri.assign(d->triangle_particle_indices, d->triangle_particle_indices + size_t(d->triangle_count) * 4);
    w->sSurf.assign(d->surface_particle_ranges, d->surface_particle_ranges + size_t(d->surface_count) * 2);
    return CN_OK;
}

} // extern "C"
