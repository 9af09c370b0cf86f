// cn_internal.h -- helpers shared by the host translation units behind the C ABI: error
// reporting, the device arena, incidence tables and the solver constants.
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cn_physics.h"
#include "cn_device.h"

namespace cn {

// Records `message` as this thread's last error and returns `status`.
cn_status setError(cn_status status, const std::string &message);
void clearError();


inline uint32_t nextPow2(uint32_t v)
{
    if (v <= 1u) return 1u;
    --v;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    return v + 1u;
}
inline uint32_t resolveIter(uint32_t o, uint32_t d) { return o > 0u ? o : d; }

// Bump allocator over one device allocation.  Running a layout with a null base sizes it.
class Arena {
public:
    void reset(uint8_t *base) { base_ = base; offset_ = 0; }
    template <class T> T *take(size_t count)
    {
        const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        T *p = base_ ? reinterpret_cast<T *>(base_ + offset_) : nullptr;
        offset_ += count ? bytes : 0;
        return count ? p : nullptr;
    }
    size_t size() const { return offset_; }

private:
    uint8_t *base_ = nullptr;
    size_t offset_ = 0;
};

// Per-particle incidence lists in ascending constraint order
// (physics_scene_gpu_state.cpp:3273-3420): ranges[p] = (start, count), inc = (constraint, slot);
// dst[c * perConstraint + k] = the position of (c, k) in inc (0xffffffff when entry k names no
// particle), the gather slot of that entry's correction record.
struct Incidence {
    std::vector<uint2> ranges, inc;
    std::vector<uint32_t> dst;
};
template <class F> Incidence buildIncidence(uint32_t n, uint32_t constraints, uint32_t perConstraint, F &&particlesOf)
{
    std::vector<uint32_t> counts(n, 0);
    for (uint32_t c = 0; c < constraints; ++c)
        for (uint32_t k = 0; k < perConstraint; ++k) {
            const uint32_t p = particlesOf(c, k);
            if (p < n) ++counts[p];
        }
    Incidence out;
    out.ranges.resize(n);
    uint32_t run = 0;
    for (uint32_t i = 0; i < n; ++i) {
        out.ranges[i] = make_uint2(run, counts[i]);
        run += counts[i];
    }
    out.inc.resize(run);
    out.dst.assign(size_t(constraints) * perConstraint, 0xffffffffu);
    std::vector<uint32_t> fill(n, 0);
    for (uint32_t c = 0; c < constraints; ++c)
        for (uint32_t k = 0; k < perConstraint; ++k) {
            const uint32_t p = particlesOf(c, k);
            if (p >= n) continue;
            const uint32_t at = out.ranges[p].x + fill[p]++;
            out.inc[at] = make_uint2(c, k);
            out.dst[size_t(c) * perConstraint + k] = at;
        }
    return out;
}
// The particles a family touches, as one window [lo, hi) over its incidence ranges ((0, 0) when none).
inline uint2 incidenceWindow(const Incidence &I)
{
    uint32_t lo = uint32_t(I.ranges.size()), hi = 0;
    for (uint32_t i = 0; i < I.ranges.size(); ++i)
        if (I.ranges[i].y) {
            lo = std::min(lo, i);
            hi = i + 1;
        }
    return lo < hi ? make_uint2(lo, hi) : make_uint2(0u, 0u);
}

// Greedy graph colouring of one constraint family: constraint c, in ascending order, takes the
// lowest colour no earlier constraint sharing one of its elements has (elementOf(c, k) >= n is
// no element).  order = the constraints grouped by colour, ascending within a colour;
// starts[k] .. starts[k + 1] = colour k.  Per-element used-colour bitsets of `words` 64-bit
// words, widened when a constraint needs a colour past them.
struct Colouring {
    std::vector<uint32_t> order, starts;
    uint32_t colours() const { return starts.empty() ? 0u : uint32_t(starts.size() - 1); }
};
template <class F> Colouring colourGreedy(uint32_t n, uint32_t constraints, uint32_t perConstraint, F &&elementOf)
{
    Colouring out;
    if (constraints == 0) return out;
    uint32_t words = 1;
    std::vector<uint64_t> used(size_t(n) * words, 0ull);
    std::vector<uint32_t> colourOf(constraints, 0u);
    std::vector<uint32_t> el(perConstraint);
    uint32_t colours = 0;
    for (uint32_t c = 0; c < constraints; ++c) {
        uint32_t m = 0;
        for (uint32_t k = 0; k < perConstraint; ++k) {
            const uint32_t e = elementOf(c, k);
            if (e < n) el[m++] = e;
        }
        uint32_t colour = words * 64u;
        for (uint32_t w = 0; w < words && colour == words * 64u; ++w) {
            uint64_t taken = 0;
            for (uint32_t k = 0; k < m; ++k) taken |= used[size_t(el[k]) * words + w];
            if (~taken) colour = w * 64u + uint32_t(__builtin_ctzll(~taken));
        }
        if (colour >= words * 64u) { // every colour of the current words is taken: widen
            std::vector<uint64_t> wider(size_t(n) * (words + 1), 0ull);
            for (size_t e = 0; e < n; ++e)
                for (uint32_t w = 0; w < words; ++w) wider[e * (words + 1) + w] = used[e * words + w];
            used.swap(wider);
            ++words;
        }
        for (uint32_t k = 0; k < m; ++k) used[size_t(el[k]) * words + colour / 64u] |= 1ull << (colour % 64u);
        colourOf[c] = colour;
        colours = std::max(colours, colour + 1u);
    }
    out.starts.assign(colours + 1u, 0u);
    for (uint32_t c = 0; c < constraints; ++c) ++out.starts[colourOf[c] + 1u];
    for (uint32_t k = 0; k < colours; ++k) out.starts[k + 1u] += out.starts[k];
    out.order.resize(constraints);
    std::vector<uint32_t> fill(out.starts.begin(), out.starts.end() - 1);
    for (uint32_t c = 0; c < constraints; ++c) out.order[fill[colourOf[c]]++] = c;
    return out;
}

// A batch scene's upload image (cn_batch.cpp): validated soft-tissue content in the pool's array
// layouts with the scene's own indices, and the device bytes it is charged against the budget.
struct SceneImage {
    std::vector<uint8_t> bytes;
    AdmitImage layout;
    uint64_t budgetBytes = 0;
    uint32_t colours[2] = {0, 0}; // edge and tet colours (coloured schedules)
};
// `coloured`: the image also carries the scene's edge and tet colourings (a batch created with a
// coloured XPBD schedule).
cn_status buildSceneImage(const cn_world_soa &w, uint32_t rigidPairsPerParticle, bool coloured, SceneImage &img);
// Copies the mutable state (particles, bodies, kinematic targets) of `w` into the image.
void refreshSceneImage(const cn_world_soa &w, SceneImage &img);
// Admits the image into the batch (ranges, one transfer, the device-side scatter).
cn_status batchAdmitImage(cn_batch *b, const SceneImage &img, uint32_t *scene_id);
uint32_t batchRigidPairsPerParticle(const cn_batch *b);
bool batchColoured(const cn_batch *b);

// Particle-rigid candidate pairs per particle (0 reads as the reference's 8).
inline uint32_t rigidPairsPerParticle(const cn_solver_desc &d)
{
    return d.particle_rigid_pairs_per_particle ? d.particle_rigid_pairs_per_particle : 8u;
}

// Solver constants of one substep, from the PhysicsSolverDesc mirror.
inline Config configFromDesc(const cn_solver_desc &d)
{
    Config c{};
    c.slop = d.contact.slop;
    c.softContactRelaxation = d.contact.soft_relaxation;
    c.softMaxCorrection = d.contact.soft_max_correction_per_iteration;
    c.restitutionVelocityThreshold = d.contact.restitution_velocity_threshold;
    c.restitutionPenetrationThreshold = d.contact.restitution_penetration_slop_multiplier * d.contact.slop;
    c.positionFrictionMinDistance = d.contact.position_friction_min_distance;
    c.softInternalRelaxation = d.soft.internal_relaxation;
    c.fluidSolveCoefficient = d.fluid.constraint_relaxation;
    c.fluidRelaxation = d.fluid.position_relaxation;
    c.fluidBoundaryDensityScale = d.fluid.boundary_density_scale;
    c.fluidBoundaryDeltaScale = d.fluid.boundary_delta_scale;
    c.fluidMaxUnderDensityRatio = d.fluid.max_under_density_ratio;
    c.gravity[0] = d.gravity[0]; c.gravity[1] = d.gravity[1]; c.gravity[2] = d.gravity[2];
    c.maxTranslationCorrection = d.rigid.max_translation_correction_per_iteration;
    c.maxRotationCorrection = d.rigid.max_rotation_correction_per_iteration;
    c.maxLinearVelocityCorrection = d.rigid.max_linear_velocity_correction_per_iteration;
    c.maxAngularVelocityCorrection = d.rigid.max_angular_velocity_correction_per_iteration;
    c.rigidRestitutionThreshold = d.contact.rigid_restitution_velocity_threshold;
    c.baumgarte = d.rigid.depenetration_baumgarte;
    c.depenetrationRelaxation = d.rigid.depenetration_relaxation;
    c.maxDepenetration = d.rigid.depenetration_max_correction_per_iteration;
    c.velocityPenetrationStiffness = d.rigid.velocity_penetration_stiffness;
    c.manifoldMergeDistance = d.contact.manifold_merge_slop_multiplier * d.contact.slop;
    return c;
}

// Moving (kinematic) colliders, then static ones, each ascending by index; disabled colliders
// and colliders of missing bodies are left out.  Returns the number of moving colliders.
inline uint32_t colliderQueryOrder(const cn_world_soa &w, std::vector<uint32_t> &order)
{
    order.clear();
    std::vector<uint32_t> stat;
    for (uint32_t c = 0; c < w.collider_count; ++c) {
        const cn_collider_broadphase &bp = w.collider_broadphase[c];
        if (bp.owner_body >= w.rigid_body_count || bp.enabled_flag == 0u) continue;
        if (w.body_types[bp.owner_body] == CN_BODY_STATIC) stat.push_back(c);
        else order.push_back(c);
    }
    const uint32_t moving = uint32_t(order.size());
    order.insert(order.end(), stat.begin(), stat.end());
    return moving;
}

} // namespace cn
