"""Dynamic rigid bodies in the particle path: rigid predict with orientation integration
(physics_rigid_predict.cs.hlsl:73-81), two-way particle-rigid position and velocity contacts
(physics_particle_rigid_solve_contacts.cs.hlsl:64-141, ..._solve_contact_velocities.cs.hlsl),
the bodies' summed corrections applied per iteration (physics_rigid_apply_corrections,
physics_rigid_apply_contact_velocities) and their velocities from the pose change
(physics_rigid_update_velocities), also with fluid particles.  The reference sums a body's
corrections with float atomics, so GPU and oracle agree within tolerance, not bit for bit."""
import numpy as np
import pytest

from cn_physics import CNError, Solver, World, scenes, solver_desc
import cn_oracle


def tissue_and_sphere(offset=0.03, mass=0.5, radius=0.08, spin=False):
    w = World()
    pinned = [x * 3 * 5 + z for x in range(5) for z in range(5)]  # bottom layer of the 5x3x5 block
    w.add_soft_body_grid((0.4, 0.2, 0.4), 0.1, position=(0.0, 0.1, 0.0), radius=0.04, edge_compliance=1e-5,
                         volume_compliance=1e-6, static_particles=pinned, friction=0.3)
    inv_i = 1.0 / (0.4 * mass * radius * radius)  # solid sphere
    b = w.add_rigid_body("dynamic", position=(offset, 0.35, 0.0), mass=mass, inverse_inertia=(inv_i,) * 3)
    w.add_collider(b, "sphere", (radius,), friction=0.4)
    soa = w.soa()
    if spin:
        np.ctypeslib.as_array(soa.body_angular_velocities, (4,))[:3] = (0.0, 3.0, 1.0)
    return w, b


def test_oracle_sphere_comes_to_rest_on_the_tissue():
    w, b = tissue_and_sphere()
    o = cn_oracle.Oracle(solver_desc(substeps=4, default_iterations=10), w.soa())
    for _ in range(60):
        o.step(1.0 / 60.0)
    p, q, lin, ang = o.read_rigid_bodies()
    assert 0.28 < p[b, 1] < 0.33                       # resting on the block top (0.2 + 0.04 + 0.08)
    assert np.linalg.norm(lin[b, :3]) < 0.01            # at rest
    assert abs(np.linalg.norm(q[b]) - 1.0) < 1e-6
    x, _, _ = o.read_particles()
    assert x[:, 1].max() < 0.26                         # the tissue top is pressed, not pierced


def fluid_tank_and_sphere(mass=0.2, radius=0.06):
    """A small fluid tank (static walls) with a light dynamic sphere dropped into it: fluid
    particles take particle-rigid contacts against the dynamic body (physics_particle_count_
    particle_rigid_candidates.cs.hlsl: solid particles against every body, fluid ones against
    dynamic bodies) and push it back (the body's share, physics_particle_rigid_solve_contacts.cs.hlsl:97-140)."""
    w, desc, dt = scenes.dam_break(nx=12, ny=6, nz=12, box=(0.6, 0.6, 0.6))
    inv_i = 1.0 / (0.4 * mass * radius * radius)
    b = w.add_rigid_body("dynamic", position=(0.3, 0.42, 0.3), mass=mass, inverse_inertia=(inv_i,) * 3)
    w.add_collider(b, "sphere", (radius,), friction=0.2)
    w.soa()
    return w, desc, dt, b


def test_oracle_sphere_enters_the_fluid_and_is_held_up():
    w, desc, dt, b = fluid_tank_and_sphere()
    o = cn_oracle.Oracle(desc, w.soa())
    heights = []
    for _ in range(150):
        o.step(dt)
        heights.append(o.read_rigid_bodies()[0][b, 1])
    x, _, _ = o.read_particles()
    assert min(heights) < 0.33                          # it went into the fluid layer (top ~0.33)
    assert 0.3 < heights[-1] < 0.5                      # and floats, held up by the fluid
    assert np.isfinite(x).all()


@pytest.mark.gpu
def test_fluid_with_a_dynamic_body_against_the_oracle():
    w, desc, dt, b = fluid_tank_and_sphere()
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for frame in range(45):
        gpu.step(dt)
        ora.step(dt)
        if frame == 34:   # before the first contact: the same sums in the same order
            for a, c in zip(gpu.read_particles(), ora.read_particles()):
                np.testing.assert_allclose(a, c, rtol=1e-5, atol=1e-6)
    # the first contacts: the body's share is summed with float atomics (GPU) or in pair order
    # (oracle), as the reference's order is the GPU's schedule
    for a, c in zip(gpu.read_particles(), ora.read_particles()):
        np.testing.assert_allclose(a, c, rtol=1e-4, atol=1e-4)
    gb, ob = gpu.read_rigid_bodies(), ora.read_rigid_bodies()
    np.testing.assert_allclose(gb[0][b, :3], ob[0][b, :3], rtol=1e-4, atol=1e-4)
    assert gpu.validate_gpu_meta()["status"] == "OK"


@pytest.mark.gpu
def test_free_dynamic_body_integrates_like_the_oracle():
    w = World()
    b = w.add_rigid_body("dynamic", position=(0.0, 1.0, 0.0), mass=2.0, inverse_inertia=(3.0, 2.0, 1.0))
    w.add_collider(b, "box", (0.1, 0.05, 0.2))
    soa = w.soa()
    np.ctypeslib.as_array(soa.body_linear_velocities, (4,))[:3] = (0.5, 2.0, 0.0)
    np.ctypeslib.as_array(soa.body_angular_velocities, (4,))[:3] = (1.0, -2.0, 0.5)
    desc = solver_desc(substeps=4)
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(30):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    for a, o in zip(gpu.read_rigid_bodies(), ora.read_rigid_bodies()):
        np.testing.assert_allclose(a, o, rtol=1e-5, atol=1e-6)   # sin / cos: CUDA's and libm's last bits


@pytest.mark.gpu
@pytest.mark.parametrize("spin", [False, True])
def test_sphere_on_tissue_two_way_coupling_matches_the_oracle(spin):
    w, b = tissue_and_sphere(spin=spin)
    desc = solver_desc(substeps=4, default_iterations=10)
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for k in range(12):  # fall and impact
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    for a, o in zip(gpu.read_rigid_bodies(), ora.read_rigid_bodies()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-5)
    for a, o in zip(gpu.read_particles(), ora.read_particles()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-5)
    for k in range(48):  # settling: the drift bar
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    pg, qg, lg, _ = gpu.read_rigid_bodies()
    po, qo, lo, _ = ora.read_rigid_bodies()
    assert np.abs(pg[b, :3] - po[b, :3]).max() < 1e-3
    assert np.linalg.norm(lg[b, :3]) < 0.02 and 0.28 < pg[b, 1] < 0.33
    assert gpu.validate_gpu_meta()["status"] == "OK"
