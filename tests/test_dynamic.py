"""Dynamic rigid bodies in the particle path: rigid predict with orientation integration
(physics_rigid_predict.cs.hlsl:73-81), two-way particle-rigid position and velocity contacts
(physics_particle_rigid_solve_contacts.cs.hlsl:64-141, ..._solve_contact_velocities.cs.hlsl),
the bodies' summed corrections applied per iteration (physics_rigid_apply_corrections,
physics_rigid_apply_contact_velocities) and their velocities from the pose change
(physics_rigid_update_velocities).  The reference sums a body's corrections with float atomics,
so GPU and oracle agree within tolerance, not bit for bit."""
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


@pytest.mark.gpu
def test_fluid_with_dynamic_bodies_is_rejected():
    w, _ = tissue_and_sphere()
    w.add_fluid_grid((0.1, 0.1, 0.1), 0.05, position=(1.0, 0.5, 0.0), radius=0.03)
    sv = Solver(solver_desc())
    with pytest.raises(CNError):
        sv.sync_world(w.soa())


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
