"""Rigid proxy particles: spheres carried with a rigid body
(physics_particle_sync_rigid_proxy_particles.cs.hlsl), colliding with particles through the
explicit contacts -- the body takes the proxy's share (physics_particle_solve_explicit_contacts,
..._solve_contact_velocities) -- and with other bodies' colliders through proxy contacts in the
rigid contact solve (physics_rigid_generate_proxy_contacts.cs.hlsl).  World packing follows
PhysicsWorld::rebuildSoftParticleLayout (physics_world.cpp:4931-5023): proxies first."""
import numpy as np
import pytest

from cn_physics import CNError, Solver, World, scenes, solver_desc
import cn_oracle

Q_Z30 = (0.0, 0.0, 0.2588190, 0.9659258)
DESC = dict(substeps=4, default_iterations=10)


def lattice(n=3, spacing=0.04):
    g = (np.arange(n) - (n - 1) / 2.0) * spacing
    return np.array([(x, y, z) for x in g for y in g for z in g], np.float32)


def qrot(q, v):
    q = np.asarray(q, np.float64)
    u, w = q[:3], q[3]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def proxy_drop(orientation=(0, 0, 0, 1), y0=0.3):
    """A dynamic body made only of 27 proxies (no colliders) dropped onto the ground box."""
    w = World()
    scenes.ground(w)
    b = w.add_rigid_body("dynamic", position=(0.0, y0, 0.0), orientation=orientation, mass=0.5,
                         inverse_inertia=(800.0,) * 3)
    w.set_rigid_proxy_particles(b, lattice(), 0.02, friction=0.5)
    return w, b


def tissue_and_proxies(body_type="dynamic", y0=0.3):
    """Pinned soft tissue (9 x 3 x 9 particles, 0.05 apart) with a proxy cluster above it."""
    w = World()
    pinned = [x * 3 * 9 + z for x in range(9) for z in range(9)]   # bottom layer
    w.add_soft_body_grid((0.4, 0.1, 0.4), 0.05, position=(0.0, 0.05, 0.0), radius=0.025, edge_compliance=1e-5,
                         volume_compliance=1e-6, static_particles=pinned, friction=0.3)
    kw = dict(mass=0.2, inverse_inertia=(2000.0,) * 3) if body_type == "dynamic" else {}
    b = w.add_rigid_body(body_type, position=(0.03, y0, 0.0), **kw)
    w.set_rigid_proxy_particles(b, lattice(), 0.025, friction=0.4)
    return w, b


def test_world_packs_proxies_first():
    w = World()
    w.add_soft_body_grid((0.2, 0.2, 0.2), 0.1, position=(0.0, 1.0, 0.0), radius=0.04)
    b0 = w.add_rigid_body("kinematic", position=(1.0, 2.0, 3.0), orientation=Q_Z30, scale=(2.0, 1.0, 1.0))
    b1 = w.add_rigid_body("static")
    w.set_rigid_proxy_particles(b0, [(0.1, 0.0, 0.0), (0.0, 0.2, 0.0)], 0.03, friction=0.7, layer=4)
    w.set_rigid_proxy_particles(b1, [(0.0, 0.0, 0.0)], 0.0)   # radius 0: skipped, as the reference does
    soa = w.soa()
    n = soa.particle_count
    owners = np.ctypeslib.as_array(soa.owner_types, (n,))
    idx = np.ctypeslib.as_array(soa.owner_indices, (n,))
    assert owners[:2].tolist() == [4, 4] and idx[:2].tolist() == [b0, b0] and (owners[2:] == 1).all()
    x = w.positions()
    local = np.ctypeslib.as_array(soa.rigid_proxy_local_positions, (n, 4))
    np.testing.assert_allclose(local[:2, :3], [(0.2, 0.0, 0.0), (0.0, 0.2, 0.0)], atol=1e-7)  # scaled
    assert (local[2:] == 0).all() and (x[:2, 3] == 0).all()
    want = np.array([qrot(Q_Z30, local[k, :3]) + (1.0, 2.0, 3.0) for k in range(2)])
    np.testing.assert_allclose(x[:2, :3], want, atol=1e-6)
    meta = w.array("metadata")
    # phase group past the soft body (proxy base = soft bodies + cloths + strands + fluids), no self collision
    assert meta[0, 1] == (1 + b0) and meta[0, 2] == 4
    mats = np.ctypeslib.as_array(soa.body_proxy_contact_materials, (2, 4))
    np.testing.assert_allclose(mats[b0], (0.7, 0.0, 0.0, 0.7))
    assert (mats[b1] == 0).all()


def sphere_collider_twin(orientation):
    """The proxy body of proxy_drop rebuilt from 27 sphere colliders at the proxy points."""
    w = World()
    scenes.ground(w)
    b = w.add_rigid_body("dynamic", position=(0.0, 0.3, 0.0), orientation=orientation, mass=0.5,
                         inverse_inertia=(800.0,) * 3)
    for l in lattice():
        w.add_collider(b, "sphere", (0.02,), local_position=tuple(map(float, l)), friction=0.5)
    return w, b


@pytest.mark.parametrize("orientation", [(0, 0, 0, 1), Q_Z30])
def test_oracle_proxy_body_moves_like_its_sphere_collider_twin(orientation):
    """A proxy against the ground box is the sphere-box primitive of a sphere collider at the proxy
    point, in the same contact order: the two bodies fall, land and settle identically."""
    w, b = proxy_drop(orientation)
    o = cn_oracle.Oracle(solver_desc(**DESC), w.soa())
    w2, b2 = sphere_collider_twin(orientation)
    o2 = cn_oracle.Oracle(solver_desc(**DESC), w2.soa())
    for _ in range(120):
        o.step(1.0 / 60.0)
        o2.step(1.0 / 60.0)
    for a, c in zip(o.read_rigid_bodies(), o2.read_rigid_bodies()):
        np.testing.assert_array_equal(a[b], c[b2])
    x, _, _ = o.read_particles()
    assert abs(x[:27, 1].min() - 0.02) < 3e-3            # the lowest proxies rest on the ground top
    m = o.meta()
    assert m["proxy_contacts"] > 0 and m["required_proxy_contacts"] == m["proxy_contacts"]


def test_oracle_tissue_holds_a_dynamic_proxy_body():
    w, b = tissue_and_proxies()
    o = cn_oracle.Oracle(solver_desc(**DESC), w.soa())
    for _ in range(90):
        o.step(1.0 / 60.0)
    p, _, lin, _ = o.read_rigid_bodies()
    x, _, _ = o.read_particles()
    assert 0.12 < p[b, 1] < 0.2                      # held by the tissue (top particle centres at 0.1)
    assert np.linalg.norm(lin[b, :3]) < 0.1
    assert x[27:, 1].max() < 0.11                    # the tissue is pressed, not lifted
    assert o.meta()["active_particle_contacts"] > 0


def pair(w, desc):
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    return gpu, cn_oracle.Oracle(desc, soa)


@pytest.mark.gpu
def test_kinematic_proxies_follow_the_body_and_press_the_tissue():
    w, b = tissue_and_proxies("kinematic", y0=0.18)
    gpu, ora = pair(w, solver_desc(**DESC))
    x0 = w.positions()
    top = np.where((np.abs(x0[:, 1] - 0.1) < 1e-3) & (np.arange(len(x0)) >= 27))[0]
    for k in range(12):
        target = (0.03, 0.18 - 0.004 * (k + 1), 0.0)
        gpu.set_kinematic_target(b, target, Q_Z30)
        ora.set_kinematic_target(b, target, Q_Z30)
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    xg, vg, _ = gpu.read_particles()
    xo, vo, _ = ora.read_particles()
    np.testing.assert_allclose(xg[:27], xo[:27], rtol=1e-6, atol=1e-6)   # the sync: same pose, same formula
    np.testing.assert_allclose(xg, xo, rtol=1e-4, atol=1e-5)             # float atomics in the contacts
    np.testing.assert_allclose(vg, vo, rtol=1e-4, atol=1e-4)
    assert xg[top, 1].mean() < 0.095                                     # the top layer is pressed down
    assert gpu.validate_gpu_meta()["status"] == "OK"


@pytest.mark.gpu
def test_dynamic_proxy_body_on_tissue_matches_the_oracle():
    w, b = tissue_and_proxies()
    gpu, ora = pair(w, solver_desc(**DESC))
    for _ in range(20):   # fall and impact
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    for a, o in zip(gpu.read_rigid_bodies(), ora.read_rigid_bodies()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-5)
    for a, o in zip(gpu.read_particles(), ora.read_particles()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-4)
    for _ in range(60):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    pg = gpu.read_rigid_bodies()[0]
    po = ora.read_rigid_bodies()[0]
    assert np.abs(pg[b, :3] - po[b, :3]).max() < 1e-3
    assert gpu.validate_gpu_meta()["status"] == "OK"


@pytest.mark.gpu
@pytest.mark.parametrize("orientation", [(0, 0, 0, 1), Q_Z30])
def test_proxy_body_drop_matches_the_oracle(orientation):
    w, b = proxy_drop(orientation)
    gpu, ora = pair(w, solver_desc(**DESC))
    for _ in range(20):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    for a, o in zip(gpu.read_rigid_bodies(), ora.read_rigid_bodies()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-5)
    m = gpu.validate_gpu_meta()
    om = ora.meta()
    assert m["status"] == "OK"
    assert m["required_proxy_rigid_contact_count"] == om["required_proxy_contacts"] > 0
    for _ in range(100):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    pg = gpu.read_rigid_bodies()[0]
    po = ora.read_rigid_bodies()[0]
    assert np.abs(pg[b, :3] - po[b, :3]).max() < 1e-3
    xg = gpu.read_particles()[0]
    assert abs(xg[:27, 1].min() - 0.02) < 3e-3


@pytest.mark.gpu
def test_proxy_particles_are_not_batched():
    from cn_physics import Batch, batch_desc
    w, _ = proxy_drop()
    bt = Batch(batch_desc(solver_desc(**DESC)))
    with pytest.raises(CNError):
        bt.add_scene(w.soa())


@pytest.mark.gpu
def test_small_rigid_pile_with_proxy_bodies_matches_the_oracle():
    """Spheres, capsules and boxes in two layers with proxy-particle bodies dropped on them: the
    same candidate pairs frame by frame while the pile forms, states within tolerance."""
    w, desc, dt, bodies = scenes.rigid_pile(layers=2, per_side=4)
    gpu, ora = pair(w, desc)
    for k in range(12):
        gpu.step(dt)
        ora.step(dt)
        m, om = gpu.validate_gpu_meta(), ora.meta()
        assert m["status"] == "OK"
        assert m["required_rigid_rigid_candidate_count"] == om["required_rigid_rigid_pairs"], k
        assert m["required_proxy_rigid_contact_count"] == om["required_proxy_contacts"], k
    pg, po = gpu.read_rigid_bodies()[0], ora.read_rigid_bodies()[0]
    assert np.abs(pg[:, :3] - po[:, :3]).max() < 1e-3   # the drift bar: contact order and float atomics


@pytest.mark.gpu
def test_kinematic_proxy_tool_stirs_fluid_like_the_oracle():
    """Proxy particles of a kinematic tool moving through a fluid block: explicit fluid-proxy
    contacts (the proxy side immovable), the fluid solve with its superset lists validated by each
    particle's move, GPU against the oracle."""
    w = World()
    w.add_fluid_grid((0.3, 0.2, 0.3), 0.02, position=(0.0, 0.11, 0.0), radius=0.012)
    scenes.ground(w)
    tool = w.add_rigid_body("kinematic", position=(0.0, 0.12, 0.0))
    rod = [(0.0, 0.025 * k - 0.05, 0.0) for k in range(5)]
    w.set_rigid_proxy_particles(tool, rod, 0.02, friction=0.2)
    desc = solver_desc(substeps=2, default_iterations=4, fluid_iterations=4)
    gpu, ora = pair(w, desc)
    touched = 0
    for k in range(6):
        target = (0.01 * (k + 1), 0.12, 0.0)
        gpu.set_kinematic_target(tool, target)
        ora.set_kinematic_target(tool, target)
        gpu.step(1.0 / 120.0)
        ora.step(1.0 / 120.0)
        n = gpu.validate_gpu_meta()["active_particle_contact_count"]
        assert n == ora.meta()["active_particle_contacts"], k   # contacts of the last iteration
        touched = max(touched, n)
    xg, vg, _ = gpu.read_particles()
    xo, vo, _ = ora.read_particles()
    np.testing.assert_allclose(xg[:5], xo[:5], rtol=1e-6, atol=1e-6)       # the proxies: the tool's pose
    np.testing.assert_allclose(xg, xo, rtol=1e-4, atol=1e-5)               # float atomics in the contacts
    assert touched > 0


@pytest.mark.gpu
def test_incremental_update_moves_proxy_points():
    """cn_solver_update_world with the particle attributes uploads new proxy local positions:
    the proxies take them at the next substep's sync, as after a full sync."""
    w, b = proxy_drop(y0=0.5)
    soa = w.soa()
    gpu = Solver(solver_desc(**DESC))
    gpu.sync_world(soa)
    gpu.step(1.0 / 60.0)
    local = np.ctypeslib.as_array(soa.rigid_proxy_local_positions, (soa.particle_count, 4))
    local[:27, :3] *= 1.5
    gpu.update_world(soa, "particle_attributes")
    gpu.step(1.0 / 60.0)
    x = gpu.read_particles()[0]
    p, q = gpu.read_rigid_bodies()[:2]
    want = np.array([qrot(q[b], local[k, :3]) + p[b, :3] for k in range(27)])
    np.testing.assert_allclose(x[:27, :3], want, atol=2e-5)


def crowded_proxies():
    """A 4 x 4 x 4 proxy body (64 proxies of radius 0.02) inside a lattice of small static spheres
    0.025 apart: each proxy is a candidate of ~166 bodies (10,648 pairs), far more than the
    reference's fixed 8 pairs per particle."""
    w = World()
    g = (np.arange(9) - 4.0) * 0.025
    for x in g:
        for y in g:
            for z in g:
                s = w.add_rigid_body("static", position=(float(x), 0.5 + float(y), float(z)))
                w.add_collider(s, "sphere", (0.008,), friction=0.5)
    b = w.add_rigid_body("kinematic", position=(0.0, 0.5, 0.0))
    w.set_rigid_proxy_particles(b, lattice(4, 0.04), 0.02, friction=0.5)
    return w, b


@pytest.mark.parametrize("rate", [0, 8, 192])
def test_particle_rigid_candidate_rate_sizes_the_pair_buffer_in_the_oracle(rate):
    """particle_rigid_pairs_per_particle: 0 and 8 are the reference's max(particles x 8, 64) pairs
    (an overflow here), 192 holds every candidate."""
    w, _ = crowded_proxies()
    soa = w.soa()
    ora = cn_oracle.Oracle(solver_desc(**DESC, particle_rigid_pairs_per_particle=rate), soa)
    ora.step(1.0 / 60.0)
    m = ora.meta()
    cap = max(64 * (rate or 8), 64)
    assert m["required_rigid_pairs"] > 8 * 64, m
    assert m["rigid_pairs"] == min(m["required_rigid_pairs"], cap), m
    ora.close()


@pytest.mark.gpu
def test_particle_rigid_candidate_rate_matches_the_oracle_and_clears_the_overflow():
    w, _ = crowded_proxies()
    for rate, status in ((0, "CAPACITY"), (192, "OK")):
        desc = solver_desc(**DESC, particle_rigid_pairs_per_particle=rate)
        gpu, ora = pair(w, desc)
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
        m, om = gpu.validate_gpu_meta(), ora.meta()
        assert m["status"] == status, m
        assert m["required_particle_rigid_candidate_count"] == om["required_rigid_pairs"]
        assert m["required_proxy_rigid_contact_count"] == om["required_proxy_contacts"]
        xg, xo = gpu.read_particles()[0], ora.read_particles()[0]
        assert np.abs(xg - xo).max() < 1e-5
        gpu.close()
        ora.close()


@pytest.mark.gpu
def test_particle_rigid_candidate_rate_is_bounded():
    s = Solver(solver_desc(**DESC, particle_rigid_pairs_per_particle=1000))
    w, _ = proxy_drop()
    with pytest.raises(CNError):
        s.sync_world(w.soa())
    s.close()
