"""Rigid-rigid contacts of dynamic bodies: the rigid broadphase (an LBVH on the GPU, every pair
tested on the CPU: the same pair set), the narrow phase of physics_rigid_contact_primitives.hlsli
with the box-box manifold of physics_rigid_box_box_manifold.hlsli, depenetration and the
body-pair velocity solve.  Bodies' corrections are summed with float atomics on the GPU (as in
the reference) and in pair order by the oracle, so they agree within tolerance."""
import numpy as np
import pytest

from cn_physics import Solver, World, scenes, solver_desc
import cn_oracle

Q_TILT_Z30 = (0.0, 0.0, 0.2588190, 0.9659258)
Q_Z90 = (0.0, 0.0, 0.7071068, 0.7071068)


def drop(shape, params, y0=0.5, tilt=(0, 0, 0, 1)):
    w = World()
    scenes.ground(w)
    b = w.add_rigid_body("dynamic", position=(0.0, y0, 0.0), orientation=tilt, mass=1.0, inverse_inertia=(20.0,) * 3)
    w.add_collider(b, shape, params, friction=0.5)
    return w, b


def stack():
    w = World()
    scenes.ground(w)
    lower = w.add_rigid_body("dynamic", position=(0.0, 0.06, 0.0), mass=1.0, inverse_inertia=(30.0,) * 3)
    w.add_collider(lower, "box", (0.15, 0.05, 0.15), friction=0.6)
    upper = w.add_rigid_body("dynamic", position=(0.02, 0.2, 0.0), mass=0.5, inverse_inertia=(60.0,) * 3)
    w.add_collider(upper, "box", (0.08, 0.04, 0.08), friction=0.6)
    ball = w.add_rigid_body("dynamic", position=(0.3, 0.3, 0.0), mass=0.3, inverse_inertia=(150.0,) * 3)
    w.add_collider(ball, "sphere", (0.05,), friction=0.4)
    return w, (lower, upper, ball)


def pile(n=24, seed=0):
    rng = np.random.default_rng(seed)
    w = World()
    scenes.ground(w)
    bodies = []
    for k in range(n):
        p = (float(rng.uniform(-0.2, 0.2)), 0.05 + 0.09 * k, float(rng.uniform(-0.2, 0.2)))
        b = w.add_rigid_body("dynamic", position=p, mass=0.2, inverse_inertia=(200.0,) * 3)
        shape = ("sphere", (0.05,)) if k % 3 == 0 else (("capsule", (0.03, 0.05)) if k % 3 == 1 else ("box", (0.04, 0.04, 0.04)))
        w.add_collider(b, *shape, friction=0.5)
        bodies.append(b)
    return w, bodies


DESC = dict(substeps=4, default_iterations=10)


@pytest.mark.parametrize("shape,params,rest,tilt", [
    ("sphere", (0.1,), 0.1, (0, 0, 0, 1)),
    ("box", (0.1, 0.05, 0.2), 0.05, (0, 0, 0, 1)),
    ("capsule", (0.05, 0.1), 0.15, (0, 0, 0, 1)),
    ("box", (0.1, 0.1, 0.1), 0.1, Q_TILT_Z30),
    ("capsule", (0.05, 0.1), 0.05, Q_Z90),
])
def test_oracle_bodies_come_to_rest_on_the_ground(shape, params, rest, tilt):
    w, b = drop(shape, params, tilt=tilt)
    o = cn_oracle.Oracle(solver_desc(**DESC), w.soa())
    for _ in range(120):
        o.step(1.0 / 60.0)
    p, q, lin, ang = o.read_rigid_bodies()
    assert abs(p[b, 1] - rest) < 3e-3                   # resting height (within the contact slop)
    assert np.linalg.norm(lin[b, :3]) < 1e-2 and np.linalg.norm(ang[b, :3]) < 5e-2


def test_oracle_stack_settles():
    w, (lower, upper, ball) = stack()
    o = cn_oracle.Oracle(solver_desc(**DESC), w.soa())
    for _ in range(120):
        o.step(1.0 / 60.0)
    p, _, lin, _ = o.read_rigid_bodies()
    assert abs(p[lower, 1] - 0.05) < 3e-3 and abs(p[upper, 1] - 0.14) < 5e-3 and abs(p[ball, 1] - 0.05) < 3e-3
    assert np.abs(lin[:, :3]).max() < 2e-2


@pytest.mark.gpu
@pytest.mark.parametrize("shape,params,tilt", [
    ("sphere", (0.1,), (0, 0, 0, 1)),
    ("box", (0.1, 0.05, 0.2), (0, 0, 0, 1)),
    ("box", (0.1, 0.1, 0.1), Q_TILT_Z30),
    ("capsule", (0.05, 0.1), Q_Z90),
])
def test_drop_matches_the_oracle(shape, params, tilt):
    w, b = drop(shape, params, tilt=tilt)
    desc = solver_desc(**DESC)
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(20):  # free fall and the first contact frames
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    for a, o in zip(gpu.read_rigid_bodies(), ora.read_rigid_bodies()):
        np.testing.assert_allclose(a, o, rtol=1e-4, atol=1e-5)
    for _ in range(100):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    pg, qg, _, _ = gpu.read_rigid_bodies()
    po, qo, _, _ = ora.read_rigid_bodies()
    assert np.abs(pg[b, :3] - po[b, :3]).max() < 1e-3
    assert gpu.validate_gpu_meta()["status"] == "OK"


@pytest.mark.gpu
def test_stack_matches_the_oracle():
    w, bodies = stack()
    desc = solver_desc(**DESC)
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(120):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    pg = gpu.read_rigid_bodies()[0]
    po = ora.read_rigid_bodies()[0]
    assert np.abs(pg[:, :3] - po[:, :3]).max() < 1e-3


@pytest.mark.gpu
def test_bvh_pairs_equal_the_all_pairs_set():
    """The GPU's LBVH traversal finds as many candidate pairs as the oracle's all-pairs test, frame
    after frame while a 24-body pile collapses (same AABBs, same pair rules)."""
    w, bodies = pile()
    desc = solver_desc(**DESC)
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for k in range(6):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
        m = gpu.validate_gpu_meta()
        om = ora.meta()
        assert m["required_rigid_rigid_candidate_count"] == om["required_rigid_rigid_pairs"], k
    assert om["required_rigid_rigid_pairs"] > len(bodies)   # the pile touches
    for _ in range(60):
        gpu.step(1.0 / 60.0)
    p = gpu.read_rigid_bodies()[0][bodies]   # body 0 is the static ground slab
    assert np.isfinite(p).all() and p[:, 1].min() > 0.0 and p[:, 1].max() < 2.5
    assert gpu.validate_gpu_meta()["status"] == "OK"
