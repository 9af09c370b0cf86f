"""Edge cases of the substep against the oracle: an empty world, a lone particle, cells whose
32-bit hash keys collide, neighbour lists cut at max_fluid_neighborhood, and a full
particle-rigid candidate buffer (the capacities and their overflow reporting of
physics_solver.cpp:458-459 and validateGpuMetaBlocking, :1403-1491)."""
import numpy as np
import pytest

from cn_physics import Solver, World, scenes, solver_desc
import cn_oracle

pytestmark = pytest.mark.gpu

CELL = 0.1  # h = max((2 / 0.6) r, 2 r) for r = 0.03


def pair(world, desc):
    soa = world.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    return gpu, cn_oracle.Oracle(desc, soa), soa


def step_both(gpu, ora, dt, frames):
    for _ in range(frames):
        gpu.step(dt)
        ora.step(dt)


def same_state(gpu, ora):
    for a, b in zip(gpu.read_particles(), ora.read_particles()):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)


def same_lists(gpu, ora, max_neighbours=128):
    """Counts and the valid entries of every list (entries past a count are not part of it)."""
    counts = gpu.debug_read("fluid_neighbor_counts").view(np.uint32)
    assert np.array_equal(counts, ora.debug_read("fluid_neighbor_counts").view(np.uint32))
    gl = gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, max_neighbours)
    ol = ora.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, max_neighbours)
    for p in range(len(counts)):
        assert np.array_equal(gl[p, :counts[p]], ol[p, :counts[p]]), p
    return counts


def test_empty_world_and_bodies_only():
    gpu = Solver(solver_desc())
    w = World()
    gpu.sync_world(w.soa())
    gpu.step(1.0 / 60.0)
    x, v, p = gpu.read_particles()
    assert x.shape == (0, 4) and v.shape == (0, 4)
    assert gpu.validate_gpu_meta()["status"] == "OK"
    # a world of bodies alone steps the rigid passes with no particle work
    w = World()
    scenes.ground(w)
    tool = w.add_rigid_body("kinematic", position=(0.0, 1.0, 0.0))
    w.add_collider(tool, "sphere", (0.1,))
    gpu = Solver(solver_desc(substeps=2))
    gpu.sync_world(w.soa())
    gpu.set_kinematic_target(tool, (0.0, 0.9, 0.0))
    gpu.step(1.0 / 60.0)
    assert gpu.validate_gpu_meta()["status"] == "OK"


def test_lone_fluid_particle():
    w = World()
    w.add_fluid_grid((0.05, 0.05, 0.05), 0.05, position=(0.0, 0.5, 0.0), radius=0.03)
    assert w.counts()["particles"] == 1
    gpu, ora, _ = pair(w, solver_desc(substeps=2, fluid_iterations=4))
    step_both(gpu, ora, 1.0 / 120.0, 3)
    same_state(gpu, ora)
    assert gpu.debug_read("fluid_neighbor_counts").view(np.uint32).tolist() == [0]


def colliding_cells():
    """Two far-apart cells with equal cell keys (the reference's 32-bit XOR hash)."""
    r = np.arange(-60, 61, dtype=np.int64)
    gx, gy, gz = (a.ravel() for a in np.meshgrid(r, np.arange(0, 12), r, indexing="ij"))
    u = np.uint32
    k = (gx.astype(u) * u(73856093)) ^ (gy.astype(u) * u(19349663)) ^ (gz.astype(u) * u(83492791))
    order = np.argsort(k, kind="stable")
    ks = k[order]
    for i in np.nonzero(ks[1:] == ks[:-1])[0]:
        a, b = order[i], order[i + 1]
        ca, cb = np.array([gx[a], gy[a], gz[a]]), np.array([gx[b], gy[b], gz[b]])
        if np.abs(ca - cb).max() > 8 and ca[1] >= 1:
            return ca, cb
    raise AssertionError("no colliding cells found")


def test_hash_colliding_cells_keep_separate_neighbourhoods():
    ca, cb = colliding_cells()
    w = World()
    for c in (ca, cb):  # a 4^3 block spanning the colliding cell and its neighbours
        w.add_fluid_grid((0.2, 0.2, 0.2), 0.05, position=tuple((c + 0.5) * CELL), radius=0.03)
    soa = w.soa()
    x = w.positions()[:, :3]
    cells = np.floor(x / np.float32(CELL)).astype(np.int64)
    assert (cells == ca).all(1).any() and (cells == cb).all(1).any()
    gpu, ora, _ = pair(w, solver_desc(substeps=1, fluid_iterations=2))
    gpu.set_debug(keep_fluid_delta=True, post_update_neighbors=True)  # the oracle rebuilds them too
    step_both(gpu, ora, 1.0 / 120.0, 1)
    for name in ("cell_entries", "sorted_keys", "cell_ranges"):
        assert np.array_equal(gpu.debug_read(name), ora.debug_read(name)), name
    counts = same_lists(gpu, ora)
    same_state(gpu, ora)
    # no particle lists a neighbour from the other block
    nb = gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    for p in range(len(counts)):
        assert ((nb[p, :counts[p]] < 64) == (p < 64)).all(), p
    step_both(gpu, ora, 1.0 / 120.0, 2)
    same_state(gpu, ora)


def test_neighbour_lists_cut_at_the_maximum():
    w, desc, dt = scenes.dam_break(nx=8, ny=8, nz=8, box=(0.6, 0.6, 0.6))
    desc.max_fluid_neighborhood = 12
    gpu, ora, _ = pair(w, desc)
    ora.set_post_update_neighbors(False)  # compare the lists built inside the last iteration
    step_both(gpu, ora, dt, 2)
    counts = same_lists(gpu, ora, 12)
    assert counts.max() == 12
    same_state(gpu, ora)
    # both count cut lists (per list build; the oracle also rebuilds after the velocity update)
    assert gpu.validate_gpu_meta()["fluid_neighbor_truncations"] > 0 and ora.meta()["neighbor_truncations"] > 0


def test_full_rigid_candidate_buffer_is_reported_and_matches():
    # 8 particles inside 70 static spheres: 560 candidate pairs against a capacity of 64
    w = World()
    w.add_soft_body_grid((0.02, 0.02, 0.02), 0.02, position=(0.0, 0.5, 0.0), radius=0.01,
                         edge_compliance=1e-5, volume_compliance=1e-6)
    for k in range(70):
        b = w.add_rigid_body("static", position=(0.0005 * k, 0.5, 0.0))
        w.add_collider(b, "sphere", (0.2,))
    gpu, ora, _ = pair(w, solver_desc(substeps=1, default_iterations=2))
    step_both(gpu, ora, 1.0 / 60.0, 1)
    m = gpu.validate_gpu_meta()
    om = ora.meta()
    assert m["status"] == "CAPACITY" and m["particle_rigid_candidate_overflow"] == 1
    assert m["required_particle_rigid_candidate_count"] == om["required_rigid_pairs"] == 8 * 70
    assert m["particle_rigid_candidate_count"] == om["rigid_pairs"] == 64
    x_g, _, _ = gpu.read_particles()
    x_o, _, _ = ora.read_particles()
    np.testing.assert_allclose(x_g, x_o, rtol=1e-5, atol=1e-6)


def test_rigid_candidates_from_the_lbvh_keep_the_scan_order():
    """With more than 32 colliders and a dynamic body (so the substep builds the LBVH) the
    particle-rigid candidates come from the tree, sorted back into query order: the candidate
    counts and the contact records (candidate order) equal the oracle's linear scan."""
    w = World()
    w.add_soft_body_grid((0.4, 0.2, 0.4), 0.05, position=(0.0, 0.3, 0.0), radius=0.03,
                         edge_compliance=1e-5, volume_compliance=1e-6, friction=0.3)
    rng = np.random.default_rng(3)
    for k in range(48):   # static spheres around and inside the block
        b = w.add_rigid_body("static", position=tuple(rng.uniform((-0.3, 0.1, -0.3), (0.3, 0.5, 0.3))))
        w.add_collider(b, "sphere", (float(rng.uniform(0.02, 0.06)),))
    far = w.add_rigid_body("dynamic", position=(5.0, 1.0, 5.0), mass=1.0, inverse_inertia=(10.0,) * 3)
    w.add_collider(far, "box", (0.1, 0.1, 0.1))
    w.add_collider(far, "sphere", (0.05,), local_position=(0.0, 0.2, 0.0))
    gpu, ora, _ = pair(w, solver_desc(substeps=1, default_iterations=4))
    step_both(gpu, ora, 1.0 / 60.0, 1)
    m, om = gpu.validate_gpu_meta(), ora.meta()
    assert m["required_particle_rigid_candidate_count"] == om["required_rigid_pairs"] > 0
    g, o = gpu.debug_read("rigid_contacts"), ora.debug_read("rigid_contacts")
    assert g.size == o.size > 0 and np.array_equal(g.view(np.uint8), o.view(np.uint8))
    same_state(gpu, ora)


def multi_environment_fluid(envs=14, n=(6, 5, 6), seed=0):
    """`envs` fluid blocks, each in its own environment with its own five static walls (5 x envs
    colliders: past the 64 bits of the boundary mask, so the per-particle candidate lists over the
    collider LBVH carry the boundary), side by side along x."""
    w = World()
    sp = 0.05
    body = w.add_rigid_body("static")
    size = (n[0] * sp, n[1] * sp, n[2] * sp)
    box = (0.6, 0.5, 0.6)
    t = 0.1
    for e in range(envs):
        ox = e * 1.0
        w.add_fluid_grid(size, sp, position=(ox + 0.3, size[1] * 0.5 + 0.03, 0.3), radius=0.6 * sp,
                         environment=e)
        bx, by, bz = box
        for half, local in (((bx * 0.5 + 2 * t, t, bz * 0.5 + 2 * t), (ox + bx * 0.5, -t, bz * 0.5)),
                            ((t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (ox - t, by * 0.5, bz * 0.5)),
                            ((t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (ox + bx + t, by * 0.5, bz * 0.5)),
                            ((bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (ox + bx * 0.5, by * 0.5, -t)),
                            ((bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (ox + bx * 0.5, by * 0.5, bz + t))):
            w.add_collider(body, "box", half, local, environment=e)
    w.soa()
    x = w.positions()
    rng = np.random.default_rng(seed)
    x[:, :3] += rng.uniform(-1e-4, 1e-4, size=(x.shape[0], 3)).astype(np.float32)
    return w, solver_desc(substeps=2, fluid_iterations=4, enable_blocking_readback=0), 1.0 / 120.0


def test_fluid_against_more_than_64_colliders():
    w, desc, dt = multi_environment_fluid()
    assert w.counts()["colliders"] == 70
    gpu, ora, _ = pair(w, desc)
    step_both(gpu, ora, dt, 6)
    for a, b in zip(gpu.read_particles(), ora.read_particles()):
        assert np.array_equal(a, b)
    same_lists(gpu, ora)
    meta = gpu.validate_gpu_meta()
    assert meta["status"] == "OK" and meta["fluid_boundary_candidate_overflow"] == 0, meta
