"""Full-size (1,048,576-particle dam break, 16^3 XPBD cube) checks through size-independent
properties: the broadphase keys and permutation are recomputed independently in numpy (IEEE
float32, no fused multiply-add) and compared bit-for-bit; neighbour lists are checked for range,
distance and symmetry."""
import numpy as np
import pytest

from cn_physics import Solver, scenes

pytestmark = pytest.mark.gpu


def numpy_keys(x, v, dt, g, cell):
    """physics_soft_predict.cs.hlsl + physics_particle_build_broad_phase_entries.cs.hlsl in numpy."""
    x = x.copy()
    mov = x[:, 3] > np.float32(1e-6)
    vel = v[:, :3] + (g * np.float32(dt * 1.0))  # gravityScale 1
    x[mov, :3] = x[mov, :3] + vel[mov] * np.float32(dt)
    inv = np.float32(1.0) / np.float32(max(cell, 1e-4))
    c = np.floor(x[:, :3] * inv).astype(np.int32)
    u = c.view(np.uint32).astype(np.uint64)
    key = ((u[:, 0] * 73856093) & 0xFFFFFFFF) ^ ((u[:, 1] * 19349663) & 0xFFFFFFFF) ^ ((u[:, 2] * 83492791) & 0xFFFFFFFF)
    return c, key.astype(np.uint32)


def test_dam_break_full_size_broadphase_bit_exact():
    w, desc, dt = scenes.dam_break()
    soa = w.soa()
    assert soa.particle_count == 1048576
    gpu = Solver(desc)
    gpu.set_debug(keep_fluid_delta=True)
    gpu.sync_world(soa)
    gpu.step(dt)
    # the debug buffers hold the last substep: its entries must hash their own coordinates and
    # the permutation must be numpy's stable argsort of those keys
    ent = gpu.debug_read("cell_entries").view(np.int32).reshape(-1, 4)
    u = ent[:, :3].view(np.uint32).astype(np.uint64)
    key = (((u[:, 0] * 73856093) & 0xFFFFFFFF) ^ ((u[:, 1] * 19349663) & 0xFFFFFFFF) ^
           ((u[:, 2] * 83492791) & 0xFFFFFFFF)).astype(np.uint32)
    assert np.array_equal(key, ent[:, 3].view(np.uint32))
    sk = gpu.debug_read("sorted_keys").view(np.uint32).reshape(-1, 2)
    order = np.argsort(ent[:, 3].view(np.uint32), kind="stable")
    assert np.array_equal(sk[:, 1], order)
    assert np.array_equal(sk[:, 0], ent[order, 3].view(np.uint32))
    # cell-range table: compacted runs of the sorted keys
    cr = gpu.debug_read("cell_ranges").view(np.uint32).reshape(-1, 4)
    starts = np.flatnonzero(np.r_[True, sk[1:, 0] != sk[:-1, 0]])
    ends = np.r_[starts[1:], len(sk)]
    m = len(starts)
    assert cr.shape[0] == 1 << int(np.ceil(np.log2(2 * len(sk))))
    assert np.array_equal(cr[:m, 0], sk[starts, 0]) and np.array_equal(cr[:m, 1], starts)
    assert np.array_equal(cr[:m, 2], ends) and (cr[m:, 0] == 0xFFFFFFFF).all()
    meta = gpu.validate_gpu_meta()
    assert meta["status"] == "OK" and meta["device_wait_timeouts"] == 0


def test_dam_break_full_size_first_substep_keys_match_numpy():
    w, desc, dt = scenes.dam_break()
    desc.substeps = 1
    desc.fluid_iterations = 1
    soa = w.soa()
    x0 = w.positions().copy()
    v0 = w.velocities().copy()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    gpu.step(dt)
    c, key = numpy_keys(x0, v0, dt, np.array([0.0, -9.81, 0.0], np.float32), soa.particle_grid_cell_size)
    ent = gpu.debug_read("cell_entries").view(np.int32).reshape(-1, 4)
    assert np.array_equal(ent[:, :3], c)
    assert np.array_equal(ent[:, 3].view(np.uint32), key)
    sk = gpu.debug_read("sorted_keys").view(np.uint32).reshape(-1, 2)
    assert np.array_equal(sk[:, 1], np.argsort(key, kind="stable"))
    counts = gpu.debug_read("fluid_neighbor_counts").view(np.uint32)
    lists = gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    x1 = x0.copy()
    vel = v0[:, :3] + np.array([0.0, -9.81, 0.0], np.float32) * np.float32(dt)
    x1[:, :3] = x0[:, :3] + vel * np.float32(dt)
    rng = np.random.default_rng(0)
    sample = rng.choice(len(counts), 2000, replace=False)
    h = 0.1
    for p in sample:
        nb = lists[p, :counts[p]]
        assert len(set(nb.tolist())) == len(nb) and p not in nb
        d = np.linalg.norm(x1[nb, :3] - x1[p, :3], axis=1)
        assert (d < h).all()
        for q in nb[:8]:
            if counts[q] < 128:
                assert p in lists[q, :counts[q]]
    assert counts.mean() > 20


def test_xpbd_cube_100_steps_stays_finite_and_pinned():
    w, desc, dt = scenes.xpbd_cube()
    soa = w.soa()
    x0 = w.positions().copy()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    gpu.step_many(dt, 100)
    x, v, _ = gpu.read_particles()
    assert np.isfinite(x).all() and np.isfinite(v).all()
    pinned = x0[:, 3] == 0.0
    assert np.array_equal(x[pinned], x0[pinned])
    assert x[:, 1].min() > -0.01
