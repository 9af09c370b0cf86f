"""Full-size parity of the shipped schedule (no debug flags) with the oracle.

* The PBF dam break at its benchmark size (128 x 64 x 128 = 1,048,576 particles) for one frame:
  the sorted (cellKey, index) pairs, the cell-range table, the neighbour counts and lists of the
  last fluid iteration and the particle state are compared with the oracle bit for bit (the
  parity bars are bit-exact keys / permutations / lists and 1e-5 on the state; both sides
  evaluate the same float32 expressions without contraction, so the state is bit-identical too).
* The superset-filter schedule (the default from the second fluid iteration on) against the
  27-cell walk in every iteration, bit for bit, at full size for two frames.
* A 64 x 32 x 64 dam break for 100 frames: positions bit-identical to the oracle, and the SPH
  density of the final state within 1e-3 of the oracle's.
* The mixed surgical scene at its benchmark size (tissue 60 x 30 x 60, cloth 256 x 256, 64
  strands of 129 points, 262,144 fluid particles, the kinematic tool) for one frame, within the
  tolerance: its particle-particle contacts sum with float atomics, in an order the reference
  does not fix either.
"""
import numpy as np
import pytest

import cn_oracle
from cn_physics import Solver, scenes

pytestmark = pytest.mark.gpu


def _bit_equal(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    if not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
        bad = int((a != b).reshape(len(a), -1).any(axis=1).sum()) if a.ndim else 1
        raise AssertionError(f"{what}: {bad} rows differ")


def _lists(sim, n):
    counts = sim.debug_read("fluid_neighbor_counts").view(np.uint32)[:n].copy()
    lists = sim.debug_read("fluid_neighbors").view(np.uint32).reshape(n, -1).copy()
    lists[np.arange(lists.shape[1])[None, :] >= counts[:, None]] = 0
    return counts, lists


def test_dam_break_full_size_one_frame_bit_exact_against_oracle():
    w, desc, dt = scenes.dam_break()
    soa = w.soa()
    n = soa.particle_count
    assert n == 1048576
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    ora.set_post_update_neighbors(False)   # the shipped schedule keeps the last iteration's lists
    gpu.step(dt)
    ora.step(dt)
    for name in ("sorted_keys", "cell_ranges"):
        _bit_equal(gpu.debug_read(name), ora.debug_read(name), name)
    cg, lg = _lists(gpu, n)
    co, lo = _lists(ora, n)
    _bit_equal(cg, co, "neighbour counts")
    _bit_equal(lg, lo, "neighbour lists")
    assert cg.mean() > 20
    for a, b, what in zip(gpu.read_particles(), ora.read_particles(), ("x", "v", "x_prev")):
        _bit_equal(a, b, what)
    meta = gpu.validate_gpu_meta()
    assert meta["status"] == "OK" and meta["device_wait_timeouts"] == 0


def test_dam_break_full_size_superset_filter_equals_cell_walk_two_frames():
    w, desc, dt = scenes.dam_break()
    soa = w.soa()
    n = soa.particle_count
    out = []
    for walk in (False, True):
        gpu = Solver(desc)
        if walk:
            gpu.set_debug(walk_cells=True)
        gpu.sync_world(soa)
        gpu.set_timing(True)
        for _ in range(2):
            gpu.step(dt)
        out.append((_lists(gpu, n), gpu.read_particles(), set(gpu.kernel_times())))
        gpu.close()
    ((c0, l0), s0, k0), ((c1, l1), s1, k1) = out
    assert "fluid_neighbors_superset" in k0 and "fluid_neighbors_superset" not in k1
    _bit_equal(c0, c1, "counts")
    _bit_equal(l0, l1, "lists")
    for a, b, what in zip(s0, s1, ("x", "v", "x_prev")):
        _bit_equal(a, b, what)


def _sph_density(x, h):
    """Sum of the spiky kernel 15 / (pi h^3) (1 - r / h)^2 over neighbours within h (self included)."""
    from scipy.spatial import cKDTree
    p = x[:, :3].astype(np.float64)
    tree = cKDTree(p)
    pairs = tree.query_pairs(h, output_type="ndarray")
    r = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1)
    w = 15.0 / (np.pi * h ** 3) * (1.0 - r / h) ** 2
    rho = np.full(len(p), 15.0 / (np.pi * h ** 3))
    np.add.at(rho, pairs[:, 0], w)
    np.add.at(rho, pairs[:, 1], w)
    return rho


def test_dam_break_64x32x64_100_frames_density_drift():
    w, desc, dt = scenes.dam_break(nx=64, ny=32, nz=64, box=(6.4, 3.2, 12.8))
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    gpu.step_many(dt, 100)
    for _ in range(100):
        ora.step(dt)
    xg, vg, _ = gpu.read_particles()
    xo, vo, _ = ora.read_particles()
    _bit_equal(xg, xo, "positions after 100 frames")
    rg, ro = _sph_density(xg, 0.1), _sph_density(xo, 0.1)
    assert abs(rg.mean() - ro.mean()) <= 1e-3 * ro.mean()
    ke_g = 0.5 * (vg[:, :3].astype(np.float64) ** 2).sum()
    ke_o = 0.5 * (vo[:, :3].astype(np.float64) ** 2).sum()
    pe_g, pe_o = 9.81 * xg[:, 1].astype(np.float64).sum(), 9.81 * xo[:, 1].astype(np.float64).sum()
    assert abs((ke_g + pe_g) - (ke_o + pe_o)) <= 1e-3 * abs(ke_o + pe_o)


def test_mixed_surgical_full_size_one_frame():
    w, desc, dt, tool = scenes.mixed_surgical()
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    p = scenes.tool_path(dt)
    gpu.set_kinematic_target(tool, p)
    ora.set_kinematic_target(tool, p)
    gpu.step(dt)
    ora.step(dt)
    xg, vg, pg = gpu.read_particles()
    xo, vo, po = ora.read_particles()
    assert np.isfinite(xg).all() and np.isfinite(vg).all()
    for a, b, what in ((xg, xo, "x"), (vg, vo, "v"), (pg, po, "x_prev")):
        a3, b3 = a[:, :3].astype(np.float64), b[:, :3].astype(np.float64)
        rel = np.linalg.norm(a3 - b3) / np.linalg.norm(b3)
        assert rel <= 1e-5, (what, rel)
    np.testing.assert_allclose(xg, xo, rtol=1e-5, atol=1e-6)
    meta = gpu.validate_gpu_meta()
    assert meta["status"] == "OK", meta
