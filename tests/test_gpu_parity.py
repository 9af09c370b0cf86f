"""Parity of the sm_100a substep (through the C ABI) with the CPU oracle on the same seeded scenes.

Bars (from the build's contract):
  * cell keys, sort permutations, cell-range tables and fluid neighbour lists: bit-exact;
  * positions and velocities after one step: within 1e-5 relative (RTOL below);
  * volume / density / energy drift after 100 steps: within 1e-3 of the oracle.
Paths that use only + - * / sqrt in the reference's order are expected to be bit-exact as well
(both sides are built without fused multiply-add); paths through acos/atan2/sin/cos and float
atomics are held to the tolerance.
"""
import numpy as np
import pytest

from cn_physics import Solver, World, scenes, solver_desc
import cn_oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-5
ATOL_X = 1e-6   # m, for coordinates near zero
ATOL_V = 1e-5   # m/s


def pair(world, desc, debug=0):
    soa = world.soa()
    gpu = Solver(desc)
    if debug:
        gpu.set_debug(keep_fluid_delta=bool(debug & 1), post_update_neighbors=bool(debug & 2),
                      force_broadphase=bool(debug & 4))
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    return gpu, ora


def close(a, b, atol, rtol=RTOL, what=""):
    np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, err_msg=what)


def assert_state(gpu, ora, what, atol_x=ATOL_X, atol_v=ATOL_V, rtol=RTOL):
    xg, vg, pg = gpu.read_particles()
    xo, vo, po = ora.read_particles()
    assert np.isfinite(xg).all() and np.isfinite(vg).all(), what
    close(xg, xo, atol_x, rtol, what + " positions")
    close(vg, vo, atol_v, rtol, what + " velocities")
    close(pg, po, atol_x, rtol, what + " previous positions")
    return xg, xo


def small_fluid(n=(16, 12, 16), **kw):
    return scenes.dam_break(nx=n[0], ny=n[1], nz=n[2], box=(1.6, 1.2, 2.4), **kw)


def test_fluid_broadphase_and_neighbours_bit_exact():
    w, desc, dt = small_fluid()
    gpu, ora = pair(w, desc, debug=1 | 2 | 4)
    gpu.step(dt)
    ora.step(dt)
    for name in ("cell_entries", "sorted_keys", "cell_ranges", "fluid_neighbor_counts"):
        g, o = gpu.debug_read(name), ora.debug_read(name)
        assert g.shape == o.shape and np.array_equal(g, o), name
    counts = gpu.debug_read("fluid_neighbor_counts").view(np.uint32)
    gl = gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    ol = ora.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    for p in range(len(counts)):
        assert np.array_equal(gl[p, :counts[p]], ol[p, :counts[p]]), p
    assert counts.mean() > 8
    assert_state(gpu, ora, "dam break 1 step")
    assert gpu.validate_gpu_meta()["status"] == "OK"


def test_fluid_first_iteration_lists_and_constraints():
    w, desc, dt = small_fluid((12, 12, 12))
    desc.fluid_iterations = 1
    gpu, ora = pair(w, desc, debug=1)
    ora.set_post_update_neighbors(False)  # compare the lists built inside the iteration
    gpu.step(dt)
    ora.step(dt)
    counts = gpu.debug_read("fluid_neighbor_counts").view(np.uint32)
    assert np.array_equal(counts, ora.debug_read("fluid_neighbor_counts").view(np.uint32))
    gl = gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    ol = ora.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128)
    for p in range(len(counts)):
        assert np.array_equal(gl[p, :counts[p]], ol[p, :counts[p]]), p
    gc = gpu.debug_read("fluid_constraints").view(np.float32).reshape(-1, 4)
    oc = ora.debug_read("fluid_constraints").view(np.float32).reshape(-1, 4)
    close(gc, oc, 1e-9, what="density constraints")
    gd = gpu.debug_read("fluid_delta").view(np.float32).reshape(-1, 4)
    od = ora.debug_read("fluid_delta").view(np.float32).reshape(-1, 4)
    close(gd, od, 1e-9, what="fluid deltas")
    assert_state(gpu, ora, "fluid, 1 iteration")


def test_fluid_several_steps():
    w, desc, dt = small_fluid((14, 10, 14))
    gpu, ora = pair(w, desc)
    for k in range(5):
        gpu.step(dt)
        ora.step(dt)
    assert_state(gpu, ora, "fluid 5 steps", atol_x=1e-5, atol_v=1e-4, rtol=1e-4)


def test_xpbd_cube_one_step_full_size():
    w, desc, dt = scenes.xpbd_cube()
    assert w.counts()["tets"] == 16875
    gpu, ora = pair(w, desc)
    gpu.step(dt)
    ora.step(dt)
    assert_state(gpu, ora, "16^3 XPBD cube, 1 step")


def test_xpbd_falling_cube_with_ground_contacts():
    w, desc, dt = scenes.xpbd_cube(n=6, spacing=0.1, pin_bottom=False, lift=0.05)
    desc.substeps = 4
    gpu, ora = pair(w, desc)
    for k in range(20):
        gpu.step(dt)
        ora.step(dt)
    xg, xo = assert_state(gpu, ora, "falling cube", atol_x=1e-5, atol_v=1e-4, rtol=1e-4)
    assert xg[:, 1].min() > 0.0 and xg[:, 1].min() < 0.06   # resting on the ground
    rc = gpu.debug_read("rigid_contacts")
    assert rc.size > 0 and rc.size == ora.debug_read("rigid_contacts").size


def test_keys_with_force_broadphase_bit_exact_on_soft_body():
    w, desc, dt = scenes.xpbd_cube(n=8, spacing=0.1)
    gpu, ora = pair(w, desc, debug=4)
    gpu.step(dt)
    ora.step(dt)
    for name in ("cell_entries", "sorted_keys", "cell_ranges"):
        assert np.array_equal(gpu.debug_read(name), ora.debug_read(name)), name


def cloth_strand_world():
    w = World()
    w.add_cloth_grid((10, 10), (0.5, 0.5), position=(0.0, 0.3, 0.0), radius=0.01, structural_compliance=1e-6,
                     bend_compliance=1e-3, static_particles=[0, 9], friction=0.2)
    pts = [(-0.2 + 0.04 * k, 0.5, 0.1) for k in range(11)]
    w.add_strand(pts, radius=0.01, stretch_shear_compliance=1e-6, bend_compliance=1e-4, twist_compliance=1e-4,
                 distance_compliance=1e-6, static_particles=[0])
    scenes.ground(w)
    w.soa()
    return w


def test_cloth_and_strands():
    w = cloth_strand_world()
    desc = solver_desc(substeps=4, default_iterations=10, enable_blocking_readback=0)
    gpu, ora = pair(w, desc)
    for k in range(5):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    assert_state(gpu, ora, "cloth + strands", atol_x=1e-5, atol_v=1e-4, rtol=1e-4)
    close(gpu.read_strand_orientations(), ora.read_strand_orientations(), 1e-5, 1e-4, "strand frames")


def test_mixed_scene_with_tool_and_cross_contacts():
    w, desc, dt, tool = scenes.mixed_surgical(tissue=(6, 4, 6), cloth=(8, 8), strands=(3, 9), fluid=(6, 6, 6))
    desc.substeps = 2
    desc.default_iterations = 8
    gpu, ora = pair(w, desc)
    for k in range(4):
        p = scenes.tool_path(dt * (k + 1))
        gpu.set_kinematic_target(tool, p)
        ora.set_kinematic_target(tool, p)
        gpu.step(dt)
        ora.step(dt)
    # float atomics in the explicit contact solve make the summation order differ
    assert_state(gpu, ora, "mixed scene", atol_x=1e-5, atol_v=1e-4, rtol=1e-4)
    meta = gpu.validate_gpu_meta()
    assert meta["status"] == "OK", meta


def tet_volume(x, tets):
    p0, p1, p2, p3 = (x[tets[:, k], :3].astype(np.float64) for k in range(4))
    return np.abs(np.einsum("ij,ij->i", np.cross(p1 - p0, p2 - p0), p3 - p0)).sum() / 6.0


def test_xpbd_cube_volume_and_energy_drift_100_steps():
    w, desc, dt = scenes.xpbd_cube()
    tets = w.array("tets")[:, :4].astype(np.int64)
    gpu, ora = pair(w, desc)
    for k in range(100):
        gpu.step(dt)
        ora.step(dt)
    xg, vg, _ = gpu.read_particles()
    xo, vo, _ = ora.read_particles()
    vol_g, vol_o = tet_volume(xg, tets), tet_volume(xo, tets)
    assert abs(vol_g - vol_o) <= 1e-3 * vol_o
    ke_g = 0.5 * (vg[:, :3].astype(np.float64) ** 2).sum()
    ke_o = 0.5 * (vo[:, :3].astype(np.float64) ** 2).sum()
    pe_g, pe_o = 9.81 * xg[:, 1].astype(np.float64).sum(), 9.81 * xo[:, 1].astype(np.float64).sum()
    assert abs((ke_g + pe_g) - (ke_o + pe_o)) <= 1e-3 * abs(ke_o + pe_o)


def test_dam_break_density_drift_20_steps():
    w, desc, dt = small_fluid((16, 16, 16))
    gpu, ora = pair(w, desc, debug=1)
    for k in range(20):
        gpu.step(dt)
        ora.step(dt)
    cg = gpu.debug_read("fluid_constraints").view(np.float32).reshape(-1, 4)[:, 3].astype(np.float64)
    co = ora.debug_read("fluid_constraints").view(np.float32).reshape(-1, 4)[:, 3].astype(np.float64)
    assert abs(cg.mean() - co.mean()) <= 1e-3 * max(abs(co.mean()), 1e-12) + 1e-12


def fluid_with_distant_tissue():
    """Fluid block plus a pinned soft body out of its reach: particle-particle contacts are on (the
    contacts may move fluid x, so the superset lists are validated by each particle's move since
    their build) but none forms, so the run is free of float atomics."""
    w, desc, dt = small_fluid((12, 10, 12))
    pinned = [x * 3 * 4 + z for x in range(4) for z in range(4)]
    w.add_soft_body_grid((0.3, 0.2, 0.3), 0.1, position=(5.0, 0.2, 5.0), radius=0.03, edge_compliance=1e-5,
                         volume_compliance=1e-6, static_particles=pinned)
    return w, desc, dt


def test_superset_lists_with_contacts_equal_the_cell_walk():
    w, desc, dt = fluid_with_distant_tissue()
    desc.fluid_iterations = 4
    soa = w.soa()
    runs = []
    for walk in (False, True):
        gpu = Solver(desc)
        gpu.set_debug(keep_fluid_delta=True, walk_cells=walk)
        gpu.sync_world(soa)
        gpu.set_timing(True)
        for _ in range(3):
            gpu.step(dt)
        runs.append((gpu.debug_read("fluid_neighbor_counts").view(np.uint32).copy(),
                     gpu.debug_read("fluid_neighbors").view(np.uint32).reshape(-1, 128).copy(),
                     gpu.read_particles(), set(gpu.kernel_times())))
    (c0, l0, s0, k0), (c1, l1, s1, k1) = runs
    assert "fluid_neighbors_superset" in k0 and "fluid_neighbors_superset" not in k1
    assert np.array_equal(c0, c1)
    for p in range(len(c0)):
        assert np.array_equal(l0[p, :c0[p]], l1[p, :c0[p]]), p
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)
    ora = cn_oracle.Oracle(desc, soa)
    ora.set_post_update_neighbors(False)
    for _ in range(3):
        ora.step(dt)
    assert np.array_equal(c0, ora.debug_read("fluid_neighbor_counts").view(np.uint32))
    for a, b in zip(s0, ora.read_particles()):
        np.testing.assert_allclose(a, b, rtol=RTOL, atol=ATOL_V)
