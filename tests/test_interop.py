"""Zero-copy DLPack view of the scene buffers and incremental world updates."""
import numpy as np
import pytest

from cn_physics import Solver, scenes

pytestmark = pytest.mark.gpu


def test_dlpack_view_is_the_device_buffer():
    import torch
    w, desc, dt = scenes.xpbd_cube(n=6, spacing=0.1)
    sv = Solver(desc)
    sv.sync_world(w)
    sv.step(dt)
    torch.cuda.synchronize()
    x = sv.export_dlpack("positions_inv_mass")
    assert x.is_cuda and x.shape == (6 ** 3, 4) and x.dtype == torch.float32
    xr, vr, _ = sv.read_particles()
    assert np.array_equal(x.cpu().numpy(), xr)
    gen = sv.gpu_scene_view()["binding_generation"]
    x[:, 1] += 1.0  # writes go straight into the solver's state
    torch.cuda.synchronize()
    assert np.array_equal(sv.read_particles()[0][:, 1], xr[:, 1] + 1.0)
    k = sv.export_dlpack("kinds")
    assert k.dtype == torch.uint32 and k.shape == (6 ** 3,)
    assert sv.gpu_scene_view()["binding_generation"] == gen
    with pytest.raises(Exception):
        sv.export_dlpack("no_such_buffer")


def test_incremental_update_equals_a_fresh_sync():
    w, desc, dt = scenes.xpbd_cube(n=6, spacing=0.1)
    a = Solver(desc)
    a.sync_world(w)
    gen = a.gpu_scene_view()["binding_generation"]
    ptr = a.gpu_scene_view()["positions_inv_mass"]
    # new velocities and stiffer tets, uploaded in place
    v = w.velocities()
    v[:, 0] = 0.3
    tets = w.array("tets").view(np.float32)
    tets[:, 5] *= 0.5
    a.update_world(w, "particle_state", "constraints")
    assert a.gpu_scene_view()["binding_generation"] == gen and a.gpu_scene_view()["positions_inv_mass"] == ptr
    b = Solver(desc)
    b.sync_world(w)
    for _ in range(3):
        a.step(dt)
        b.step(dt)
    xa, va, _ = a.read_particles()
    xb, vb, _ = b.read_particles()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_step_io_equals_write_step_read():
    """cn_solver_step_io (upload, frame, blocking readback on one stream) gives the bits of the
    three separate calls."""
    import ctypes as C
    import torch
    w, desc, dt = scenes.xpbd_cube(n=8, spacing=0.1, pin_bottom=False, lift=0.02)
    soa = w.soa()
    a, b = Solver(desc), Solver(desc)
    a.sync_world(soa)
    b.sync_world(soa)
    x0, v0, _ = a.read_particles()
    x0 = x0.copy()
    x0[:, 1] += 0.01
    n = x0.shape[0]
    xh = torch.from_numpy(x0.copy()).pin_memory()
    vh = torch.from_numpy(v0.copy()).pin_memory()
    f = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_float))
    for _ in range(3):
        assert a._lib.cn_solver_step_io(a._h, C.c_float(dt), f(xh), f(vh), f(xh), f(vh), None) == 0
    b.write_particles(x0, v0)
    for _ in range(3):
        xb, vb, _ = b.read_particles()
        b.write_particles(xb, vb)
        b.step(dt)
    xb, vb, _ = b.read_particles()
    assert np.array_equal(xh.numpy(), xb) and np.array_equal(vh.numpy(), vb)


def body_on_ground_with_tissue():
    from cn_physics import World
    w = World()
    w.add_soft_body_grid((0.2, 0.1, 0.2), 0.05, position=(0.6, 0.06, 0.0), radius=0.02)
    scenes.ground(w)
    tilt = (0.0871557, 0.0, 0.0, 0.9961947)   # 10 degrees about x: lands on an edge
    b = w.add_rigid_body("dynamic", position=(0.0, 0.15, 0.0), orientation=tilt, mass=1.0,
                         inverse_inertia=(3.0, 2.0, 1.0))
    w.add_collider(b, "box", (0.1, 0.05, 0.2), friction=0.5)
    w.soa()
    return w, b


def test_incremental_body_update_includes_the_inverse_inertia():
    """CN_SYNC_RIGID_BODIES uploads the inverse inertia too (as uploadRigidBodyRange,
    physics_scene_gpu_state.cpp:2702-2730): a box landing on an edge after the update moves as in
    a fresh sync of the updated world."""
    from cn_physics import solver_desc
    w, b = body_on_ground_with_tissue()
    desc = solver_desc(substeps=4, default_iterations=10)
    a = Solver(desc)
    a.sync_world(w)
    w.array("body_inverse_inertia")[b, :3] = (30.0, 20.0, 10.0)
    a.update_world(w, "rigid_bodies")
    fresh = Solver(desc)
    fresh.sync_world(w)
    for _ in range(30):
        a.step(1.0 / 60.0)
        fresh.step(1.0 / 60.0)
    for u, v in zip(a.read_rigid_bodies(), fresh.read_rigid_bodies()):
        assert np.array_equal(u, v)
    # the inertia matters here: the same frames with the synced inertia end elsewhere
    w.array("body_inverse_inertia")[b, :3] = (3.0, 2.0, 1.0)
    old = Solver(desc)
    old.sync_world(w)
    for _ in range(30):
        old.step(1.0 / 60.0)
    assert not np.array_equal(old.read_rigid_bodies()[1], fresh.read_rigid_bodies()[1])


def test_incremental_update_refuses_topology_and_body_type_changes():
    """The incidence tables and colourings are built from the constraints' particle indices, and
    the structural flags from the body types: changing either through cn_solver_update_world is
    refused (a full cn_solver_sync_world rebuilds them)."""
    from cn_physics import CNError, solver_desc
    w, b = body_on_ground_with_tissue()
    a = Solver(solver_desc(substeps=2))
    a.sync_world(w)
    edges = w.array("edges")
    edges[0, [0, 1]] = edges[0, [1, 0]]
    with pytest.raises(CNError):
        a.update_world(w, "constraints")
    edges[0, [0, 1]] = edges[0, [1, 0]]
    a.update_world(w, "constraints")            # same indices: accepted
    w.array("body_types")[b] = 1                 # dynamic -> kinematic
    with pytest.raises(CNError):
        a.update_world(w, "rigid_bodies")


def test_incremental_attribute_update_equals_a_fresh_sync_unless_it_changes_the_kernels():
    """A fluid material's viscosity uploaded in place gives the bits of a fresh sync; switching
    surface tension on would need the kernels built with those terms, so the update is refused."""
    from cn_physics import CNError
    w, desc, dt = scenes.dam_break(nx=12, ny=8, nz=12, box=(1.2, 0.8, 1.2))
    import ctypes as C
    from cn_physics import _abi
    soa = w.soa()
    fm = C.cast(C.c_void_p(soa.fluid_materials), C.POINTER(_abi.FluidMaterial))
    a = Solver(desc)
    a.sync_world(soa)
    fm[0].viscosity = fm[0].viscosity * 4.0
    a.update_world(soa, "particle_attributes")
    fresh = Solver(desc)
    fresh.sync_world(soa)
    for _ in range(3):
        a.step(dt)
        fresh.step(dt)
    xa, va, _ = a.read_particles()
    xf, vf, _ = fresh.read_particles()
    assert np.array_equal(xa, xf) and np.array_equal(va, vf)
    fm[0].surface_tension = 0.5
    with pytest.raises(CNError):
        a.update_world(soa, "particle_attributes")


def test_refused_incremental_update_uploads_nothing():
    """Disabling a collider changes the colliders that are queried: refused (a full sync rebuilds
    the query order), and the particle state flagged in the same call is not uploaded either."""
    import ctypes as C
    from cn_physics import CNError, solver_desc
    w, b = body_on_ground_with_tissue()
    desc = solver_desc(substeps=2, default_iterations=8)
    soa = w.soa()
    a, ref = Solver(desc), Solver(desc)
    a.sync_world(soa)
    ref.sync_world(soa)
    w.velocities()[:, 0] += 1.0
    words = np.ctypeslib.as_array(C.cast(C.c_void_p(soa.collider_broadphase), C.POINTER(C.c_uint32)),
                                  (soa.collider_count, 8))
    enabled = 5   # cn_collider_broadphase.enabled_flag
    assert words[:, enabled].all()
    words[-1, enabled] = 0
    with pytest.raises(CNError):
        a.update_world(soa, "particle_state", "colliders")
    for _ in range(3):
        a.step(1.0 / 60.0)
        ref.step(1.0 / 60.0)
    xa, va, _ = a.read_particles()
    xr, vr, _ = ref.read_particles()
    assert np.array_equal(xa, xr) and np.array_equal(va, vr)


def test_incremental_constraint_update_under_a_coloured_schedule_equals_a_fresh_sync():
    """The coloured schedules read colour-ordered copies of the edges and tets: an in-place update
    of the tet compliances refreshes them."""
    from cn_physics._abi import XPBD_COLOUR_GAUSS_SEIDEL
    w, desc, dt = scenes.xpbd_cube(n=6, spacing=0.1)
    desc.soft.xpbd_schedule = XPBD_COLOUR_GAUSS_SEIDEL
    a = Solver(desc)
    a.sync_world(w)
    tets = w.array("tets").view(np.float32)
    tets[:, 5] = tets[:, 5] * 0.25 + 1e-7
    a.update_world(w, "constraints")
    fresh = Solver(desc)
    fresh.sync_world(w)
    for _ in range(3):
        a.step(dt)
        fresh.step(dt)
    xa, va, _ = a.read_particles()
    xf, vf, _ = fresh.read_particles()
    assert np.array_equal(xa, xf) and np.array_equal(va, vf)
