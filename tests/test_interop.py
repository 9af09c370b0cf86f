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
