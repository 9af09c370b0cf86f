"""The allocation-free broadphase sort (cn_sort_cell_keys_noalloc) against the solver's own sort.

This entry point serves callers that may not allocate device memory while they run (engines that
own every device byte through their own pool, frame loops that cannot take the allocator's
implicit synchronisation).  The test feeds it the cell keys of a real broadphase step and checks
its (key, index) output bit-for-bit against the sort the solver ran through cn_solver_step, on two
calls in a row with different keys, so contents the shared scratch keeps from the first call
cannot leak into the second.  A second test sorts random keys (with many duplicates and the
largest key 0xffffffff) of sizes from one key to the limit, largest first, so stale look-back
words of a bigger call would show in a smaller one, and reads the timeout count each time.
This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from cn_physics import Solver, load, scenes


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_rejects_counts_above_the_limit_without_touching_the_gpu():
    lib = load()
    status = lib.cn_sort_cell_keys_noalloc(None, None, None, (1 << 20) + 1, None, None)
    assert status == 5  # CN_ERR_CAPACITY
    assert b"1048576" in lib.cn_last_error()


def test_rejects_aliased_buffers_without_touching_the_gpu():
    lib = load()
    buf = C.c_void_p(0x10000)
    status = lib.cn_sort_cell_keys_noalloc(buf, buf, C.c_void_p(0x20000), 16, None, None)
    assert status == 1  # CN_ERR_INVALID_ARGUMENT
    assert b"alias" in lib.cn_last_error()


@pytest.mark.gpu
def test_noalloc_sort_matches_solver_sort_on_two_calls():
    import torch

    lib = load()
    w, desc, dt = scenes.dam_break(nx=48, ny=32, nz=48)      # 73,728 particles
    solver = Solver(desc)
    solver.set_debug(force_broadphase=True)
    solver.sync_world(w.soa())
    previous = None
    for call in range(2):
        solver.step(dt)
        entries = solver.debug_read("cell_entries").view(np.int32).reshape(-1, 4)
        keys = entries[:, 3].view(np.uint32).copy()
        expected = solver.debug_read("sorted_keys").view(np.uint32).reshape(-1, 2)
        if previous is not None:
            assert not np.array_equal(keys, previous)           # the second call sorts new keys
        previous = keys
        n = keys.size
        d_keys = torch.from_numpy(keys.view(np.int32)).cuda()
        d_sorted = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        d_index = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        d_timeouts = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        status = lib.cn_sort_cell_keys_noalloc(_ptr(d_keys), _ptr(d_sorted), _ptr(d_index), n, _ptr(d_timeouts),
                                               C.c_void_p(stream))
        assert status == 0, lib.cn_last_error()
        torch.cuda.synchronize()
        got_keys = d_sorted.cpu().numpy().view(np.uint32)
        got_index = d_index.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_keys, expected[:, 0]), call
        assert np.array_equal(got_index, expected[:, 1]), call
        assert np.array_equal(d_keys.cpu().numpy().view(np.uint32), keys)   # input untouched
        assert int(d_timeouts.item()) == 0


@pytest.mark.gpu
def test_noalloc_sort_sizes_largest_first_against_stable_argsort():
    import torch

    lib = load()
    rng = np.random.default_rng(7)
    stream = torch.cuda.current_stream().cuda_stream
    for n in (1 << 20, 1_000_003, 4097, 4096, 1):
        keys = rng.integers(0, 4096, size=n, dtype=np.uint64).astype(np.uint32) * np.uint32(1048573)
        keys[rng.random(n) < 0.05] = 0xFFFFFFFF
        expected = np.argsort(keys, kind="stable").astype(np.uint32)
        d_keys = torch.from_numpy(keys.view(np.int32)).cuda()
        d_sorted = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        d_index = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        d_timeouts = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        status = lib.cn_sort_cell_keys_noalloc(_ptr(d_keys), _ptr(d_sorted), _ptr(d_index), n, _ptr(d_timeouts),
                                               C.c_void_p(stream))
        assert status == 0, lib.cn_last_error()
        torch.cuda.synchronize()
        assert int(d_timeouts.item()) == 0, n
        assert np.array_equal(d_index.cpu().numpy().view(np.uint32), expected), n
        assert np.array_equal(d_sorted.cpu().numpy().view(np.uint32), keys[expected]), n
