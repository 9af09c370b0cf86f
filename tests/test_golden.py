"""The committed golden vectors (tests/golden/*.npz, written by tests/golden/make_golden.py).

CPU: the oracle still reproduces every file bit for bit (it may not drift).
GPU: the sm_100a path, through the C ABI, reproduces every file bit for bit -- positions,
velocities, previous positions, the sorted (cellKey, index) pairs, neighbour counts and the
SHA-256 of the neighbour lists of the last substep -- except the scenes whose constraints go
through acos (make_golden.TRANSCENDENTAL), held to 1e-5.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

NAMES = sorted(make_golden.SCENES)


def _compare(name, got):
    ref = np.load(GOLDEN / f"{name}.npz")
    assert sorted(ref.files) == sorted(got), name
    for key in ref.files:
        a, b = np.asarray(got[key]), ref[key]
        assert a.shape == b.shape and a.dtype == b.dtype, (name, key)
        if not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
            diff = np.abs(a.astype(np.float64) - b.astype(np.float64)).max() if a.dtype.kind == "f" else "-"
            raise AssertionError(f"{name}/{key} differs from the golden file (max abs diff {diff})")


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    _compare(name, make_golden.run(make_golden.oracle_stepper, name))


def _gpu_stepper(desc, soa):
    from cn_physics import Solver
    s = Solver(desc)
    s.set_debug(post_update_neighbors=True)  # the oracle's lists are rebuilt after the update
    s.sync_world(soa)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_golden(name):
    got = make_golden.run(_gpu_stepper, name)
    if name in make_golden.TRANSCENDENTAL:
        make_golden.assert_state_close(name, got, np.load(GOLDEN / f"{name}.npz"))
        return
    _compare(name, got)


def _gpu_default_stepper(desc, soa):
    from cn_physics import Solver
    s = Solver(desc)          # the shipped schedule: no debug flags
    s.sync_world(soa)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_default_schedule_reproduces_golden_state(name):
    """Without the post-update neighbour rebuild (which only feeds vorticity confinement and
    render anisotropy) the state and the sorted key pairs are the golden file's, bit for bit."""
    got = make_golden.run(_gpu_default_stepper, name)
    ref = np.load(GOLDEN / f"{name}.npz")
    if name in make_golden.TRANSCENDENTAL:
        make_golden.assert_state_close(name, got, ref)
        return
    for key in ("x", "v", "x_prev", "sorted_keys"):
        if key in ref.files:
            assert np.array_equal(np.asarray(got[key]).view(np.uint8), ref[key].view(np.uint8)), (name, key)
