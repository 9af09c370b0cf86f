"""Reference fixtures: the golden scenes stepped by the reference's OWN compute shaders.

oracle/ref_build.py compiles the reference's HLSL kernels (assets/shaders/physics/**) for the host
and oracle/ref_driver.py dispatches them in PhysicsSolver::step's order.  This script steps every
scene of make_golden.SCENES through them and writes tests/golden/ref_<scene>.npz: the state after
the scene's frames (plus, for fluid scenes, the sorted (cellKey, index) pairs and the neighbour
lists of the last build) and, for fluid scenes, the state after the first frame.

    python oracle/ref_build.py && python tests/golden/make_ref_golden.py

It needs the reference tree (CN_REFERENCE_ROOT, default /root/reference) and runs only where it
is present; the fixtures it writes are committed, so the tests that read them need neither.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (ROOT / "cressim-neo_b200", ROOT / "oracle", HERE):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import make_golden  # noqa: E402


def ref_stepper(desc, soa):
    import ref_driver
    return ref_driver.RefSolver(desc, soa)


def fixture(name: str) -> dict:
    out = make_golden.run(ref_stepper, name)
    if make_golden.SCENES[name][2]:
        one = make_golden.run(ref_stepper, name, frames=1)
        for k, v in one.items():
            out["frame1_" + k] = v
    return out


def main(names=None):
    import ref_build
    if ref_build.build() is None:
        raise SystemExit("reference tree not found (set CN_REFERENCE_ROOT)")
    for name in names or make_golden.SCENES:
        arrays = fixture(name)
        np.savez_compressed(HERE / f"ref_{name}.npz", **arrays)
        print(name, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main(sys.argv[1:] or None)
