"""Shared test setup: import paths, markers and library builds."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "cressim-neo_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _libraries():
    """Builds the CPU oracle and the sm_100a library in-tree when they are missing."""
    import cn_oracle  # noqa: F401  (test infrastructure)
    if not cn_oracle.LIB.exists():
        cn_oracle.build()
    lib = ROOT / "cressim-neo_b200" / "libcn_physics.so"
    if not lib.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("cn_build", ROOT / "cressim-neo_b200" / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    yield


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
