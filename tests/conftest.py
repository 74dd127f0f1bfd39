"""Shared test setup: the `gpu` marker, import paths, and an in-tree build of
the product library and the oracle when they are missing."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "general-simulator_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


def _ensure_built():
    import build  # general-simulator_b200/build.py

    if not os.path.exists(build.LIB):
        build.build_lib()
    if not os.path.exists(build.LIB_BC):
        build.build_lib(bounds_check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        build.build_oracle()


_ensure_built()


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gb():
    import gs_b200

    return gs_b200


@pytest.fixture(scope="session")
def orc():
    import oracle_py

    return oracle_py


def rel_l2(a, b):
    import numpy as np

    a = np.asarray(a)
    b = np.asarray(b)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d
