import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cmc-fluid-solver_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_oracle():
    lib = os.path.join(ORACLE, "liboracle_adi.so")
    src = [os.path.join(ORACLE, f) for f in ("adi_oracle.c", "adi_oracle_body.h")]
    if not os.path.exists(lib) or any(os.path.getmtime(s) > os.path.getmtime(lib) for s in src):
        subprocess.run(["make", "-C", ORACLE, "oracle"], check=True, stdout=subprocess.DEVNULL)


_ensure_oracle()


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="session")
def adi_lib():
    """libadi_b200.so, built in-tree if it is missing or stale."""
    sys.path.insert(0, PKG)
    import build_adi as adi_build  # cmc-fluid-solver_b200/build_adi.py
    adi_build.build()
    import adi_b200
    return adi_b200
