"""Shared test set-up: import paths, the gpu marker and oracle fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "fe-c_eutectoid_phase-field_simulation_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200 host)")


@pytest.fixture(scope="session")
def port():
    from oracle import pyoracle

    return pyoracle.port()


@pytest.fixture(scope="session")
def reference():
    """The unmodified reference solver; skips where its source was never available."""
    from oracle import pyoracle

    ref = pyoracle.reference()
    if ref is None:
        pytest.skip("reference solver not built here (its source is absent)")
    return ref


@pytest.fixture(scope="session")
def gpu_lib():
    import pearl_gpu
    from pearl_gpu import build

    build.build()
    return pearl_gpu.library()
