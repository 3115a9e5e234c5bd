"""Shared fixtures: built libraries, generated reference-format runs, the CPU oracle."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def native_libs():
    from si3d_b200 import build
    build.build_all()
    from si3d_b200 import native
    return native


@pytest.fixture(scope="session")
def tracer_dirs(tmp_path_factory):
    """The small runs with three conservative tracers (a step, a Gaussian band, a uniform field)."""
    from si3d_b200 import synth
    base = tmp_path_factory.mktemp("tracer_runs")
    out = {}
    for name in ("t0", "t1", "c0"):
        d = str(base / name)
        synth.make(name, d, ntr=3)
        out[name] = d
    return out


@pytest.fixture(scope="session")
def turb_dirs(tmp_path_factory):
    """The small runs with the Mellor-Yamada 2.5 closure (iturb = 1)."""
    from si3d_b200 import synth
    base = tmp_path_factory.mktemp("turb_runs")
    out = {}
    for name in ("t0", "t1", "c0"):
        d = str(base / name)
        synth.make(name, d, iturb=1)
        out[name] = d
    return out


@pytest.fixture(scope="session")
def run_dirs(tmp_path_factory):
    """Small reference-format runs shared by the tests."""
    from si3d_b200 import synth
    base = tmp_path_factory.mktemp("runs")
    out = {}
    for name in ("t0", "t1", "c0"):
        d = str(base / name)
        synth.make(name, d)
        out[name] = d
    return out
