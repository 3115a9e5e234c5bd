"""Committed fixtures (tests/golden/, made by tests/golden/make_golden.py from the CPU oracle).

CPU: the oracle still reproduces them.  GPU: the CUDA path matches them without running the
oracle (plain FP64: zeta to 1e-10 m, velocities and temperature to 1e-9 relative, iteration counts
within 2 per solve; the standalone solve to 1e-9 of the solution's scale)."""
import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = os.path.join(ROOT, "tests", "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLD, name)))


@pytest.mark.parametrize("name", ["t0", "t1"])
def test_oracle_reproduces_fixture(oracle_lib, run_dirs, name):
    g = _load(f"{name}_oracle_10steps.npz")
    o = oracle_lib.OracleRun(run_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(int(g["steps"]))
    np.testing.assert_allclose(o.get("s")[:o.lm], g["s"], rtol=1e-12, atol=1e-15)
    for f in ("uh", "vh", "sal", "wp"):
        if f in g:
            np.testing.assert_allclose(o.get(f)[:, :o.lm], g[f], rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal([s["iters"] for s in o.solves()], g["iters"])


def test_oracle_reproduces_pcg_fixture(oracle_lib):
    g = _load("pcg_48x32.npz")
    x, info = oracle_lib.pcg(g["coef"], g["jcoef"], g["rhs"], np.zeros_like(g["rhs"]), pcg_test=5, tol=1e-12,
                             itmax=500, ordering=1)
    assert info["iters"] == int(g["iters"])
    np.testing.assert_allclose(x, g["x"], rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t0", "t1"])
def test_gpu_matches_fixture(native_libs, run_dirs, name):
    from si3d_b200.model import GpuRun
    g = _load(f"{name}_oracle_10steps.npz")
    run = GpuRun(run_dirs[name], pcg_itmax=2000)
    try:
        stats = run.run(int(g["steps"]))
        s = run.get("s")[:run.lm]
        assert np.abs(s - g["s"]).max() <= 1e-10
        for f in ("uh", "vh", "sal"):
            if f in g:
                a = run.get(f)[:, :run.lm]
                scale = max(np.abs(g[f]).max(), 1e-30)
                assert np.abs(a - g[f]).max() <= 1e-9 * scale, f
        iters = [st.iters[i] for st in stats for i in range(st.nsolves)]
        assert len(iters) == len(g["iters"])
        assert max(abs(a - b) for a, b in zip(iters, g["iters"])) <= 2
    finally:
        run.close()


@pytest.mark.gpu
def test_gpu_standalone_solve_matches_fixture(native_libs):
    from si3d_b200.model import solve_zeta
    g = _load("pcg_48x32.npz")
    x, info = solve_zeta(g["coef"], g["jcoef"], g["rhs"], np.zeros_like(g["rhs"]), itmax=500)
    assert info["ier"] == 0 and info["stptst"] < 1e-12
    assert abs(info["iters"] - int(g["iters"])) <= 2
    assert np.abs(x - g["x"]).max() <= 1e-9 * np.abs(g["x"]).max()


TRACERS = ("tracer1", "tracer2", "tracer3")


def test_oracle_reproduces_tracer_fixture(oracle_lib, tracer_dirs):
    g = _load("t0_tracers3_oracle_10steps.npz")
    o = oracle_lib.OracleRun(tracer_dirs["t0"], ordering=1, pcg_itmax=2000)
    o.run(int(g["steps"]))
    for f in TRACERS:
        np.testing.assert_allclose(o.get(f)[:, :o.lm], g[f], rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_gpu_matches_tracer_fixture(native_libs, tracer_dirs):
    """Three conservative tracers after 10 steps on t0, against the stored oracle values."""
    from si3d_b200.model import GpuRun
    g = _load("t0_tracers3_oracle_10steps.npz")
    run = GpuRun(tracer_dirs["t0"], pcg_itmax=2000)
    try:
        run.run(int(g["steps"]))
        assert np.abs(run.get("s")[:run.lm] - g["s"]).max() <= 1e-10
        for f in TRACERS:
            assert np.abs(run.get(f)[:, :run.lm] - g[f]).max() <= 1e-9 * np.abs(g[f]).max(), f
    finally:
        run.close()
