"""Conservative tracers on the GPU (exTracer + ImTracer for all tracers in two launches, the
persistent flux arrays brought to the reference's final state by a third), through the C ABI,
against the CPU oracle.  Runs carry three tracers: a step, a Gaussian band and a uniform field."""
import numpy as np
import pytest

from test_gpu_parity import STATE_2D, STATE_3D, STATE_I

pytestmark = pytest.mark.gpu

TRACERS = [f"tracer{t}" for t in (1, 2, 3)] + [f"tracerpp{t}" for t in (1, 2, 3)]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)


@pytest.mark.parametrize("name", ["t0", "c0"])
def test_initial_tracers_match_oracle(tracer_dirs, oracle_lib, native_libs, name):
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(tracer_dirs[name])
    g = GpuRun(tracer_dirs[name])
    try:
        for f in TRACERS:
            np.testing.assert_array_equal(g.get(f), o.get(f), err_msg=f)
    finally:
        g.close()


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_tracer_stage_matches_oracle(tracer_dirs, oracle_lib, native_libs, name):
    """One exTracer + ImTracer pass for every tracer from the oracle's state after three steps:
    tracers and the persistent flux arrays the pass leaves behind."""
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(tracer_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(3)
    for st in ("momentum", "matcon", "solve", "vel", "scalar"):
        o.stage(st, 2)
    g = GpuRun(tracer_dirs[name], pcg_itmax=2000)
    try:
        for f in STATE_3D + TRACERS:
            g.set(f, o.get(f))
        for f in STATE_2D:
            g.set(f, o.get(f))
        for f in STATE_I:
            g.set(f, o.geti(f))
        o.stage("tracer", 2)
        g.stage("tracer", 2)
        for f in ("tracer1", "tracer2", "tracer3", "Bth2", "Bth3", "Bth4"):
            assert _rel(o.get(f), g.get(f)) <= 1e-12, f
        for t in (1, 2, 3):   # tracerpp is an input only
            np.testing.assert_array_equal(g.get(f"tracerpp{t}"), o.get(f"tracerpp{t}"))
    finally:
        g.close()


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_tracer_runs_match_oracle(tracer_dirs, oracle_lib, native_libs, name):
    """30 whole steps (the tracer block runs on the last trapezoidal iteration of each step, and
    save hands tracer to tracerpp): tracers agree with the oracle, the GPU conserves tracer mass,
    and the uniform tracer stays uniform."""
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(tracer_dirs[name], ordering=1, pcg_itmax=2000)
    g = GpuRun(tracer_dirs[name], pcg_itmax=2000)
    try:
        kmz = o.geti("kmz")[:o.lm]
        K = np.arange(1, o.km1 + 1)[:, None]
        wet = (K >= 2) & (K <= kmz[None, :])

        def mass(t):
            return float((g.get(f"tracerpp{t}")[:, :o.lm] * g.get("hp")[:, :o.lm] * wet).sum())

        m0 = [mass(t) for t in (1, 2, 3)]
        o.run(30)
        st = g.run(30)
        assert all(s.ier[i] == 0 for s in st for i in range(s.nsolves))
        for f in TRACERS:
            assert _rel(o.get(f), g.get(f)) <= 1e-9, f
        for t in (1, 2, 3):
            np.testing.assert_array_equal(g.get(f"tracer{t}"), g.get(f"tracerpp{t}"))
        m1 = [mass(t) for t in (1, 2, 3)]
        for a, b in zip(m0, m1):
            assert abs(b - a) <= 1e-12 * a, (m0, m1)
        k1z = g.get("k1z")[:o.lm]
        top = (K >= k1z[None, :]) & (K <= kmz[None, :])
        assert np.abs(g.get("tracer3")[:, :o.lm][top] - 0.5).max() <= 1e-13
    finally:
        g.close()


def test_tracer_fields_through_the_abi(tracer_dirs, native_libs):
    """Setting one tracer field leaves the other time level alone; unknown tracer numbers are
    refused."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    g = GpuRun(tracer_dirs["t0"])
    try:
        g.run(2)
        before = g.get("tracerpp2")
        x = np.random.default_rng(1).uniform(0, 1, before.shape)
        g.set("tracer2", x)
        np.testing.assert_array_equal(g.get("tracer2"), x)
        np.testing.assert_array_equal(g.get("tracerpp2"), before)
        with pytest.raises(native.Si3dError):
            g.get("tracer4")
        g.run(1)   # the next save copies instead of swapping; the run goes on
        np.testing.assert_array_equal(g.get("tracer2"), g.get("tracerpp2"))
    finally:
        g.close()
