"""Mellor-Yamada 2.5 closure (iturb = 1) on the GPU, through the C ABI, against the CPU oracle: the
closure stage from the oracle's state (q2, q2l and the eddy coefficients), and whole runs in which
the eddy coefficients feed back into momentum and temperature."""
import numpy as np
import pytest

from test_gpu_parity import STATE_2D, STATE_3D, STATE_I

pytestmark = pytest.mark.gpu

TURB = ["q2", "q2p", "q2pp", "q2l", "q2lp", "q2lpp", "u", "v"]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_closure_stage_matches_oracle(turb_dirs, oracle_lib, native_libs, name):
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(turb_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(3)
    for st in ("momentum", "matcon", "solve", "vel", "scalar", "vel2"):
        o.stage(st, 2)
    g = GpuRun(turb_dirs[name], pcg_itmax=2000)
    try:
        for f in STATE_3D + TURB:
            g.set(f, o.get(f))
        for f in STATE_2D:
            g.set(f, o.get(f))
        for f in STATE_I:
            g.set(f, o.geti(f))
        o.stage("turbulence", 2)
        g.stage("turbulence", 2)
        for f in ("q2", "q2l", "Av", "Dv"):
            assert _rel(o.get(f), g.get(f)) <= 1e-12, f
    finally:
        g.close()


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_closure_runs_match_oracle(turb_dirs, oracle_lib, native_libs, name):
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(turb_dirs[name], ordering=1, pcg_itmax=2000)
    g = GpuRun(turb_dirs[name], pcg_itmax=2000)
    try:
        for f in TURB[:6]:
            np.testing.assert_array_equal(g.get(f), o.get(f), err_msg=f)
        o.run(20)
        st = g.run(20)
        assert all(s.ier[i] == 0 for s in st for i in range(s.nsolves))
        assert np.abs(o.get("s") - g.get("s")).max() <= 1e-9
        for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("sal", 1e-10), ("q2", 1e-8), ("q2l", 1e-8), ("Av", 1e-8),
                       ("Dv", 1e-8)):
            assert _rel(o.get(f), g.get(f)) <= tol, f
    finally:
        g.close()


def test_closure_with_tracers_and_outputs(tmp_path, oracle_lib, native_libs):
    """Every addition at once on t1: the closure feeds Dv to temperature and tracer diffusion and Av
    to momentum, two tracers, and the plane, tracer and ptrack files; 12 steps against the oracle."""
    import os
    import shutil
    from si3d_b200 import synth
    from si3d_b200.model import GpuRun
    from test_outputs_oracle import read_records
    out = dict(iop=4, planes=(3, 99), ipxml=6, iotr=4)
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "oracle")
    synth.make("t1", dg, ntr=2, iturb=1, outputs=out)
    shutil.copytree(dg, do)
    g = GpuRun(dg, pcg_itmax=2000)
    o = oracle_lib.OracleRun(do, ordering=1, pcg_itmax=2000)
    try:
        g.run(12)
        o.run(12)
        assert np.abs(o.get("s") - g.get("s")).max() <= 1e-9
        for f, tol in (("uh", 1e-8), ("sal", 1e-10), ("tracer1", 1e-9), ("tracer2", 1e-9), ("q2", 1e-8), ("Dv", 1e-8)):
            assert _rel(o.get(f), g.get(f)) <= tol, f
        for name in ("si3d_3D", "tracer_1", "tracer_2", "plane_3", "plane_99"):
            rg, ro = read_records(os.path.join(dg, name)), read_records(os.path.join(do, name))
            assert [len(r) for r in rg] == [len(r) for r in ro] and rg[:3] == ro[:3], name
    finally:
        g.close()
        o.close()
