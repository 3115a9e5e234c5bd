"""The reference's own preconditioner ordering on the GPU (SI3D_ORDER_NATURAL) against the oracle's
natural-order NSPCG mic1 + cg (nspcg.f:21759-21805, :22875-22922, :22729-22777, itcg :8967-9092).

With the same ordering the GPU and the oracle run the same algorithm row for row; only the order of
the dot-product sums differs, so iteration counts agree within one and the solutions to the
stopping tolerance.  Stopping test 2 at 1e-6 is the reference's setting (si3d_procedures.f90:
1989-1995) with chgcon's adaptive eigenvalue estimate; test 5 at 1e-12 is the parity setting."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _purdue_system(o):
    """SolverSparse's Purdue arrays (coeffA, jcoefA, rhs, x0) of the oracle's current matcon state."""
    lm, lm1 = o.lm, o.lm1
    lEC, lWC, lNC, lSC = (o.geti(n) for n in ("lEC", "lWC", "lNC", "lSC"))
    sx, sy, rr, qq, sp = (o.get(n) for n in ("sx", "sy", "rr", "qq", "sp"))
    m = np.arange(lm)
    coef = np.zeros((lm, 5))
    jco = np.zeros((lm, 5), dtype=np.int32)
    coef[:, 0] = rr[m]
    coef[:, 1] = -sx[lWC[m] - 1]
    coef[:, 2] = -sy[lSC[m] - 1]
    coef[:, 3] = -sy[m]
    coef[:, 4] = -sx[m]
    jco[:, 0] = m + 1
    for c, nb in ((1, lWC), (2, lSC), (3, lNC), (4, lEC)):
        jco[:, c] = np.where(nb[m] == lm1, 0, nb[m])
    return coef, jco, qq[:lm].copy(), sp[:lm].copy()


@pytest.mark.parametrize("test,tol", [(2, 1e-6), (5, 1e-12)])
def test_natural_standalone_fixture(native_libs, oracle_lib, test, tol):
    from si3d_b200 import native
    from si3d_b200.model import solve_zeta
    g = np.load(os.path.join(ROOT, "tests", "golden", "pcg_48x32.npz"))
    x0 = np.zeros_like(g["rhs"])
    x_o, r_o = oracle_lib.pcg(g["coef"], g["jcoef"], g["rhs"], x0, pcg_test=test, tol=tol, itmax=500, ordering=0)
    x_g, r_g = solve_zeta(g["coef"], g["jcoef"], g["rhs"], x0, pcg_test=test, tol=tol, itmax=500,
                          ordering=native.SI3D_ORDER_NATURAL)
    assert r_o["ier"] == 0 and r_g["ier"] == 0
    assert abs(r_g["iters"] - r_o["iters"]) <= 1, (r_g["iters"], r_o["iters"])
    if test == 2:
        assert r_g["emin"] == pytest.approx(r_o["emin"], rel=1e-6)
        assert r_g["emax"] == pytest.approx(r_o["emax"], rel=1e-6)
    assert np.abs(x_g - x_o).max() <= (1e-5 if test == 2 else 1e-10) * np.abs(x_o).max()


@pytest.mark.parametrize("name", ["t1", "c0"])
@pytest.mark.parametrize("test,tol", [(2, 1e-6), (5, 1e-12)])
def test_natural_standalone_zeta_system(native_libs, oracle_lib, run_dirs, name, test, tol):
    """The zeta system SolverSparse hands NSPCG after a few steps of t1 and c0."""
    from si3d_b200 import native
    from si3d_b200.model import solve_zeta
    o = oracle_lib.OracleRun(run_dirs[name], ordering=0)
    o.run(2)
    o.stage("momentum", 2)
    o.stage("matcon", 2)
    coef, jco, b, x0 = _purdue_system(o)
    x_o, r_o = oracle_lib.pcg(coef, jco, b, x0, pcg_test=test, tol=tol, itmax=2000, ordering=0)
    x_g, r_g = solve_zeta(coef, jco, b, x0, pcg_test=test, tol=tol, itmax=2000, ordering=native.SI3D_ORDER_NATURAL)
    assert r_o["ier"] == 0 and r_g["ier"] == 0
    assert abs(r_g["iters"] - r_o["iters"]) <= 1, (r_g["iters"], r_o["iters"])
    scale = max(np.abs(x_o).max(), 1e-3)
    assert np.abs(x_g - x_o).max() <= (1e-6 if test == 2 else 1e-11) * scale


def test_natural_steps_stopping_test_2(native_libs, oracle_lib, run_dirs):
    """Whole time steps with the reference's solver settings (natural-order MIC, test 2, 1e-6, at most
    200 iterations): per-solve iteration counts within one of the oracle's."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    steps = 5
    o = oracle_lib.OracleRun(run_dirs["t1"], pcg_test=2, pcg_tol=1e-6, pcg_itmax=200, ordering=0)
    o.run(steps)
    it_o = [s["iters"] for s in o.solves()]
    run = GpuRun(run_dirs["t1"], pcg_test=2, pcg_tol=1e-6, pcg_itmax=200, ordering=native.SI3D_ORDER_NATURAL)
    try:
        st = run.run(steps)
        it_g = [s.iters[i] for s in st for i in range(s.nsolves)]
        assert len(it_g) == len(it_o)
        assert max(abs(a - b) for a, b in zip(it_g, it_o)) <= 1, (it_g, it_o)
        s_o = o.get("s")[:o.lm]
        assert np.abs(run.get("s")[:run.lm] - s_o).max() <= 1e-6 * max(np.abs(s_o).max(), 1e-3)
    finally:
        run.close()


def test_natural_steps_match_oracle(native_libs, oracle_lib, run_dirs):
    """30 steps of c0 at test 5, 1e-12 with the natural ordering on both sides: iteration counts
    within one per solve, zeta within 1e-9 m, velocities and temperature at the plain tolerances."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    steps = 30
    o = oracle_lib.OracleRun(run_dirs["c0"], ordering=0, pcg_itmax=2000)
    o.run(steps)
    run = GpuRun(run_dirs["c0"], pcg_itmax=2000, ordering=native.SI3D_ORDER_NATURAL)
    try:
        st = run.run(steps)
        it_o = [s["iters"] for s in o.solves()]
        it_g = [s.iters[i] for s in st for i in range(s.nsolves)]
        assert len(it_g) == len(it_o)
        assert max(abs(a - b) for a, b in zip(it_g, it_o)) <= 1, (it_g[:9], it_o[:9])
        assert np.abs(run.get("s") - o.get("s")).max() <= 1e-9
        for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("sal", 1e-10)):
            a = o.get(f)
            assert np.abs(run.get(f) - a).max() <= tol * np.abs(a).max(), f
    finally:
        run.close()
