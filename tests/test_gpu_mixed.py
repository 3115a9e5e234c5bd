"""Mixed-precision forms: FP32 inner solves (MIC-PCG, or aggregation-multigrid PCG) inside FP64
iterative refinement, through the C ABI, against the FP64 oracle.  The stopping test stays test 5 at
1e-12 on the FP64 residual."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["MIXED_IR", "MIXED_MG"])
@pytest.mark.parametrize("name,steps", [("t0", 30), ("t1", 30), ("c0", 30)])
def test_mixed_ir_matches_fp64_oracle(run_dirs, oracle_lib, native_libs, name, steps, precision):
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(run_dirs[name], ordering=1, pcg_itmax=2000)
    g = GpuRun(run_dirs[name], pcg_itmax=2000, precision=getattr(native, f"SI3D_{precision}"))
    o.run(steps)
    st = g.run(steps)
    relres = [s.relres[i] for s in st for i in range(s.nsolves)]
    assert max(relres) < 1e-12, max(relres)
    assert all(s.ier[i] == 0 for s in st for i in range(s.nsolves))
    ds = np.abs(o.get("s") - g.get("s")).max()
    assert ds <= 1e-9, f"max |dzeta| {ds:.3e} m"
    for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("sal", 1e-10)):
        a, b = o.get(f), g.get(f)
        err = np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)
        assert err <= tol, f"{name}:{f} rel err {err:.3e}"


def test_mixed_standalone_solve(run_dirs, oracle_lib, native_libs):
    from si3d_b200 import native
    from si3d_b200.model import solve_zeta
    o = oracle_lib.OracleRun(run_dirs["t1"], ordering=1)
    o.run(2)
    o.stage("momentum", 1)
    o.stage("matcon", 1)
    lm, lm1 = o.lm, o.lm1
    lEC, lWC, lNC, lSC = (o.geti(n) for n in ("lEC", "lWC", "lNC", "lSC"))
    sx, sy, rr, qq, sp = (o.get(n) for n in ("sx", "sy", "rr", "qq", "sp"))
    m = np.arange(lm)
    coef = np.stack([rr[m], -sx[lWC[m] - 1], -sy[lSC[m] - 1], -sy[m], -sx[m]], axis=1)
    jco = np.zeros((lm, 5), dtype=np.int32)
    jco[:, 0] = m + 1
    for c, nb in ((1, lWC), (2, lSC), (3, lNC), (4, lEC)):
        jco[:, c] = np.where(nb[m] == lm1, 0, nb[m])
    x_o, r_o = oracle_lib.pcg(coef, jco, qq[:lm], sp[:lm], ordering=0, itmax=2000)
    x_g, r_g = solve_zeta(coef, jco, qq[:lm], sp[:lm], itmax=2000, precision=native.SI3D_MIXED_IR)
    assert r_g["stptst"] < 1e-12
    assert np.abs(x_g - x_o).max() <= 1e-10 * max(np.abs(x_o).max(), 1e-3)


def test_multigrid_inner_solves_need_few_iterations(run_dirs, native_libs):
    """The multigrid V-cycle makes the inner iteration count nearly independent of the system: on
    t1 every step's MG inner iterations stay below a quarter of the MIC inner iterations."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    its = {}
    for prec in ("MIXED_IR", "MIXED_MG"):
        g = GpuRun(run_dirs["t1"], pcg_itmax=2000, precision=getattr(native, f"SI3D_{prec}"))
        try:
            st = g.run(10)
            its[prec] = [s.total_iters for s in st]
        finally:
            g.close()
    assert all(4 * m < i for m, i in zip(its["MIXED_MG"], its["MIXED_IR"])), its


def test_multigrid_needs_the_grid_image():
    """Without the (i, j) maps the hierarchy cannot be built: the standalone solve refuses the MG
    form instead of falling back to another solver."""
    import numpy as np
    from si3d_b200 import native
    from si3d_b200.model import solve_zeta
    coef = np.array([[4.0, -1.0, 0, 0, 0], [4.0, 0, 0, 0, -1.0]])
    jco = np.array([[1, 2, 0, 0, 0], [2, 0, 0, 0, 1]], dtype=np.int32)
    with pytest.raises(Exception):
        solve_zeta(coef, jco, np.ones(2), np.zeros(2), itmax=50, precision=native.SI3D_MIXED_MG)


@pytest.mark.parametrize("istep", [1, 2])
@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_multigrid_solve_matches_restatement(run_dirs, oracle_lib, native_libs, name, istep):
    """One MIXED_MG zeta solve against the numpy restatement of the same solve (same hierarchy,
    half-sweeps, FP32 CG recurrences and FP64 refinement): the inner iteration totals agree up to
    reduction-order rounding and both zeta meet the 1e-12 test."""
    from oracle import mg_numpy
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    from test_gpu_parity import STATE_2D, STATE_3D, STATE_I
    o = oracle_lib.OracleRun(run_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(2)
    o.stage("momentum", istep)
    o.stage("matcon", istep)
    g = GpuRun(run_dirs[name], pcg_itmax=2000, precision=native.SI3D_MIXED_MG)
    try:
        for f in STATE_3D:
            g.set(f, o.get(f))
        for f in STATE_2D:
            g.set(f, o.get(f))
        for f in STATE_I:
            g.set(f, o.geti(f))
        maps = [o.geti(n) for n in ("l2i", "l2j", "lEC", "lWC", "lNC", "lSC")]
        sx, sy, qq, sp = (o.get(n) for n in ("sx", "sy", "qq", "sp"))
        z, info = mg_numpy.solve(o.lm, *maps, sx, sy, qq, sp, o.im1, o.jm1)
        st = g.stage("solve", istep)
        assert st.nsolves == 1 and st.ier[0] == 0 and st.relres[0] < 1e-12
        assert abs(st.iters[0] - info["iters"]) <= 2, (st.iters[0], info)
        zg = g.get("s")[:o.lm]
        assert np.abs(zg - z).max() <= 1e-10 * max(np.abs(z).max(), 1e-3)
    finally:
        g.close()
