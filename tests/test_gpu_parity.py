"""GPU path vs the CPU oracle, through the C ABI.

Stage tests start both from the same state (the oracle's state after a few steps, copied into the
device) and run one routine on each side; the column stages must agree to the last bit or within a
few ulps, the zeta solve to its stopping tolerance.  Run tests advance whole time steps
(si3d.f90:324-458) on both sides and compare every prognostic field.
"""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

STATE_3D = ("uh uhp uhpp up upp hu hup hupp agx arx vh vhp vhpp vp vpp hv hvp hvpp agy ary h hp hpp sal salp salpp "
            "rhop Av Dv wp Bth2 Bth3 Bth4").split()
STATE_2D = "s sp spp eagx earx eagy eary sx sy dd qq rr uair vair cdw".split()
STATE_I = ("k1z", "k1u", "k1v")


def _pair(run_dir, oracle_lib, steps, itmax=2000):
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(run_dir, ordering=1, pcg_itmax=itmax)
    if steps:
        o.run(steps)
    g = GpuRun(run_dir, pcg_itmax=itmax)
    for f in STATE_3D:
        g.set(f, o.get(f))
    for f in STATE_2D:
        g.set(f, o.get(f))
    for f in STATE_I:
        g.set(f, o.geti(f))
    return o, g


def _cmp(o, g, fields, rtol, label):
    worst = {}
    for f in fields:
        a = o.geti(f) if f in STATE_I else o.get(f)
        b = g.get(f)
        if f in STATE_I:
            np.testing.assert_array_equal(b, a, err_msg=f"{label}:{f}")
            continue
        scale = max(np.abs(a).max(), 1e-300)
        err = np.abs(a - b).max() / scale
        worst[f] = err
        assert err <= rtol, f"{label}: {f} rel err {err:.3e} > {rtol:.1e}"
    return worst


def test_initial_state_matches_oracle(run_dirs, oracle_lib, native_libs):
    from si3d_b200.model import GpuRun
    for name in ("t0", "t1", "c0"):
        o = oracle_lib.OracleRun(run_dirs[name])
        g = GpuRun(run_dirs[name])
        for f in ("h", "hp", "hpp", "hu", "hup", "hupp", "hv", "hvp", "hvpp", "sal", "salp", "salpp", "Av", "Dv"):
            np.testing.assert_array_equal(g.get(f), o.get(f), err_msg=f"{name}:{f}")
        # rhop is computed on the device from the same profile: bitwise as well
        np.testing.assert_array_equal(g.get("rhop")[1:, :], o.get("rhop")[1:, :], err_msg=f"{name}:rhop")
        for f in ("s", "sp", "spp"):
            np.testing.assert_array_equal(g.get(f)[:-1], o.get(f)[:-1], err_msg=f"{name}:{f}")
        for f in STATE_I:
            np.testing.assert_array_equal(g.get(f), o.geti(f), err_msg=f"{name}:{f}")


@pytest.mark.parametrize("istep", [1, 2])
def test_stage_by_stage(run_dirs, oracle_lib, native_libs, istep):
    o, g = _pair(run_dirs["t1"], oracle_lib, steps=3)
    seq = [("momentum", ["agx", "arx", "agy", "ary", "eagx", "earx", "eagy", "eary"], 1e-14),
           ("matcon", ["sx", "sy", "dd", "qq", "rr"], 1e-14),
           ("solve", ["s", "h", "hu", "hv"], 1e-11),
           ("vel", ["uh", "vh", "wp", "k1z", "k1u", "k1v"], 1e-9),
           ("scalar", ["sal", "Bth2", "Bth3", "Bth4"], 1e-9),
           ("vel2", ["h", "hu", "hv", "uh", "vh"], 1e-9)]
    for stage, fields, tol in seq:
        o.stage(stage, istep)
        g.stage(stage, istep)
        _cmp(o, g, fields, tol, f"{stage}/istep{istep}")
        # re-synchronise so that the next stage starts from identical inputs
        for f in STATE_3D:
            g.set(f, o.get(f))
        for f in STATE_2D:
            g.set(f, o.get(f))
        for f in STATE_I:
            g.set(f, o.geti(f))


@pytest.mark.parametrize("stage,istep", [("settrap", 2), ("settrap2", 2), ("save", 1), ("save", 2)])
def test_bookkeeping_stages_bitwise(run_dirs, oracle_lib, native_libs, stage, istep):
    o, g = _pair(run_dirs["t1"], oracle_lib, steps=2)
    o.stage(stage, istep)
    g.stage(stage, istep)
    _cmp(o, g, STATE_3D + ["s", "sp", "spp"] + list(STATE_I), 0.0, stage)


@pytest.mark.parametrize("name,steps", [("t0", 30), ("t1", 30), ("c0", 30)])
def test_time_steps_match_oracle(run_dirs, oracle_lib, native_libs, name, steps):
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(run_dirs[name], ordering=1, pcg_itmax=2000)
    g = GpuRun(run_dirs[name], pcg_itmax=2000)
    o.run(steps)
    st = g.run(steps)
    ds = np.abs(o.get("s") - g.get("s")).max()
    assert ds <= 1e-9, f"max |dzeta| {ds:.3e} m"
    for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("sal", 1e-10), ("wp", 1e-7), ("h", 1e-10)):
        a, b = o.get(f), g.get(f)
        err = np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)
        assert err <= tol, f"{name}:{f} rel err {err:.3e}"
    # same number of CG iterations per solve, up to +-2 from reduction-order rounding
    it_o = [s["iters"] for s in o.solves()]
    it_g = [s.iters[i] for s in st for i in range(s.nsolves)]
    assert len(it_o) == len(it_g)
    assert max(abs(a - b) for a, b in zip(it_o, it_g)) <= 2, (it_o[:12], it_g[:12])


def test_standalone_solve_matches_oracle(run_dirs, oracle_lib, native_libs):
    """si3d_gpu_solve_zeta on the Purdue arrays SolverSparse builds."""
    from si3d_b200.model import solve_zeta
    o = oracle_lib.OracleRun(run_dirs["t1"], ordering=1)
    o.run(2)
    o.stage("momentum", 2)
    o.stage("matcon", 2)
    lm, lm1 = o.lm, o.lm1
    lEC, lWC, lNC, lSC = (o.geti(n) for n in ("lEC", "lWC", "lNC", "lSC"))
    sx, sy, rr, qq, sp = (o.get(n) for n in ("sx", "sy", "rr", "qq", "sp"))
    coef = np.zeros((lm, 5))
    jco = np.zeros((lm, 5), dtype=np.int32)
    m = np.arange(lm)
    coef[:, 0] = rr[m]
    coef[:, 1] = -sx[lWC[m] - 1]
    coef[:, 2] = -sy[lSC[m] - 1]
    coef[:, 3] = -sy[m]
    coef[:, 4] = -sx[m]
    jco[:, 0] = m + 1
    for c, nb in ((1, lWC), (2, lSC), (3, lNC), (4, lEC)):
        jco[:, c] = np.where(nb[m] == lm1, 0, nb[m])
    x_o, r_o = oracle_lib.pcg(coef, jco, qq[:lm], sp[:lm], ordering=1, itmax=2000)
    x_g, r_g = solve_zeta(coef, jco, qq[:lm], sp[:lm], itmax=2000)
    assert r_g["ier"] == 0 and r_o["ier"] == 0
    assert abs(r_g["iters"] - r_o["iters"]) <= 2
    assert np.abs(x_g - x_o).max() <= 1e-11 * max(np.abs(x_o).max(), 1e-3)
    assert r_g["stptst"] < 1e-12


@pytest.mark.gpu
def test_stopping_test_2_standalone_matches_oracle(native_libs, oracle_lib):
    """Stopping test 2 (the reference's own setting, 1e-6) with chgcon's adaptive emin/emax on the
    device: same iteration count, eigenvalue estimates and solution as the oracle's red-black MIC-PCG."""
    from si3d_b200.model import solve_zeta
    g = np.load(os.path.join(ROOT, "tests", "golden", "pcg_48x32.npz"))
    x0 = np.zeros_like(g["rhs"])
    x_o, r_o = oracle_lib.pcg(g["coef"], g["jcoef"], g["rhs"], x0, pcg_test=2, tol=1e-6, itmax=500, ordering=1)
    x_g, r_g = solve_zeta(g["coef"], g["jcoef"], g["rhs"], x0, pcg_test=2, tol=1e-6, itmax=500)
    assert r_o["ier"] == 0 and r_g["ier"] == 0
    assert abs(r_g["iters"] - r_o["iters"]) <= 1
    assert r_g["emin"] == pytest.approx(r_o["emin"], rel=1e-6)
    assert r_g["emax"] == pytest.approx(r_o["emax"], rel=1e-6)
    assert np.abs(x_g - x_o).max() <= 1e-6 * np.abs(x_o).max()


@pytest.mark.gpu
def test_stopping_test_2_steps_match_oracle(native_libs, oracle_lib, run_dirs):
    """Whole time steps with stopping test 2 at 1e-6: per-solve iteration counts within one of the
    oracle's and the surface elevation within the solve tolerance's reach."""
    from si3d_b200.model import GpuRun
    steps = 5
    o = oracle_lib.OracleRun(run_dirs["t1"], pcg_test=2, pcg_tol=1e-6, pcg_itmax=200, ordering=1)
    o.run(steps)
    it_o = [s["iters"] for s in o.solves()]
    run = GpuRun(run_dirs["t1"], pcg_test=2, pcg_tol=1e-6, pcg_itmax=200)
    try:
        st = run.run(steps)
        it_g = [s.iters[i] for s in st for i in range(s.nsolves)]
        assert len(it_g) == len(it_o)
        assert max(abs(a - b) for a, b in zip(it_g, it_o)) <= 1
        s_o = o.get("s")[:o.lm]
        assert np.abs(run.get("s")[:run.lm] - s_o).max() <= 1e-6 * max(np.abs(s_o).max(), 1e-3)
    finally:
        run.close()


@pytest.mark.parametrize("x0", ["LAST", "HIST"])
@pytest.mark.parametrize("precision", ["FP64", "MIXED_IR", "MIXED_MG"])
def test_initial_guess_modes_match_oracle(run_dirs, oracle_lib, native_libs, x0, precision):
    """The initial guess changes where each CG solve starts, not the system it solves: 30 steps with
    x0 = the latest solution (LAST) or the latest solution plus the same solve's correction one step
    earlier (HIST) stay within the plain tolerances of the oracle's sp-started run."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(run_dirs["t1"], ordering=1, pcg_itmax=2000)
    g = GpuRun(run_dirs["t1"], pcg_itmax=2000, x0_mode=getattr(native, f"SI3D_X0_{x0}"),
               precision=getattr(native, f"SI3D_{precision}"))
    try:
        o.run(30)
        st = g.run(30)
        assert all(s.ier[i] == 0 for s in st for i in range(s.nsolves))
        assert max(s.relres[i] for s in st for i in range(s.nsolves)) < 1e-12
        ds = np.abs(o.get("s") - g.get("s")).max()
        assert ds <= 1e-9, f"max |dzeta| {ds:.3e} m"
        for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("sal", 1e-10)):
            a, b = o.get(f), g.get(f)
            err = np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)
            assert err <= tol, f"{x0}/{precision}:{f} rel err {err:.3e}"
    finally:
        g.close()


def test_column_tridiag_matches_oracle_trid(native_libs, oracle_lib):
    """si3d_gpu_column_tridiag (the batched trid, one factorisation and two right-hand sides per
    column) against the oracle's trid (si3d_procedures.f90:3210-3289) column by column, on
    diagonally dominant systems of the momentum solve's shape."""
    from si3d_b200.model import column_tridiag
    rng = np.random.default_rng(3210)
    n, nsys = 62, 3000
    a = -rng.uniform(0.0, 1.0, (n, nsys))
    c = -rng.uniform(0.0, 1.0, (n, nsys))
    b = 2.2 + rng.uniform(0.0, 1.0, (n, nsys))
    a[0] = 0.0
    c[-1] = 0.0
    g = rng.standard_normal((n, nsys))
    r = rng.standard_normal((n, nsys))
    ag, ar = column_tridiag(a, b, c, g, r)
    for s in range(0, nsys, 37):
        ag_o, ar_o = oracle_lib.trid(a[:, s], b[:, s], c[:, s], g[:, s], r[:, s])
        np.testing.assert_allclose(ag[:, s], ag_o, rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(ar[:, s], ar_o, rtol=1e-13, atol=1e-15)


def test_single_precision_field_copies(native_libs, run_dirs):
    """si3d_gpu_set_field_f32 / get_field_f32, the boundary for the reference as shipped (default
    REAL of 4 bytes): floats widen exactly on the way in and round to nearest on the way out, for
    3-D and 2-D fields alike."""
    import ctypes as C

    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    g = native.gpu()
    run = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    try:
        run.run(2)
        for name, shape in (("uh", (run.km1, run.lm1)), ("s", (run.lm1,))):
            ref = run.get(name)
            out = np.empty(shape, dtype=np.float32, order="F")
            assert g.si3d_gpu_get_field_f32(run.gh, name.encode(), C.c_void_p(out.ctypes.data)) == 0
            np.testing.assert_array_equal(out, ref.astype(np.float32))
            vals = np.asfortranarray((np.random.default_rng(7).standard_normal(shape)).astype(np.float32))
            assert g.si3d_gpu_set_field_f32(run.gh, name.encode(), C.c_void_p(vals.ctypes.data)) == 0
            np.testing.assert_array_equal(run.get(name), vals.astype(np.float64))
        assert g.si3d_gpu_set_field_f32(run.gh, b"nosuch", C.c_void_p(out.ctypes.data)) == -103
    finally:
        run.close()
