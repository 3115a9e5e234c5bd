"""Known-answer tests of the CPU oracle (the FP64 restatement of the reference's semi-implicit core).

The reference ships no tests, golden outputs or fixtures for this path, so the oracle is pinned by
published check values (the UNESCO equation of state), by exact linear algebra (tridiagonal and
5-point systems against dense solves), by invariants of the discrete equations (closed-basin
volume), by the steady wind set-up of shallow-water theory, and by the reference's own failure
semantics (NSPCG ier codes).  All of these run on the CPU.
"""
import dataclasses
import os

import numpy as np
import pytest

from si3d_b200 import synth


# ---------------------------------------------------------------------------- small linear algebra
def _tridiag_dense(a, b, c):
    n = len(b)
    A = np.diag(b)
    A[np.arange(1, n), np.arange(n - 1)] = a[1:]
    A[np.arange(n - 1), np.arange(1, n)] = c[:-1]
    return A


@pytest.mark.parametrize("n", [1, 2, 7, 60])
def test_trid_two_rhs_matches_dense(oracle_lib, n):
    """trid (si3d_procedures.f90:3210-3289): one factorisation, two right-hand sides."""
    rng = np.random.default_rng(n)
    a = -rng.uniform(0.1, 1.0, n)
    c = -rng.uniform(0.1, 1.0, n)
    b = 2.5 + rng.uniform(0.0, 1.0, n)
    g, r = rng.standard_normal(n), rng.standard_normal(n)
    ag, ar = oracle_lib.trid(a, b, c, g, r)
    A = _tridiag_dense(a, b, c)
    np.testing.assert_allclose(ag, np.linalg.solve(A, g), rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(ar, np.linalg.solve(A, r), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("n", [1, 3, 60])
def test_trid1_matches_dense(oracle_lib, n):
    """trid1 (si3d_procedures.f90:3292-3352), the scalar-transport solve."""
    rng = np.random.default_rng(100 + n)
    a = -rng.uniform(0.0, 1.0, n)
    c = -rng.uniform(0.0, 1.0, n)
    b = 2.1 + rng.uniform(0.0, 1.0, n)
    d = rng.standard_normal(n)
    x = oracle_lib.trid1(a, b, c, d)
    np.testing.assert_allclose(x, np.linalg.solve(_tridiag_dense(a, b, c), d), rtol=1e-12, atol=1e-13)


# ---------------------------------------------------------------------------- equation of state
def test_densty_pure_water_check_values(oracle_lib):
    """UNESCO (1981) check values of the one-atmosphere equation of state for pure water."""
    assert oracle_lib.densty(5.0, 0.0, 0.0) == pytest.approx(999.96675, abs=2e-5)
    assert oracle_lib.densty(25.0, 0.0, 0.0) == pytest.approx(997.04796, abs=2e-5)


def test_densty_keeps_the_integer_exponent(oracle_lib):
    """densty_s writes salinity**(3/2), which Fortran evaluates as salinity**1 (integer
    division, si3d_utils.f90:3902).  At S = 35, T = 5 the UNESCO check value 1027.67547 is shifted by
    exactly (S - S**1.5) times the C(T) coefficient of the S**1.5 term."""
    t, s = 5.0, 35.0
    c_t = -5.72466e-3 + 1.0227e-4 * t - 1.6546e-6 * t * t
    expect = 1027.67547 + (s - s ** 1.5) * c_t
    assert oracle_lib.densty(t, s, 0.0) == pytest.approx(expect, abs=2e-5)


def test_densty_increases_with_depth(oracle_lib):
    """The pressure fixed point (si3d_utils.f90:3909-3945) makes water denser with depth."""
    r = [oracle_lib.densty(10.0, 4e-5, z) for z in (0.5, 10.0, 100.0, 1000.0)]
    assert all(b > a for a, b in zip(r, r[1:]))
    assert r[-1] - r[0] == pytest.approx(4.6, rel=0.1)   # ~4.6 kg/m^3 per km near 10 C


# ---------------------------------------------------------------------------- the zeta system
def _five_point_system(nx, ny, seed, land=0.2):
    """A random wet mask and an SPD 5-point system in SolverSparse's Purdue form
    (si3d_procedures.f90:1950-1967): row l = [rr, -sx_W, -sy_S, -sy, -sx] with
    rr = 1 + sx + sx_W + sy + sy_S, jcoef = [l, lW, lS, lN, lE] (0 = no neighbour)."""
    rng = np.random.default_rng(seed)
    wet = rng.uniform(size=(nx, ny)) > land
    idx = -np.ones((nx, ny), dtype=np.int64)
    cells = [(i, j) for i in range(nx) for j in range(ny) if wet[i, j]]   # l order: i outer, j inner
    for l, (i, j) in enumerate(cells):
        idx[i, j] = l
    n = len(cells)
    sx = rng.uniform(0.5, 50.0, size=(nx, ny))
    sy = rng.uniform(0.5, 50.0, size=(nx, ny))
    coef = np.zeros((n, 5))
    jcoef = np.zeros((n, 5), dtype=np.int32)
    A = np.zeros((n, n))

    def nb(i, j):
        return idx[i, j] if 0 <= i < nx and 0 <= j < ny and wet[i, j] else -1

    for l, (i, j) in enumerate(cells):
        W, S, N, E = nb(i - 1, j), nb(i, j - 1), nb(i, j + 1), nb(i + 1, j)
        sxE = sx[i, j] if E >= 0 else 0.0
        syN = sy[i, j] if N >= 0 else 0.0
        sxW = sx[i - 1, j] if W >= 0 else 0.0
        syS = sy[i, j - 1] if S >= 0 else 0.0
        rr = 1.0 + sxE + sxW + syN + syS
        coef[l] = [rr, -sxW, -syS, -syN, -sxE]
        jcoef[l] = [l + 1, W + 1, S + 1, N + 1, E + 1]
        A[l, l] = rr
        for m, v in ((W, -sxW), (S, -syS), (N, -syN), (E, -sxE)):
            if m >= 0:
                A[l, m] = v
    return coef, jcoef, A


@pytest.mark.parametrize("ordering", [0, 1])
def test_pcg_manufactured_solution(oracle_lib, ordering):
    """MIC-PCG (nspcg mic1 + cg) on A x* = b recovers x* at test 5, 1e-12, in natural and
    red-black ordering."""
    coef, jcoef, A = _five_point_system(30, 20, seed=7)
    n = A.shape[0]
    assert np.allclose(A, A.T)
    rng = np.random.default_rng(8)
    xs = rng.standard_normal(n)
    b = A @ xs
    x, info = oracle_lib.pcg(coef, jcoef, b, np.zeros(n), pcg_test=5, tol=1e-12, itmax=500, ordering=ordering)
    assert info["ier"] == 0
    assert info["stptst"] < 1e-12
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-12
    np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=0, atol=1e-9 * np.abs(xs).max())
    assert 0 < info["iters"] < 200


def test_pcg_orderings_agree(oracle_lib):
    """Both orderings solve the same system to the same solution (to the tolerance)."""
    coef, jcoef, A = _five_point_system(40, 25, seed=11)
    b = A @ np.random.default_rng(12).standard_normal(A.shape[0])
    x0, _ = oracle_lib.pcg(coef, jcoef, b, np.zeros_like(b), ordering=0)
    x1, _ = oracle_lib.pcg(coef, jcoef, b, np.zeros_like(b), ordering=1)
    assert np.abs(x0 - x1).max() < 1e-10 * np.abs(x0).max()


def test_pcg_stopping_test_2(oracle_lib):
    """Stopping test 2 (pstops, nspcg.f:26034) with the adaptive eigenvalue estimate converges
    at the reference's own default tolerance."""
    coef, jcoef, A = _five_point_system(20, 20, seed=3)
    b = A @ np.ones(A.shape[0])
    x, info = oracle_lib.pcg(coef, jcoef, b, np.zeros_like(b), pcg_test=2, tol=1e-6, itmax=200, ordering=0)
    assert info["ier"] == 0
    assert np.abs(x - 1.0).max() < 1e-4
    assert 0.0 < info["emin"] <= info["emax"]


def test_pcg_itmax_reached(oracle_lib):
    """itcg returns ier = 1 when itmax is reached (nspcg.f:9052-9055)."""
    coef, jcoef, A = _five_point_system(30, 20, seed=5)
    b = A @ np.random.default_rng(6).standard_normal(A.shape[0])
    _, info = oracle_lib.pcg(coef, jcoef, b, np.zeros_like(b), itmax=2)
    assert info["ier"] == 1
    assert info["iters"] == 2


def test_pcg_zero_rhs_is_an_error(oracle_lib):
    """With r = 0 exactly, (r, z) = 0 and itcg stops with ier = -7 (nspcg.f:9042-9045): NSPCG
    treats a zero right-hand side with a zero initial guess as a breakdown."""
    coef, jcoef, A = _five_point_system(10, 10, seed=1)
    n = A.shape[0]
    _, info = oracle_lib.pcg(coef, jcoef, np.zeros(n), np.zeros(n))
    assert info["ier"] == -7


def test_pcg_indefinite_is_an_error(oracle_lib):
    """A negative-definite system cannot pass CG: (r, z) or (p, Ap) turns non-positive."""
    coef, jcoef, A = _five_point_system(10, 10, seed=2)
    n = A.shape[0]
    b = np.ones(n)
    _, info = oracle_lib.pcg(-coef, jcoef, b, np.zeros(n))
    assert info["ier"] < 0


# ---------------------------------------------------------------------------- whole time steps
def _run(tmp_path, basin, name):
    d = str(tmp_path / name)
    synth.write_run(basin, d)
    return d


def test_quiescent_lake_without_baroclinic_term_stops_the_solver(oracle_lib, tmp_path):
    """Uniform temperature, no wind and ibc = 0: every right-hand side of the zeta system is zero,
    so NSPCG reports ier = -7 and si3d stops with 'fatal error in matrix solution'
    (si3d_procedures.f90:2005-2016).  The oracle keeps that behaviour."""
    b = dataclasses.replace(synth.config("t0", nsteps=5), wa=0.0, t_top=15.0, t_bottom=15.0, ibc=0)
    o = oracle_lib.OracleRun(_run(tmp_path, b, "rest"))
    with pytest.raises(RuntimeError, match="matrix solution"):
        o.run(2)


def test_lake_at_rest_stays_near_rest(oracle_lib, tmp_path):
    """No wind, uniform temperature, baroclinic term on: only the compressibility of densty_s
    between neighbouring partial bottom cells drives motion, and it stays below a micrometre."""
    b = dataclasses.replace(synth.config("c0", nsteps=30), wa=0.0, t_top=15.0, t_bottom=15.0)
    o = oracle_lib.OracleRun(_run(tmp_path, b, "rest1"))
    o.run(10)
    assert np.abs(o.get("s")).max() < 1e-6
    assert np.abs(o.get("uh")).max() < 1e-4
    sal = o.get("sal")[1:, :o.lm]
    assert np.abs(sal - 15.0).max() < 1e-12


def test_closed_basin_volume_is_conserved(oracle_lib, tmp_path):
    """sum(s) dx dy over the wet columns (the volume si3d.f90:400-410 reports) is invariant in a
    closed basin, to round-off, under wind forcing and stratification."""
    b = synth.config("c0", nsteps=100)
    o = oracle_lib.OracleRun(_run(tmp_path, b, "vol"))
    s0 = o.get("s")[:o.lm].sum()
    for _ in range(4):
        o.run(10)
        s = o.get("s")[:o.lm]
        assert np.abs(s).max() > 1e-3                       # the surface does move
        assert abs(s.sum() - s0) < 1e-13 * o.lm * max(np.abs(s).max(), 1.0)


def test_wind_setup(oracle_lib, tmp_path):
    """A steady eastward stress tau tilts the surface up downwind with slope tau / (rho g H):
    averaged over the seiche that the spin-up excites, the east-west set-up of the c0 bowl
    (mean depth 10 m) is within a factor 2 of the steady shallow-water value."""
    b = synth.config("c0", nsteps=200)
    o = oracle_lib.OracleRun(_run(tmp_path, b, "setup"))
    l2i = o.geti("l2i")[:o.lm]
    east, west = l2i > 70, l2i < 30
    hhs = o.get("hhs")[:o.lm]
    diffs = []
    for _ in range(12):
        o.run(10)
        s = o.get("s")[:o.lm]
        diffs.append(s[east].mean() - s[west].mean())
    tau, rho, g = 0.1, 1000.0, 9.806
    dx = b.dx
    separation = (l2i[east].mean() - l2i[west].mean()) * dx
    steady = tau * separation / (rho * g * hhs.mean())
    mean = float(np.mean(diffs))
    assert mean > 0
    assert 0.5 * steady < mean < 2.0 * steady
