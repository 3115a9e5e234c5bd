"""Known answers for the oracle's Mellor-Yamada 2.5 closure (iturb = 1, si3d_mixing.f90:33-889).
The reference ships no turbulence test data, so the restatement is pinned by what the scheme
imposes: the boundary rows of the q2 system are Dirichlet conditions q2 = B1^(2/3) u*^2 at the
surface (wind stress) and the bottom (drag), q2l is held at its floor there, the stability
functions at neutral stratification reduce to Sh = A2 (1 - 6 A1 / B1) and Sm = B1^(-1/3), every
eddy coefficient inside a column is at least the molecular value, and the closure leaves a basin
at rest quiet."""
import numpy as np
import pytest

B1, A1, A2 = 16.6, 0.92, 0.74


def _prepared(o):
    o.run(3)
    for st in ("momentum", "matcon", "solve", "vel", "scalar", "vel2"):
        o.stage(st, 2)


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_boundary_rows_are_the_friction_velocities(turb_dirs, oracle_lib, name):
    o = oracle_lib.OracleRun(turb_dirs[name], ordering=1, pcg_itmax=2000)
    _prepared(o)
    o.stage("turbulence", 2)
    lm = o.lm
    kmz, k1z = o.geti("kmz")[:lm], o.geti("k1z")[:lm]
    k1u, k1v = o.geti("k1u"), o.geti("k1v")   # lm1 entries: neighbours may be the dry column
    lW, lS = o.geti("lWC")[:lm] - 1, o.geti("lSC")[:lm] - 1
    up, vp, u, v, q2, q2l = (o.get(n) for n in ("up", "vp", "u", "v", "q2", "q2l"))
    uair, vair, cdw = o.get("uair"), o.get("vair"), o.get("cdw")
    wet = np.nonzero(kmz - k1z + 1 > 1)[0]
    c = np.arange(lm)
    usurf = 0.5 * (up[k1u[c] - 1, c] + up[k1u[lW] - 1, lW])
    vsurf = 0.5 * (vp[k1v[c] - 1, c] + vp[k1v[lS] - 1, lS])
    us2 = cdw[:lm] * 1.3 * ((uair[:lm] - usurf) ** 2 + (vair[:lm] - vsurf) ** 2) / 1000.
    ub2 = 0.0025 * ((0.5 * (u[kmz - 1, c] + u[kmz - 1, lW])) ** 2 + (0.5 * (v[kmz - 1, c] + v[kmz - 1, lS])) ** 2)
    top = q2[k1z - 1, c]
    bot = q2[kmz, c]
    np.testing.assert_allclose(top[wet], np.maximum(2e-6, B1 ** (2 / 3) * us2[wet]), rtol=1e-13)
    np.testing.assert_allclose(bot[wet], np.maximum(2e-6, B1 ** (2 / 3) * ub2[wet]), rtol=1e-13)
    assert np.all(q2l[k1z - 1, c][wet] == 6.80236723501e-9) and np.all(q2l[kmz, c][wet] == 6.80236723501e-9)


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_eddy_coefficients_and_bounds(turb_dirs, oracle_lib, name):
    o = oracle_lib.OracleRun(turb_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(10)
    lm = o.lm
    kmz, k1z = o.geti("kmz")[:lm], o.geti("k1z")[:lm]
    Av, Dv, q2, q2l = (o.get(n)[:, :lm] for n in ("Av", "Dv", "q2", "q2l"))
    K = np.arange(1, o.km1 + 1)[:, None]
    inner = (K > k1z[None, :]) & (K <= kmz[None, :]) & ((kmz - k1z + 1) > 1)[None, :]
    assert np.all(Av[inner] >= 1.3e-6) and np.all(Dv[inner] >= 1.4e-7)
    assert np.all(Av[~inner & (K != k1z[None, :] + 1)] == 0.0)
    assert np.all(q2[inner] >= 2e-6) and np.all(q2l[inner] >= 6.80236723501e-9)
    assert np.isfinite(q2).all() and np.isfinite(Av).all()


def test_neutral_stability_functions():
    """With N2 = 0 (Gh = 0) the Kantha-Clayson quasi-equilibrium functions are t1 and t3."""
    t1 = A2 * (1. - 6. * A1 / B1)
    t3 = B1 ** (-1. / 3.)
    Gh = 0.0
    Sh = t1 / (1. - Gh * 3. * A2 * (6. * A1 + 10.1 * (1. - 0.2)))
    Sm = (t3 + Sh * Gh * 9. * A1 * (2. * A1 + A2 * (1. - 0.7))) / (1. - 9. * A1 * A2 * Gh)
    assert Sh == t1 and Sm == t3 and abs(Sm - 0.39199) < 1e-4 and abs(Sh - 0.49393) < 1e-4


def test_host_reads_the_closure(turb_dirs, native_libs):
    import ctypes as C
    h = native_libs.host()
    hm = C.c_int(-1)
    err = C.create_string_buffer(256)
    assert h.si3d_host_open(turb_dirs["t0"].encode(), None, C.byref(hm), err, 256) == 0, err.value
    h.si3d_host_close(hm.value)


def test_closure_keeps_a_lake_at_rest_quiet(tmp_path, oracle_lib):
    """No wind, uniform temperature: the friction velocities vanish, so both boundary rows sit at
    q2_min; the flow stays below a micrometre per second as without the closure, q2 never rises
    above its initial maximum, and the closure keeps every eddy coefficient finite."""
    import dataclasses
    from si3d_b200 import synth
    b = dataclasses.replace(synth.config("c0", nsteps=30), wa=0.0, t_top=15.0, t_bottom=15.0, iturb=1)
    d = str(tmp_path / "rest_turb")
    synth.write_run(b, d)
    o = oracle_lib.OracleRun(d, ordering=1, pcg_itmax=2000)
    q0 = o.get("q2").max()
    o.run(10)
    assert np.abs(o.get("s")).max() < 1e-6
    assert np.abs(o.get("uh")).max() < 1e-4
    q2 = o.get("q2")[:, :o.lm]
    assert q2.max() <= q0 * (1 + 1e-12)
    k1z, kmz = o.geti("k1z")[:o.lm], o.geti("kmz")[:o.lm]
    c = np.arange(o.lm)
    assert np.all(q2[k1z - 1, c] == 2e-6)
    assert np.isfinite(o.get("Av")).all() and np.isfinite(o.get("Dv")).all()
