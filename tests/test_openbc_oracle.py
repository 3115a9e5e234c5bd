"""Open boundaries with a specified water-surface elevation (itype 1) in the oracle restatement
(oracle/oracle_obc.cpp), pinned by what such a boundary imposes: the reference ships no open-boundary
data for this path.

* after every time step the boundary cells carry the series value at that time, interpolated
  parabolically as parab does (si3d_utils.f90:895-920);
* a boundary held at the basin's own level, with no wind, leaves a lake at rest at rest;
* a boundary held 2 cm above the basin fills it: the interior level oscillates about the boundary's.
"""
import dataclasses
import math

import numpy as np
import pytest

from si3d_b200 import synth


def _parab(x, fx, dx):
    m = int(x / dx)
    theta = (x - m * dx) / dx
    if m == 0:
        m, theta = 2, theta - 1.0
    else:
        m = m + 1
    f = lambda i: fx[i - 1]  # noqa: E731
    return f(m) + 0.5 * theta * (f(m + 1) - f(m - 1) + theta * (f(m + 1) + f(m - 1) - 2.0 * f(m)))


def _boundary_cells(b, o):
    l2i, l2j = o.geti("l2i")[:o.lm], o.geti("l2j")[:o.lm]
    ij = {(int(i), int(j)): l for l, (i, j) in enumerate(zip(l2i, l2j))}
    out = []
    for (side, isbc, jsbc, iebc, jebc) in b.obc:
        cells = [(isbc, j) for j in range(jsbc, jebc + 1)] if side in (1, 3) else [(i, jsbc) for i in range(isbc, iebc + 1)]
        out.append([ij[c] for c in cells])
    return out


@pytest.mark.parametrize("name", ["t2", "t3"])
def test_boundary_cells_follow_the_series(oracle_lib, tmp_path, name):
    d = str(tmp_path / name)
    b = synth.make(name, d)
    o = oracle_lib.OracleRun(d, ordering=0, pcg_itmax=2000)
    cells = _boundary_cells(b, o)
    for n in range(1, 13):
        o.run(1)
        s = o.get("s")
        for q, ls in enumerate(cells):
            want = _parab(n * b.dt / 3600.0, b.obc_wse[q], b.obc_dtsec / 3600.0)
            np.testing.assert_allclose(s[ls], want, rtol=0, atol=1e-15)
    assert all(x["ier"] == 0 for x in o.solves())


def _flat(tmp_path, name, level):
    b = synth.config("t2")
    b.name = name
    b.wa = 0.0
    b.t_top = b.t_bottom = 15.0
    b.obc_wse = (tuple([level] * 40),)
    b.obc_temp = (tuple([15.0] * 40),)
    d = str(tmp_path / name)
    synth.write_run(b, d)
    return b, d


def test_lake_at_rest_stays_at_rest(oracle_lib, tmp_path):
    b, d = _flat(tmp_path, "rest", 0.0)
    o = oracle_lib.OracleRun(d, ordering=0, pcg_itmax=2000)
    o.run(20)
    assert np.abs(o.get("s")[:o.lm]).max() < 1e-9
    assert np.abs(o.get("uh")).max() < 1e-9


def test_raised_boundary_fills_the_basin(oracle_lib, tmp_path):
    b, d = _flat(tmp_path, "fill", 0.02)
    o = oracle_lib.OracleRun(d, ordering=0, pcg_itmax=2000)
    cells = set(_boundary_cells(b, o)[0])
    interior = np.array([l for l in range(o.lm) if l not in cells])
    means = []
    for _ in range(12):
        o.run(20)
        means.append(o.get("s")[interior].mean())
    # the interior level seiches about the boundary's 2 cm: its time average sits there
    assert 0.015 < float(np.mean(means)) < 0.025, means


def test_host_reads_and_refuses(native_libs, tmp_path):
    """The C++ host reads the open-boundary records and series, and refuses what is not built: flow
    boundaries (itype 2) and tracers with open boundaries."""
    import ctypes as C
    from si3d_b200 import native
    h = native.host()
    d = str(tmp_path / "ok")
    synth.make("t3", d)
    hm = C.c_int(-1)
    err = C.create_string_buffer(256)
    assert h.si3d_host_open(d.encode(), None, C.byref(hm), err, 256) == 0, err.value
    h.si3d_host_close(hm.value)
    bad = str(tmp_path / "flow")
    synth.make("t2", bad)
    txt = open(bad + "/si3d_inp.txt").read().replace(" itype       !                  1 !", " itype       !                  2 !")
    open(bad + "/si3d_inp.txt", "w").write(txt)
    assert h.si3d_host_open(bad.encode(), None, C.byref(hm), err, 256) == -101
    assert b"itype" in err.value
    tr = str(tmp_path / "tr")
    synth.make("t2", tr, ntr=2)
    assert h.si3d_host_open(tr.encode(), None, C.byref(hm), err, 256) == -101
