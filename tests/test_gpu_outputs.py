"""Output writers on the GPU path: frames packed on the device (si3d_gpu_output_frame) against the
oracle's state rounded to 4-byte floats, bit for bit, and whole output files written by the host
against the files the oracle writes for the same run."""
import ctypes as C
import os
import shutil

import numpy as np
import pytest

from test_gpu_parity import STATE_2D, STATE_3D, STATE_I
from test_outputs_oracle import OUT, frame, read_records

pytestmark = pytest.mark.gpu


def _frame(g, kind, arg, first):
    from si3d_b200 import native
    lib = native.gpu()
    cnt = C.c_longlong(0)
    native.check(lib.si3d_gpu_output_frame(g.gh, kind, arg, first, None, 0, C.byref(cnt)))
    out = np.empty(cnt.value, dtype=np.float32)
    native.check(lib.si3d_gpu_output_frame(g.gh, kind, arg, first, native.ptr(out), cnt.value, C.byref(cnt)))
    return out


def test_device_frames_are_the_rounded_state(tracer_dirs, oracle_lib, native_libs):
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    o = oracle_lib.OracleRun(tracer_dirs["t1"], ordering=1, pcg_itmax=2000)
    o.run(3)
    g = GpuRun(tracer_dirs["t1"], pcg_itmax=2000)
    try:
        tr = [f"tracer{t}" for t in (1, 2, 3)]
        for f in STATE_3D + tr + [f"tracerpp{t}" for t in (1, 2, 3)]:
            g.set(f, o.get(f))
        for f in STATE_2D:
            g.set(f, o.get(f))
        for f in STATE_I:
            g.set(f, o.geti(f))
        kmz = o.geti("kmz")[:o.lm]
        cols = np.repeat(np.arange(o.lm), kmz)
        ks = np.concatenate([np.arange(2, k + 2) for k in kmz])
        l2i, l2j = o.geti("l2i")[:o.lm], o.geti("l2j")[:o.lm]
        pts = lambda f: o.get(f)[:, :o.lm][ks - 1, cols].astype(np.float32)
        v = _frame(g, native.SI3D_OUT_PTRACK, 0, 0).reshape(-1, 5)
        for j, f in enumerate(("hp", "up", "vp", "wp", "salp")):
            np.testing.assert_array_equal(v[:, j], pts(f), err_msg=f)
        v = _frame(g, native.SI3D_OUT_PTRACK, 0, 1).reshape(-1, 8)
        np.testing.assert_array_equal(v[:, 0], l2i[cols].astype(np.float32))
        np.testing.assert_array_equal(v[:, 1], l2j[cols].astype(np.float32))
        np.testing.assert_array_equal(v[:, 2], ks.astype(np.float32))
        np.testing.assert_array_equal(v[:, 7], pts("salp"))
        v = _frame(g, native.SI3D_OUT_TRACER, 2, 0)
        np.testing.assert_array_equal(v, pts("tracer2"))
        km = o.km
        up, vp, wp, Av, hp, sal = (o.get(f) for f in ("up", "vp", "wp", "Av", "hp", "salp"))
        s = o.get("s")
        lw, ls = o.geti("lWC")[:o.lm] - 1, o.geti("lSC")[:o.lm] - 1
        for kp in (2, 5, km + 1):
            sel = np.arange(o.lm) if kp > km else np.nonzero(kmz >= kp)[0]
            kb = (kmz[sel] if kp > km else np.full(len(sel), kp)) - 1
            v = _frame(g, native.SI3D_OUT_PLANE, kp, 0).reshape(-1, 6)
            np.testing.assert_array_equal(v[:, 0], ((up[kb, sel] + up[kb, lw[sel]]) / 2.).astype(np.float32))
            np.testing.assert_array_equal(v[:, 1], ((vp[kb, sel] + vp[kb, ls[sel]]) / 2.).astype(np.float32))
            np.testing.assert_array_equal(v[:, 2], ((wp[kb, sel] + wp[kb + 1, sel]) / 2.).astype(np.float32))
            np.testing.assert_array_equal(v[:, 3], np.where(hp[kb, sel] <= 0, -99., sal[kb, sel]).astype(np.float32))
            np.testing.assert_array_equal(v[:, 4], (0.5 * (Av[kb, sel] + Av[kb + 1, sel])).astype(np.float32))
            np.testing.assert_array_equal(v[:, 5], s[sel].astype(np.float32))
        with pytest.raises(native.Si3dError):
            _frame(g, native.SI3D_OUT_PLANE, 1, 0)
        with pytest.raises(native.Si3dError):
            _frame(g, native.SI3D_OUT_TRACER, 4, 0)
    finally:
        g.close()


def test_output_files_match_the_oracle(tmp_path, oracle_lib, native_libs):
    """t0 with two tracers, six steps: planes every 2 steps, tracers every 3, ptrack every step.
    Record layout, headers and time stamps are identical; the initial frames are bit-identical (the
    same initial state); later frames agree to the float rounding of states that agree to 1e-9."""
    from si3d_b200 import synth
    from si3d_b200.model import GpuRun
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "oracle")
    synth.make("t0", dg, ntr=2, outputs=OUT)
    shutil.copytree(dg, do)
    g = GpuRun(dg, pcg_itmax=2000)
    try:
        g.run(6)
    finally:
        g.close()
    o = oracle_lib.OracleRun(do, ordering=1, pcg_itmax=2000)
    o.run(6)
    o.close()
    names = ["si3d_3D", "tracer_1", "tracer_2"] + [f"plane_{k}" for k in OUT["planes"]]
    for name in names:
        rg, ro = read_records(os.path.join(dg, name)), read_records(os.path.join(do, name))
        assert [len(r) for r in rg] == [len(r) for r in ro], name
        assert rg[0] == ro[0] and rg[1] == ro[1], name
        assert rg[2] == ro[2], f"{name}: initial frame"
        for a, b in zip(rg[3:], ro[3:]):
            assert a[:20] == b[:20], f"{name}: time stamp"
            x, y = np.frombuffer(a[20:], dtype="<f4"), np.frombuffer(b[20:], dtype="<f4")
            np.testing.assert_allclose(x, y, rtol=1e-6, atol=1e-7 * max(np.abs(y).max(), 1e-30), err_msg=name)


def test_space_xml_matches_oracle(native_libs, oracle_lib, tmp_path):
    """The host's outs (ipxml < 0) writes the same XML header as the oracle's, line for line except
    runNumber (the wall-clock date), and the same two empty binary space files."""
    import os

    from si3d_b200 import synth
    from si3d_b200.model import GpuRun
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "orc")
    for d in (dg, do):
        synth.make("t1", d, outputs={"ipxml": -1, "itspf": 0})
    g = GpuRun(dg, pcg_itmax=2000)
    try:
        g.run(3)
    finally:
        g.close()
    o = oracle_lib.OracleRun(do, ordering=1, pcg_itmax=2000)
    o.run(3)
    a = open(os.path.join(dg, "spacefile.xml")).read().split("\n")
    b = open(os.path.join(do, "spacefile.xml")).read().split("\n")
    assert len(a) == len(b)
    for x, y in zip(a, b):
        if "runNumber=" in y:
            assert x.startswith('        runNumber="') and len(x) == len(y)
        else:
            assert x == y
    for f in ("spacefile2d.bin", "spacefile3d.bin"):
        assert os.path.getsize(os.path.join(dg, f)) == 0
