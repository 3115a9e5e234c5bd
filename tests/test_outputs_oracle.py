"""The oracle's restatement of the reference's binary writers (outp, outz, outh: si3d_utils.f90:
2142-2602) and of its calendar (compute_date, :3546-3674), checked on CPU: Fortran unformatted
record framing, header records, frame counts, coordinates, time stamps, and frame values equal to
the oracle's state rounded to 4-byte floats."""
import os
import struct

import numpy as np
import pytest

OUT = dict(iop=2, itspfh=0, planes=(2, 4, 99), ipxml=1, itspf=0, iotr=3, itspftr=0)


def read_records(path):
    """Fortran unformatted sequential records: 4-byte length, payload, the same length."""
    recs = []
    with open(path, "rb") as fh:
        data = fh.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        payload = data[i + 4:i + 4 + n]
        (n2,) = struct.unpack_from("<i", data, i + 4 + n)
        assert n == n2, "record markers differ"
        recs.append(payload)
        i += 8 + n
    return recs


def frame(rec, nv):
    n, yr, mo, dy = struct.unpack_from("<4i", rec, 0)
    (hr,) = struct.unpack_from("<f", rec, 16)
    vals = np.frombuffer(rec[20:], dtype="<f4").reshape(-1, nv)
    return (n, yr, mo, dy, hr), vals


@pytest.fixture(scope="module")
def out_run(tmp_path_factory):
    from si3d_b200 import synth
    d = str(tmp_path_factory.mktemp("outputs") / "t0")
    synth.make("t0", d, ntr=2, outputs=OUT)
    return d


def test_ptrack_file(out_run, oracle_lib):
    o = oracle_lib.OracleRun(out_run, ordering=1, pcg_itmax=2000)
    kmz = o.geti("kmz")[:o.lm]
    pts = int((kmz + 2 - 2).sum())
    # the initial frame is written when the run is opened
    recs = read_records(os.path.join(out_run, "si3d_3D"))
    assert struct.unpack("<i", recs[0])[0] == (o.nts - 0) // 1
    assert struct.unpack("<i", recs[1])[0] == pts
    (n, yr, mo, dy, hr), v = frame(recs[2], 8)
    assert (n, yr, mo, dy, hr) == (0, 2024, 1, 1, 0.0)
    l2i, l2j = o.geti("l2i")[:o.lm], o.geti("l2j")[:o.lm]
    cols = np.repeat(np.arange(o.lm), kmz)   # k1 .. kmz + 1: kmz points per column (k1 = 2)
    ks = np.concatenate([np.arange(2, k + 2) for k in kmz])
    np.testing.assert_array_equal(v[:, 0], l2i[cols].astype(np.float32))
    np.testing.assert_array_equal(v[:, 1], l2j[cols].astype(np.float32))
    np.testing.assert_array_equal(v[:, 2], ks.astype(np.float32))
    o.run(3)
    recs = read_records(os.path.join(out_run, "si3d_3D"))
    assert len(recs) == 2 + 4
    (n, yr, mo, dy, hr), v = frame(recs[-1], 5)
    assert n == 3 and (yr, mo, dy) == (2024, 1, 1)
    assert hr == np.float32(round(3 * 60 / 3600 * 100))   # ihr = NINT(hours * 100); t0 has dt = 60 s
    for j, f in enumerate(("hp", "up", "vp", "wp", "salp")):
        a = o.get(f)[:, :o.lm]
        np.testing.assert_array_equal(v[:, j], a[ks - 1, cols].astype(np.float32), err_msg=f)


def test_tracer_and_plane_files(out_run, oracle_lib):
    o = oracle_lib.OracleRun(out_run, ordering=1, pcg_itmax=2000)
    o.run(6)
    kmz = o.geti("kmz")[:o.lm]
    cols = np.repeat(np.arange(o.lm), kmz)
    ks = np.concatenate([np.arange(2, k + 2) for k in kmz])
    for t in (1, 2):
        recs = read_records(os.path.join(out_run, f"tracer_{t}"))
        assert len(recs) == 2 + 1 + 2   # header, n = 0, steps 3 and 6
        assert [frame(r, 1)[0][0] for r in recs[2:3]] == [0]
        _, v = frame(recs[-1], 1)
        np.testing.assert_array_equal(v[:, 0], o.get(f"tracer{t}")[:, :o.lm][ks - 1, cols].astype(np.float32))
    km = o.km
    for kp in OUT["planes"]:
        recs = read_records(os.path.join(out_run, f"plane_{kp}"))
        sel = np.arange(o.lm) if kp > km else np.nonzero(kmz >= kp)[0]
        assert struct.unpack("<i", recs[1])[0] == len(sel)
        assert len(recs) == 2 + 1 + 3   # n = 0, 2, 4, 6
        (n, *_), v = frame(recs[-1], 6)
        assert n == 6
        kb = kmz[sel] if kp > km else np.full(len(sel), kp)
        s = o.get("s")[:o.lm]
        np.testing.assert_array_equal(v[:, 5], s[sel].astype(np.float32))
        up, wp = o.get("up"), o.get("wp")
        lw = o.geti("lWC")[:o.lm][sel] - 1
        np.testing.assert_array_equal(v[:, 0], ((up[kb - 1, sel] + up[kb - 1, lw]) / 2.).astype(np.float32))
        np.testing.assert_array_equal(v[:, 2], ((wp[kb - 1, sel] + wp[kb, sel]) / 2.).astype(np.float32))


def test_calendar_rolls_over_days_and_months(tmp_path, oracle_lib):
    """A run that starts on 31 January at 23.98 h with 60 s steps crosses into February at its
    second step (the hour stamp is NINT(decimal hours * 100))."""
    from si3d_b200 import synth
    d = str(tmp_path / "cal")
    synth.make("t0", d, outputs=dict(ipxml=1))
    p = os.path.join(d, "si3d_inp.txt")
    lines = open(p).read().splitlines()
    for lab, val in (("day", 31), ("hour", 2398)):
        i = next(i for i, ln in enumerate(lines) if ln.startswith(f" {lab:<12}!"))
        lines[i] = synth._rec(lab, val)
    open(p, "w").write("\n".join(lines) + "\n")
    o = oracle_lib.OracleRun(d, ordering=1, pcg_itmax=2000)
    o.run(3)
    stamps = [frame(r, 5 if k else 8)[0] for k, r in enumerate(read_records(os.path.join(d, "si3d_3D"))[2:])]
    assert [s[1:] for s in stamps] == [(2024, 1, 31, 2398.0), (2024, 1, 31, 2400.0), (2024, 2, 1, 1.0),
                                       (2024, 2, 1, 3.0)]


def test_calendar_rolls_over_the_year(tmp_path, oracle_lib):
    """31 December 23.98 h with 60 s steps: the second step is 1 January of the next year."""
    from si3d_b200 import synth
    d = str(tmp_path / "year")
    synth.make("t0", d, outputs=dict(ipxml=1))
    p = os.path.join(d, "si3d_inp.txt")
    lines = open(p).read().splitlines()
    for lab, val in (("month", 12), ("day", 31), ("hour", 2398)):
        i = next(i for i, ln in enumerate(lines) if ln.startswith(f" {lab:<12}!"))
        lines[i] = synth._rec(lab, val)
    open(p, "w").write("\n".join(lines) + "\n")
    o = oracle_lib.OracleRun(d, ordering=1, pcg_itmax=2000)
    o.run(2)
    stamps = [frame(r, 5 if k else 8)[0][1:] for k, r in enumerate(read_records(os.path.join(d, "si3d_3D"))[2:])]
    assert stamps == [(2024, 12, 31, 2398.0), (2024, 12, 31, 2400.0), (2025, 1, 1, 1.0)]


def test_later_first_frame_and_interval(tmp_path, oracle_lib):
    """ptrack frames every 2 steps from step 4 (itspf = 4), after the initial frame; the header's
    frame count is (nts - itspf) / ipxml."""
    from si3d_b200 import synth
    d = str(tmp_path / "later")
    synth.make("t0", d, outputs=dict(ipxml=2, itspf=4))
    o = oracle_lib.OracleRun(d, ordering=1, pcg_itmax=2000)
    o.run(7)
    recs = read_records(os.path.join(d, "si3d_3D"))
    assert struct.unpack("<i", recs[0])[0] == (o.nts - 4) // 2
    assert [frame(r, 5 if k else 8)[0][0] for k, r in enumerate(recs[2:])] == [0, 4, 6]


def test_turbulence_variables_in_ptrack_output_are_refused(tmp_path, oracle_lib, native_libs):
    """iTurbVars = 1 asks outp for the turbulence fields, which only a closure provides."""
    import ctypes as C
    from si3d_b200 import synth
    d = str(tmp_path / "tv")
    synth.make("t0", d, outputs=dict(ipxml=1))
    p = os.path.join(d, "si3d_inp.txt")
    lines = open(p).read().splitlines()
    i = lines.index(synth._rec("iTurbVars", 0))
    lines[i] = synth._rec("iTurbVars", 1)
    open(p, "w").write("\n".join(lines) + "\n")
    with pytest.raises(RuntimeError, match="turbulence"):
        oracle_lib.OracleRun(d)
    h = native_libs.host()
    hm = C.c_int(-1)
    err = C.create_string_buffer(256)
    assert h.si3d_host_open(d.encode(), None, C.byref(hm), err, 256) == -101
    assert b"turbulence" in err.value


def test_space_xml_header(oracle_lib, tmp_path):
    """outs with ipxml < 0 (si3d_utils.f90:2605-2760): the Gr header on the first call only, the
    run parameters in FORMAT 1, the start time of the output and its time step (ipxml * idt, signed
    as the reference computes it), and the two binary space files left empty (outs_bin has no
    caller in the reference)."""
    import os

    from si3d_b200 import synth
    d = str(tmp_path / "xml")
    synth.make("t0", d, outputs={"ipxml": -1, "itspf": 0})
    o = oracle_lib.OracleRun(d, ordering=1, pcg_itmax=2000)
    o.run(3)
    lines = open(os.path.join(d, "spacefile.xml")).read().split("\n")
    assert lines[0] == '<?xml version="1.0"?>' and lines[1] == " "
    assert lines[4] == "<!-- Run Parameters:  dt =60.00 s  dz = 1.00 m  im =   25  jm =   17"
    assert lines[5] == "     itrsca = 4  itrap = 1  cd =  0.0025  ismooth = 0  beta = 0.050  niter = 2"
    assert lines[6] == "     itrmom = 1  f = 0.0001  wa =     8.0 -->"
    assert lines[10] == '        runTitle="SYNTHETIC t0 24x16x8"'
    assert lines[12] == '        startTime="2024/01/01 00:00:00" timeStepInSeconds="-60">'
    assert 'numDimensions="1">' in lines[17] and 'numDimensions="4">' in lines[26]
    assert lines[-3:] == ["</gov.usgs.gr>", " ", ""]
    for b in ("spacefile2d.bin", "spacefile3d.bin"):
        assert os.path.getsize(os.path.join(d, b)) == 0
