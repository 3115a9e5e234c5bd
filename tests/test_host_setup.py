"""The native host set-up (reading the reference's input files and building the grid maps) against
the oracle's restatement of input/ZGridDimensions/bathy (si3d_utils.f90:21-382, 595-892), and its
error paths.  CPU only."""
import ctypes as C
import os
import shutil

import numpy as np
import pytest

from si3d_b200 import synth

MAPS = ("l2i", "l2j", "lEC", "lWC", "lNC", "lSC", "kmz")


def _open(native, run_dir):
    h = native.host()
    hm = C.c_int(-1)
    err = C.create_string_buffer(512)
    rc = h.si3d_host_open(run_dir.encode(), None, C.byref(hm), err, 512)
    return rc, hm.value, err.value.decode()


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_maps_match_oracle(native_libs, oracle_lib, run_dirs, name):
    rc, hm, err = _open(native_libs, run_dirs[name])
    assert rc == 0, err
    h = native_libs.host()
    try:
        dims = (C.c_int * 6)()
        h.si3d_host_dims(hm, dims)
        o = oracle_lib.OracleRun(run_dirs[name])
        assert (dims[0], dims[1], dims[2], dims[3]) == (o.im1, o.jm1, o.km1, o.lm)
        for m in MAPS:
            a = np.empty(o.lm1, dtype=np.int32)
            assert h.si3d_host_get_map(hm, m.encode(), native_libs.ptr(a)) == 0
            np.testing.assert_array_equal(a, o.geti(m), err_msg=m)
        z = np.empty(o.km1)
        h.si3d_host_get_zlevel(hm, native_libs.ptr(z))
        np.testing.assert_array_equal(z, o.zlevel())
        assert h.si3d_host_get_map(hm, b"nope", native_libs.ptr(np.empty(o.lm1, dtype=np.int32))) == -103
    finally:
        h.si3d_host_close(hm)


def _copy(src, dst):
    shutil.copytree(src, dst)
    return dst


def test_missing_file(native_libs, tmp_path):
    rc, _, err = _open(native_libs, str(tmp_path))
    assert rc == -101 and "si3d_inp.txt" in err


def test_truncated_bathymetry(native_libs, run_dirs, tmp_path):
    d = _copy(run_dirs["t0"], str(tmp_path / "trunc"))
    p = os.path.join(d, "si3d_bathy")
    lines = open(p).read().splitlines()
    open(p, "w").write("\n".join(lines[: len(lines) // 2]) + "\n")
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "truncated" in err


def test_truncated_profile(native_libs, run_dirs, tmp_path):
    d = _copy(run_dirs["t0"], str(tmp_path / "prof"))
    p = os.path.join(d, "si3d_init.txt")
    lines = open(p).read().splitlines()
    open(p, "w").write("\n".join(lines[:-2]) + "\n")
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "si3d_init.txt" in err


@pytest.mark.parametrize("label,value", [("iturb", 2), ("iturb", -1)])
def test_options_outside_the_core_are_refused(native_libs, run_dirs, tmp_path, label, value):
    """The k-kl closure (iturb >= 2) and GOTM (iturb = -1) are not built; a run that selects them is
    refused rather than silently run without them (open boundaries other than itype 1: see
    test_openbc_oracle.py)."""
    d = _copy(run_dirs["t0"], str(tmp_path / f"opt_{label}_{value}"))
    p = os.path.join(d, "si3d_inp.txt")
    lines = open(p).read().splitlines()
    rec = synth._rec(label, 0)
    i = lines.index(rec)
    lines[i] = synth._rec(label, value)
    open(p, "w").write("\n".join(lines) + "\n")
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "outside the semi-implicit core" in err


def test_wind_override_size_mismatch(native_libs, run_dirs, tmp_path):
    d = _copy(run_dirs["t1"], str(tmp_path / "wind"))
    p = os.path.join(d, "si3d_wind_override.bin")
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "size mismatch" in err


def _set_records(path, values):
    lines = open(path).read().splitlines()
    for label, value in values:
        lines[lines.index(synth._rec(label, 0))] = synth._rec(label, value)
    open(path, "w").write("\n".join(lines) + "\n")


def test_tracer_run_opens(native_libs, oracle_lib, tmp_path):
    """Conservative tracers (ecomod = 0): the host and the oracle both read ntr and the extra
    columns of si3d_init.txt."""
    d = str(tmp_path / "tr")
    synth.make("t0", d, ntr=3)
    rc, hm, err = _open(native_libs, d)
    assert rc == 0, err
    native_libs.host().si3d_host_close(hm)
    assert oracle_lib.OracleRun(d).ntr == 3


def test_tracer_models_other_than_conservative_are_refused(native_libs, oracle_lib, tmp_path):
    """Water quality, tracer clouds, size structure and sediment (ecomod != 0) are refused by the
    host and by the oracle instead of being run as conservative tracers."""
    d = str(tmp_path / "eco")
    synth.make("t0", d, ntr=2)
    _set_records(os.path.join(d, "si3d_inp.txt"), [("ecomod", 1)])
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "conservative" in err
    with pytest.raises(RuntimeError, match="conservative"):
        oracle_lib.OracleRun(d)


def test_tracer_columns_missing_from_profile(native_libs, oracle_lib, run_dirs, tmp_path):
    """ntr > 0 with a one-column si3d_init.txt: a formatted read pads the short records with blanks,
    which read as zero, so the tracers start at zero (the host and the oracle both open the run)."""
    d = _copy(run_dirs["t0"], str(tmp_path / "ntr_noprof"))
    _set_records(os.path.join(d, "si3d_inp.txt"), [("ntr", 2)])
    rc, hm, err = _open(native_libs, d)
    assert rc == 0, err
    native_libs.host().si3d_host_close(hm)
    o = oracle_lib.OracleRun(d)
    assert o.ntr == 2 and not o.get("tracer2").any()


@pytest.mark.parametrize("label,value", [("nnodes", 2)])
def test_unbuilt_writers_are_refused(native_libs, oracle_lib, run_dirs, tmp_path, label, value):
    """Time series at nodes (outt) are not built: a run that asks for them is refused instead of
    running without its files."""
    d = _copy(run_dirs["t0"], str(tmp_path / f"w_{label}"))
    _set_records(os.path.join(d, "si3d_inp.txt"), [(label, value)])
    rc, _, err = _open(native_libs, d)
    assert rc == -101 and "not built" in err
    with pytest.raises(RuntimeError, match="not restated"):
        oracle_lib.OracleRun(d)
