"""The C-ABI boundary on the CPU: both libraries load, export every function that include/*.h
declares, and refuse to run without an sm_100 device (there is no CPU fallback)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT

DECL = re.compile(r"^\s*(?:const\s+)?(?:int|void|char|double|size_t)\s*\*?\s*(si3d_\w+)\s*\(", re.M)


def _declared(header: str):
    with open(header) as fh:
        return sorted(set(DECL.findall(fh.read())))


def test_headers_declare_the_boundary():
    gpu = _declared(os.path.join(ROOT, "include", "si3d_gpu.h"))
    host = _declared(os.path.join(ROOT, "include", "si3d_host.h"))
    for name in ("si3d_gpu_init", "si3d_gpu_fd", "si3d_gpu_settrap", "si3d_gpu_settrap2", "si3d_gpu_save",
                 "si3d_gpu_solve_zeta", "si3d_gpu_column_tridiag", "si3d_gpu_column_tridiag_noalloc",
                 "si3d_gpu_strerror", "si3d_gpu_finalize"):
        assert name in gpu
    assert "si3d_host_open" in host and "si3d_host_run" in host


@pytest.mark.parametrize("header,lib", [("si3d_gpu.h", "libsi3d_gpu.so"), ("si3d_learn.h", "libsi3d_gpu.so"),
                                        ("si3d_host.h", "libsi3d_host.so")])
def test_library_exports_every_declared_symbol(native_libs, header, lib):
    native_libs.gpu()   # the host library resolves CUDA-core symbols from it
    so = C.CDLL(os.path.join(ROOT, "si3d_b200", "_lib", lib))
    missing = [n for n in _declared(os.path.join(ROOT, "include", header)) if not hasattr(so, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_python_bindings_cover_the_headers(native_libs):
    gpu = set(_declared(os.path.join(ROOT, "include", "si3d_gpu.h")))
    gpu |= set(_declared(os.path.join(ROOT, "include", "si3d_learn.h")))
    host = set(_declared(os.path.join(ROOT, "include", "si3d_host.h")))
    assert gpu == set(native_libs.GPU_SYMBOLS)
    assert host == set(native_libs.HOST_SYMBOLS)


def test_fortran_interface_binds_the_same_names():
    """The ISO_C_BINDING module names exactly the exported entry points it binds."""
    f90 = glob.glob(os.path.join(ROOT, "si3d_b200", "fortran", "*.f90"))
    assert f90
    text = open(f90[0]).read()
    bound = set(re.findall(r'BIND\(C,\s*NAME="(si3d_\w+)"\)', text, re.I))
    declared = set(_declared(os.path.join(ROOT, "include", "si3d_gpu.h")))
    declared |= set(_declared(os.path.join(ROOT, "include", "si3d_learn.h")))
    assert bound and bound <= declared


def test_error_strings(native_libs):
    g = native_libs.gpu()
    for code in (0, 1, 2, 5, -6, -7, -12, -100, -101, -102, -103, -104, -105, -106, -107, -108):
        s = g.si3d_gpu_strerror(code).decode()
        assert s and s != "unknown error", code
    assert g.si3d_gpu_strerror(-999).decode() == "unknown error"


def _tiny_grid():
    """A 2 x 1 wet-column grid with valid maps (lm1 = 3 is the dry sentinel)."""
    keep = []

    def arr(v, t):
        a = np.ascontiguousarray(v, dtype=t)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_int if t == np.int32 else C.c_double))

    from si3d_b200 import native
    g = native.Grid()
    g.im1, g.jm1, g.km1, g.k1, g.lm = 4, 3, 4, 2, 2
    g.l2i, g.l2j = arr([2, 3, 0], np.int32), arr([2, 2, 0], np.int32)
    g.lEC, g.lWC = arr([2, 3, 3], np.int32), arr([3, 1, 3], np.int32)
    g.lNC, g.lSC = arr([3, 3, 3], np.int32), arr([3, 3, 3], np.int32)
    g.kmz = arr([3, 3, 0], np.int32)
    g.hhs = g.hhu = g.hhv = arr([2.0, 2.0, 0.0], np.float64)
    g.zlevel = arr([-100.0, 0.0, 1.0, 2.0], np.float64)
    p = native.Params()
    p.dt, p.dx, p.dy, p.theta, p.itrmom, p.pcg_test, p.pcg_tol, p.pcg_itmax = 30.0, 100.0, 100.0, 1.0, 1, 5, 1e-12, 10
    p.srelpr = 2.220446049250313e-16
    return g, p, keep


def test_bad_arguments_are_rejected(native_libs):
    g = native_libs.gpu()
    h = C.c_int(-1)
    grid, prm, _keep = _tiny_grid()
    grid.k1 = 3                                     # the core is built for k1 = 2 only
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101
    grid.k1 = 2
    prm.itrmom = 2                                  # only itrmom = 1 is on the path
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101
    prm.itrmom = 1
    prm.ordering = 3                                # red-black (0, 1) or natural (2)
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101
    prm.ordering, prm.precision = 2, 1              # the natural ordering is the plain FP64 solve
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101
    prm.ordering, prm.precision = 1, 0
    assert g.si3d_gpu_fd(12345, 1, 1, 0, None) == -102
    assert g.si3d_gpu_sync(-1) == -102


def test_maps_and_depths_out_of_range_are_rejected(native_libs):
    """The kernels index neighbours through the maps and layers down to kmz + 1; maps outside
    [1, lm + 1], a bottom layer outside [k1, km1 - 1] and more tracers than ntrmax are refused at
    init, before any device work."""
    g = native_libs.gpu()
    h = C.c_int(-1)
    for field, bad in (("kmz", [4, 3, 0]), ("kmz", [1, 3, 0]), ("lEC", [4, 3, 3]), ("lSC", [0, 3, 3])):
        grid, prm, keep = _tiny_grid()
        a = np.ascontiguousarray(bad, dtype=np.int32)
        keep.append(a)
        setattr(grid, field, a.ctypes.data_as(C.POINTER(C.c_int)))
        assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101, field
    grid, prm, _keep = _tiny_grid()
    prm.ntr = 31
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -101


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_device_fails_loudly(native_libs):
    """Without an sm_100 device the core returns SI3D_ENODEV instead of computing anything."""
    g = native_libs.gpu()
    grid, prm, _keep = _tiny_grid()
    h = C.c_int(-1)
    assert g.si3d_gpu_init(C.byref(grid), C.byref(prm), 0, C.byref(h)) == -107
    with pytest.raises(native_libs.Si3dError, match="no sm_100"):
        native_libs.check(-107)
