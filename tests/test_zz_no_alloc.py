"""The allocation-free tridiagonal entry point, through the C ABI.

It exists for callers that cannot call cudaMalloc (a model coupled into a framework that owns the
device allocator, or a loop that must not allocate once running): they pass their own device
buffers and the solver's scratch comes from a fixed array inside the library.  Its results must
equal those of the allocating entry point, including on a second call that reuses the scratch
array after a first call left its contents behind.  This file is collected last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(rng, n, nsys):
    a = rng.uniform(-1.0, 0.0, (n, nsys))
    c = rng.uniform(-1.0, 0.0, (n, nsys))
    b = 2.5 + rng.uniform(0.0, 1.0, (n, nsys))
    a[0] = 0.0
    c[-1] = 0.0
    g = rng.standard_normal((n, nsys))
    r = rng.standard_normal((n, nsys))
    return a, b, c, g, r


def _banded(a, b, c, rhs, s):
    """System s solved by LAPACK's banded solver (an independent check of both entry points)."""
    from scipy.linalg import solve_banded
    n = a.shape[0]
    ab = np.zeros((3, n))
    ab[0, 1:] = c[:-1, s]
    ab[1] = b[:, s]
    ab[2, :-1] = a[1:, s]
    return solve_banded((1, 1), ab, rhs[:, s])


def test_noalloc_matches_allocating_entry(native_libs):
    import torch

    from si3d_b200 import native
    from si3d_b200.model import column_tridiag

    lib = native.gpu()
    rng = np.random.default_rng(20261203)
    # three calls in a row with different shapes: each reuses the scratch the one before filled; the
    # last fills the array exactly (n * nsys == SI3D_NOALLOC_MAX_ELEMS)
    for n, nsys in ((62, 9000), (41, 16384), (64, 16384)):
        a, b, c, g, r = _system(rng, n, nsys)
        ag_ref, ar_ref = column_tridiag(a, b, c, g, r)
        for s in rng.choice(nsys, 16, replace=False):
            np.testing.assert_allclose(ag_ref[:, s], _banded(a, b, c, g, s), rtol=1e-12, atol=1e-14)
            np.testing.assert_allclose(ar_ref[:, s], _banded(a, b, c, r, s), rtol=1e-12, atol=1e-14)
        # caller-owned device buffers, layer-major: element k of system s at k*nsys + s
        dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (a, b, c, g, r)]
        ag = torch.empty((n, nsys), dtype=torch.float64, device="cuda")
        ar = torch.empty_like(ag)
        torch.cuda.synchronize()
        rc = lib.si3d_gpu_column_tridiag_noalloc(n, nsys, *[C.c_void_p(t.data_ptr()) for t in dev],
                                                 C.c_void_p(ag.data_ptr()), C.c_void_p(ar.data_ptr()), None)
        assert rc == 0, lib.si3d_gpu_strerror(rc)
        np.testing.assert_allclose(ag.cpu().numpy(), ag_ref, rtol=1e-14, atol=1e-300)
        np.testing.assert_allclose(ar.cpu().numpy(), ar_ref, rtol=1e-14, atol=1e-300)


def test_noalloc_rejects_oversize(native_libs):
    from si3d_b200 import native

    lib = native.gpu()
    dummy = C.c_void_p(1)
    n = 64
    nsys = native_max = (1 << 20) // n + 1
    rc = lib.si3d_gpu_column_tridiag_noalloc(n, nsys, *([dummy] * 7), None)
    assert rc == -108, (rc, native_max)
