"""CPU restatement of the multigrid-mixed zeta solve (precision SI3D_MIXED_MG) - TEST INFRASTRUCTURE.

The SI3D_MIXED_MG form has no counterpart in the reference: it is FP64 iterative refinement around
FP32 conjugate gradients preconditioned by one symmetric aggregation-multigrid V-cycle (the design is
described in si3d_b200/csrc/mg.h and k_mg.cu).  This module restates that solve in numpy, operation
for operation in FP32 where the GPU computes in FP32 (no fused multiply-adds: the library is built
with -fmad=false), so that tests can check the GPU solve pass by pass: the hierarchy, the
half-sweeps, the restriction and prolongation, the inner CG recurrences and the refinement loop.
Reductions are summed in a different order than on the GPU, so iteration counts may differ by one
where a stopping test sits on its threshold.

Only tests import this module; the product never does.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
MIN_LEVELS = 5
COARSEST = 8192
MAX_LEVELS = 10
FACE_SCALE = F32(0.5)
MAX_OUTER = 40


class Level:
    """One level: rows x cols images of mass, faces to the next column (fc) and row (fr), 1/diag."""

    def __init__(self, mass, fc, fr, dinv):
        self.mass, self.fc, self.fr, self.dinv = mass, fc, fr, dinv
        self.rows, self.cols = mass.shape


def _pad(a):
    """Zero frame of one cell on every side."""
    return np.pad(a, 1)


def _west(a):   # value of the cell at column c - 1 (zero outside)
    return _pad(a)[1:-1, :-2]


def _east(a):   # column c + 1
    return _pad(a)[1:-1, 2:]


def _south(a):  # row r - 1
    return _pad(a)[:-2, 1:-1]


def _north(a):  # row r + 1
    return _pad(a)[2:, 1:-1]


def _diag(L: Level):
    fcw, fce, frs, frn = _west(L.fc), L.fc, _south(L.fr), L.fr
    return (((L.mass + fcw) + fce) + frs) + frn


def coarsen(F: Level) -> Level:
    rows, cols = (F.rows + 1) // 2, (F.cols + 1) // 2
    pr, pc = 2 * rows - F.rows, 2 * cols - F.cols

    def ext(a):     # the fine image extended by the frame rows/columns that the last aggregates reach
        return np.pad(a, ((1, pr + 1), (1, pc + 1)))

    m, fc, fr = ext(F.mass), ext(F.fc), ext(F.fr)
    r0 = 1 + 2 * np.arange(rows)[:, None]
    c0 = 1 + 2 * np.arange(cols)[None, :]
    mass = (m[r0, c0] + m[r0, c0 + 1]) + (m[r0 + 1, c0] + m[r0 + 1, c0 + 1])
    fcc = FACE_SCALE * (fc[r0, c0 + 1] + fc[r0 + 1, c0 + 1])
    frc = FACE_SCALE * (fr[r0 + 1, c0] + fr[r0 + 1, c0 + 1])
    fcw = FACE_SCALE * (fc[r0, c0 - 1] + fc[r0 + 1, c0 - 1])
    frs = FACE_SCALE * (fr[r0 - 1, c0] + fr[r0 - 1, c0 + 1])
    diag = (((mass + fcc) + frc) + fcw) + frs
    with np.errstate(divide="ignore"):
        dinv = np.where(diag > 0, F32(1) / np.where(diag > 0, diag, F32(1)), F32(0)).astype(F32)
    return Level(mass.astype(F32), fcc.astype(F32), frc.astype(F32), dinv)


def half_sweep(L: Level, z, b, col, G=None, eG=None):
    """Gauss-Seidel over cells with (r + c) % 2 == col; with eG, each neighbour value is its z plus
    the correction of its aggregate in the coarser level."""
    zw, ze, zs, zn = _west(z), _east(z), _south(z), _north(z)
    if eG is not None:
        gp = _pad(eG)
        r = np.arange(L.rows)[:, None]
        c = np.arange(L.cols)[None, :]
        zw = zw + gp[(r >> 1) + 1, ((c - 1) >> 1) + 1]
        ze = ze + gp[(r >> 1) + 1, ((c + 1) >> 1) + 1]
        zs = zs + gp[((r - 1) >> 1) + 1, (c >> 1) + 1]
        zn = zn + gp[((r + 1) >> 1) + 1, (c >> 1) + 1]
    s = (((b + L.fc * ze) + _west(L.fc) * zw) + L.fr * zn) + _south(L.fr) * zs
    new = L.dinv * s
    rr, cc = np.indices(z.shape)
    return np.where(((rr + cc) & 1) == col, new, z).astype(F32)


def residual(L: Level, z, b):
    fcw, fce, frs, frn = _west(L.fc), L.fc, _south(L.fr), L.fr
    az = (((_diag(L) * z - fce * _east(z)) - fcw * _west(z)) - frn * _north(z)) - frs * _south(z)
    return (b - az).astype(F32)


def restrict(F: Level, G: Level, z, b):
    """b of level G (the residual summed over 2 x 2 aggregates, children in the order (0,0), (0,1),
    (1,0), (1,1)) and z of G after the red half-sweep from zero."""
    res = residual(F, z, b)
    rp = np.pad(res, ((0, 2 * G.rows - F.rows), (0, 2 * G.cols - F.cols)))
    a = F32(0) + rp[0::2, 0::2]
    a = a + rp[0::2, 1::2]
    a = a + rp[1::2, 0::2]
    a = a + rp[1::2, 1::2]
    a = a.astype(F32)
    rr, cc = np.indices(a.shape)
    zg = np.where(((rr + cc) & 1) == 0, G.dinv * a, F32(0)).astype(F32)
    return a, zg


def vcycle_pcg(levels, r, zeta, bnorm, itmax):
    """FP32 MG-PCG from e = 0 on right-hand side r; returns (e, iterations, ier)."""
    L0 = levels[0]
    nl = len(levels)
    e = np.zeros_like(r)
    p_old = np.zeros_like(r)
    q = np.zeros_like(r)
    alpha, rz_old, it, ier = 0.0, 1.0, 0, 0
    rows, cols = np.indices(r.shape)
    red0 = ((rows + cols) & 1) == 0
    while True:
        a = F32(alpha)
        if it > 0:
            e = (e + a * p_old).astype(F32)
            r = (r - a * q).astype(F32)
        rr = float(np.sum(r.astype(np.float64) ** 2))
        z0 = np.where(red0, L0.dinv * r, F32(0)).astype(F32)
        if np.sqrt(rr) < bnorm * zeta:
            break
        if it >= itmax:
            ier = 1
            break
        # down
        zs, bs = [z0], [r]
        for k in range(nl - 1):
            zs[k] = half_sweep(levels[k], zs[k], bs[k], 1)
            bk, zk = restrict(levels[k], levels[k + 1], zs[k], bs[k])
            zs.append(zk)
            bs.append(bk)
        # coarsest: black, red
        zc = half_sweep(levels[-1], zs[-1], bs[-1], 1)
        zs[-1] = half_sweep(levels[-1], zc, bs[-1], 0)
        # up
        for k in range(nl - 2, -1, -1):
            zk = half_sweep(levels[k], zs[k], bs[k], 1, levels[k + 1], zs[k + 1])
            zs[k] = half_sweep(levels[k], zk, bs[k], 0)
        z = zs[0]
        rz = float(np.sum(r.astype(np.float64) * z.astype(np.float64)))
        if not rz > 0:
            ier = -7
            break
        beta = 0.0 if it == 0 else rz / rz_old
        rz_old = rz
        bt = F32(beta)
        if it == 0:
            pn = z.copy()
            pw, pe, ps, pnn = _west(z), _east(z), _south(z), _north(z)
        else:
            pn = (z + bt * p_old).astype(F32)
            pw = (_west(z) + bt * _west(p_old)).astype(F32)
            pe = (_east(z) + bt * _east(p_old)).astype(F32)
            ps = (_south(z) + bt * _south(p_old)).astype(F32)
            pnn = (_north(z) + bt * _north(p_old)).astype(F32)
        fcw, fce, frs, frn = _west(L0.fc), L0.fc, _south(L0.fr), L0.fr
        q = ((((_diag(L0) * pn - fce * pe) - fcw * pw) - frn * pnn) - frs * ps).astype(F32)
        pq = float(np.sum(pn.astype(np.float64) * q.astype(np.float64)))
        if not pq > 0:
            ier = -6
            break
        alpha = rz_old / pq
        p_old = pn
        it += 1
    return e, it, ier


def solve(lm, l2i, l2j, lEC, lWC, lNC, lSC, sx, sy, qq, x0, im1, jm1, *, pcg_tol=1e-12,
          srelpr=2.220446049250313e-16, itmax=2000):
    """The multigrid-mixed solve of one zeta system in column order (1-based maps, lm1 = absent).
    Returns (zeta per column, dict(iters=inner iterations over all passes, passes, stptst, ier))."""
    lm1 = lm + 1
    li = np.arange(1, lm + 1)
    r = l2i[:lm] - 1
    c = l2j[:lm] - 1
    E, W, N, S = lEC[:lm], lWC[:lm], lNC[:lm], lSC[:lm]
    sxi, syi = sx[:lm].astype(np.float64), sy[:lm].astype(np.float64)
    sxw = np.where(W != lm1, sx[np.minimum(W, lm) - 1], 0.0)
    sys_ = np.where(S != lm1, sy[np.minimum(S, lm) - 1], 0.0)
    diag = (((1.0 + sxi) + sxw) + syi) + sys_
    fN = np.where(N != lm1, syi, 0.0)
    fE = np.where(E != lm1, sxi, 0.0)
    shape = (im1, jm1)
    fc64, fr64, dg64, b64, u64 = (np.zeros(shape) for _ in range(5))
    fc64[r, c], fr64[r, c], dg64[r, c], b64[r, c], u64[r, c] = fN, fE, diag, qq[:lm], x0[:lm]
    mass0, fc0, fr0, dinv0 = (np.zeros(shape, F32) for _ in range(4))
    fc0[r, c] = fN.astype(F32)
    fr0[r, c] = fE.astype(F32)
    mass0[r, c] = ((((diag - fN) - fE) - sxw) - sys_).astype(F32)
    dinv0[r, c] = (1.0 / diag).astype(F32)
    levels = [Level(mass0, fc0, fr0, dinv0)]
    rows, cols = im1, jm1
    while True:
        n = len(levels)
        if (n >= MIN_LEVELS and rows * cols <= COARSEST) or n == MAX_LEVELS or (rows == 1 and cols == 1):
            break
        levels.append(coarsen(levels[-1]))
        rows, cols = levels[-1].rows, levels[-1].cols
    zeta = max(pcg_tol, 500.0 * srelpr)
    bn, stp, outer, total, ier = 1.0, 1.0, 0, 0, 0
    e = None
    while True:
        if outer > 0:
            u64 = u64 + e.astype(np.float64)
        y = dg64 * u64
        y = y + (-_south(fr64)) * _south(u64)
        y = y + (-_west(fc64)) * _west(u64)
        y = y + (-fc64) * _east(u64)
        y = y + (-fr64) * _north(u64)
        r64 = b64 - y
        if outer == 0:
            bn = max(np.sqrt(np.sum(b64 ** 2)), srelpr)
        rn = float(np.sqrt(np.sum(r64 ** 2)))
        stp = rn / bn
        if rn < bn * zeta:
            break
        if outer >= MAX_OUTER:
            ier = 1
            break
        e, its, iier = vcycle_pcg(levels, r64.astype(F32), max(1e-5, 0.5 * zeta * bn / rn), rn, itmax)
        total += its
        outer += 1
        if iier < 0:
            ier = iier
            break
    zc = np.zeros(lm1 + 1)
    zc[li - 1] = u64[r, c]
    return zc[:lm], dict(iters=total, passes=outer, stptst=stp, ier=ier, levels=len(levels))
