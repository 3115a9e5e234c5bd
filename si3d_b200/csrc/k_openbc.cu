// Open boundaries with a specified water-surface elevation (itype = 1): the stage adjustments of
// si3d_boundaryconditions.f90 for the cells along each boundary.
//
// Each boundary is a short list of cells (one side of the grid), so every adjustment is one small
// kernel over that list, launched per boundary in the reference's boundary order, between the
// stage kernels it modifies:
//   obc_set_s     openbcUVH CASE(1) (:900-970): zeta on the boundary cells (fd start, after the solve)
//   obc_exmom     MODexmom4openBCX/Y CASE(1) (:1801-1880, :2370-2510): the staged explicit term of the
//                 face columns at the boundary - upwind advection only (west, north, south) or zero
//                 (east, whose assignment the reference has commented out)
//   obc_qq        MODqqddrr4openBC CASE(1) (:1508-1580): the boundary value moves to the right-hand
//                 side of the interior neighbour and the face coefficient is cut (rr keeps it)
//   obc_vel       MODvel4openBC CASE(1) (:2941-3010): the velocity along the boundary is zeroed and wp
//                 copied from the interior neighbour (after every continuity)
//   obc_sca       openbcSCA CASE(1) (:3157-3250): temperature of the boundary cells after imsal
// The expressions are the reference's, in its operation order.
#include "common.cuh"
#include "kernels.h"

namespace si3d {

namespace {

constexpr int OB = 128;

__global__ void k_obc_set_s(Dev d, const int* __restrict__ cells, int n, double v) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) d.s.s[cells[t] - 1] = v;
}

__device__ __forceinline__ double pos(double a) { return a + fabs(a); }
__device__ __forceinline__ double neg(double a) { return a - fabs(a); }

// kind: 0 west (u face of the boundary cell), 1 east (u face of the cell inside), 2 north (v face of
// the cell inside), 3 south (v face of the boundary cell).  The staged explicit term lives in agx
// (agy) at the face column's wet layers until the column sweep reads it.
__global__ void k_obc_exmom(Dev d, const int* __restrict__ cols, int n, int kind) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int l = cols[t];
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const double twodt1 = d.p.twodt * d.tz;
  const double iadv = d.p.iadv;
  if (kind <= 1) {
    const int kmx = min(NB(d.g.kmz, lE), NB(d.g.kmz, l)), k1x = NB(d.s.k1u, l);
    if (kmx - k1x + 1 < 1) return;
    const int lSE = NB(d.g.lSC, lE);
    for (int k = k1x; k <= kmx; ++k) {
      const int ik = IX(d, k, l);
      if (kind == 1) { d.f.agx[ik] = 0.0; continue; }
      const double* uhp = d.f.uhp;
      const double* vhp = d.f.vhp;
      const double* wp = d.f.wp;
      const double* upp = d.f.upp;
      const double uE = uhp[IX(d, k, lE)] + uhp[ik], uW = uhp[ik] + uhp[ik];
      const double vN = vhp[IX(d, k, lE)] + vhp[ik], vS = vhp[IX(d, k, lSE)] + vhp[IX(d, k, lS)];
      const double wU = wp[IX(d, k, lE)] + wp[ik], wD = wp[IX(d, k + 1, lE)] + wp[IX(d, k + 1, l)];
      double advx = (pos(uE) * upp[ik] + neg(uE) * upp[IX(d, k, lE)] - pos(uW) * upp[ik] - neg(uW) * upp[ik]) / d.p.fourdx +
                    (pos(vN) * upp[ik] + neg(vN) * upp[IX(d, k, lN)] - pos(vS) * upp[IX(d, k, lS)] - neg(vS) * upp[ik]) /
                        d.p.fourdy;
      advx = advx + (pos(wU) * upp[ik] + neg(wU) * upp[IX(d, k - 1, l)]) / 4. -
             (pos(wD) * upp[IX(d, k + 1, l)] + neg(wD) * upp[ik]) / 4.;
      d.f.agx[ik] = d.f.uhpp[ik] - twodt1 * (advx * iadv);
    }
    (void)lW;
  } else {
    const int kmy = min(NB(d.g.kmz, lN), NB(d.g.kmz, l)), k1y = NB(d.s.k1v, l);
    if (kmy - k1y + 1 < 1) return;
    const int lWN = NB(d.g.lWC, lN);
    const bool north = kind == 2;
    for (int k = k1y; k <= kmy; ++k) {
      const int ik = IX(d, k, l);
      const double* uhp = d.f.uhp;
      const double* vhp = d.f.vhp;
      const double* wp = d.f.wp;
      const double* vpp = d.f.vpp;
      const double uE = uhp[IX(d, k, lN)] + uhp[ik], uW = uhp[IX(d, k, lWN)] + uhp[IX(d, k, lW)];
      const double vN = north ? vhp[ik] + vhp[ik] : vhp[IX(d, k, lN)] + vhp[ik];
      const double vS = north ? vhp[ik] + vhp[IX(d, k, lS)] : vhp[ik] + vhp[ik];
      const double wU = wp[IX(d, k, lN)] + wp[ik], wD = wp[IX(d, k + 1, lN)] + wp[IX(d, k + 1, l)];
      const double vNn = north ? vpp[ik] : vpp[IX(d, k, lN)];
      const double vSs = north ? vpp[IX(d, k, lS)] : vpp[ik];
      double advy = (pos(uE) * vpp[ik] + neg(uE) * vpp[IX(d, k, lE)] - pos(uW) * vpp[IX(d, k, lW)] - neg(uW) * vpp[ik]) /
                        d.p.fourdx +
                    (pos(vN) * vpp[ik] + neg(vN) * vNn - pos(vS) * vSs - neg(vS) * vpp[ik]) / d.p.fourdy;
      advy = advy + (pos(wU) * vpp[ik] + neg(wU) * vpp[IX(d, k - 1, l)]) / 4. -
             (pos(wD) * vpp[IX(d, k + 1, l)] + neg(wD) * vpp[ik]) / 4.;
      d.f.agy[ik] = d.f.vhpp[ik] - twodt1 * (advy * iadv);
    }
  }
}

// qq of the interior neighbour += face * s(boundary cell), then the face is cut.  `face` is the
// column whose sx (sy) couples the pair: the boundary cell (west, south) or the interior one (east,
// north).  One cell pair per thread; no face or interior cell is shared within a boundary.
__global__ void k_obc_qq(Dev d, const int* __restrict__ cells, const int* __restrict__ inner,
                         const int* __restrict__ face, int n, int ysx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int lb = cells[t], li = inner[t], lf = face[t];
  double* fc = ysx ? d.s.sy : d.s.sx;
  d.s.qq[li - 1] = d.s.qq[li - 1] + fc[lf - 1] * d.s.s[lb - 1];
}
__global__ void k_obc_cut(Dev d, const int* __restrict__ face, int n, int ysx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  (ysx ? d.s.sy : d.s.sx)[face[t] - 1] = 0.0;
}

// The boundary cell's velocity along the boundary (vh on west/east, uh on north/south) is zero and
// its wp is the interior neighbour's, at every level.
__global__ void k_obc_vel(Dev d, const int* __restrict__ cells, const int* __restrict__ inner, int n, int ysx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int l = cells[t], src = inner[t];
  double* f = ysx ? d.f.uh : d.f.vh;
  for (int k = 1; k <= d.g.km1; ++k) {
    f[IX(d, k, l)] = 0.0;
    d.f.wp[IX(d, k, l)] = d.f.wp[IX(d, k, src)];
  }
}

// Temperature of the boundary cells: salbc where the flow enters (and salbc > 0), the interior
// neighbour's otherwise.  side: 1 W, 2 N, 3 E, 4 S.
__global__ void k_obc_sca(Dev d, const int* __restrict__ cells, const int* __restrict__ inner, int n, int side,
                          double salbc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int l = cells[t], src = inner[t];
  for (int k = d.s.k1z[l - 1]; k <= NB(d.g.kmz, l); ++k) {
    bool in;
    switch (side) {
      case 1: in = d.f.uh[IX(d, k, l)] > 0.0; break;
      case 2: in = d.f.vh[IX(d, k, NB(d.g.lSC, l))] < 0.0; break;
      case 3: in = d.f.uh[IX(d, k, NB(d.g.lWC, l))] < 0.0; break;
      default: in = d.f.vh[IX(d, k, l)] > 0.0; break;
    }
    d.f.sal[IX(d, k, l)] = (in && salbc > 0.0) ? salbc : d.f.sal[IX(d, k, src)];
  }
}

inline int grid(int n) { return (n + OB - 1) / OB; }

}  // namespace

void obc_set_s(const Dev& d, const ObcDev& B, double v, cudaStream_t st) {
  if (B.n > 0) k_obc_set_s<<<grid(B.n), OB, 0, st>>>(d, B.cells, B.n, v);
}

void obc_exmom(const Dev& d, const ObcDev& B, int ieq, cudaStream_t st) {
  const bool x = B.side == 1 || B.side == 3;
  if ((ieq == 1) != x || B.nface <= 0) return;
  const int kind = B.side == 1 ? 0 : B.side == 3 ? 1 : B.side == 2 ? 2 : 3;
  k_obc_exmom<<<grid(B.nface), OB, 0, st>>>(d, B.mom, B.nface, kind);
}

void obc_qq(const Dev& d, const ObcDev& B, cudaStream_t st) {
  if (B.n <= 0) return;
  const int ysx = (B.side == 2 || B.side == 4) ? 1 : 0;
  k_obc_qq<<<grid(B.n), OB, 0, st>>>(d, B.cells, B.inner, B.face, B.n, ysx);
  k_obc_cut<<<grid(B.n), OB, 0, st>>>(d, B.face, B.n, ysx);
}

void obc_vel(const Dev& d, const ObcDev& B, cudaStream_t st) {
  if (B.n <= 0) return;
  const int ysx = (B.side == 2 || B.side == 4) ? 1 : 0;
  k_obc_vel<<<grid(B.n), OB, 0, st>>>(d, B.cells, B.inner, B.n, ysx);
}

void obc_sca(const Dev& d, const ObcDev& B, double salbc, cudaStream_t st) {
  if (B.n > 0) k_obc_sca<<<grid(B.n), OB, 0, st>>>(d, B.cells, B.inner, B.n, B.side, salbc);
}

}  // namespace si3d
