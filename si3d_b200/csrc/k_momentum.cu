// Momentum stage: exmom + matmom + trid, split into a cell-parallel and a column-sequential kernel.
//
// Reference: exmom (si3d_procedures.f90:578-1173), matmom (:1176-1630), bclnc_km (:1633-1746),
// trid (:3210-3289).  The work items are the u (v) face columns l whose east (north) neighbour is
// wet — the reference's id_columnCE (id_columnCN) list.
//
// k_mom_cells (block = 32 face columns x 8 layer lanes): every wet face cell independently forms
//   the parts that couple neighbouring columns - the explicit term ex(k) (advection, Coriolis,
//   horizontal diffusion) and the baroclinic increment (with bclnc_km's bottom-layer
//   interpolation) - and stages them in ag(k) and ar(k), the output arrays of this stage.  A warp
//   is 32 consecutive face columns at one layer: every field access is a coalesced run of the
//   layer-major layout, and thousands of independent cells keep the loads in flight.
// k_mom_columns (one thread per face column): everything that runs down the column - the
//   depth-mean density, the baroclinic prefix sum, explicit vertical diffusion, the tridiagonal
//   coefficients and boundary terms (wind and bottom stress) and the Thomas sweeps with two
//   right-hand sides - reading the staged ex/increment back and writing the final ag/ar.  The c'
//   coefficients of the forward sweep go to the Thomas scratch array.
// The cell kernel evaluates the reference's expressions in its operation order, except that it
// multiplies by the reciprocals of the grid constants (4 dx, 4 dy, dx^2, dy^2) where the reference
// divides by them, and forms the interpolation weights hk / (hk + hkp) as hk * (1 / (hk + hkp)).  The column kernel shares reciprocals between the tridiagonal coefficients (three
// divisions a layer instead of ten) and sums the depth totals during the back substitution (bottom
// to top), so ag, ar, eag and ear agree with the reference's arithmetic to a few units in the last
// place.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace si3d {

namespace {

constexpr int CW = 32;   // face columns per block of the cell kernel (layer lanes per column: CL)


// Horizontal-diffusion coefficient of a neighbouring face column m at layer k
// (haxpp/haypp as rebuilt by exmom each call, :623-681 / :962-1018): zero outside that
// column's wet face layers or when its face is closed.  The two depths are loaded by the caller
// unconditionally (m = lm1 is the dry column, a valid address), so the test only selects.
__device__ __forceinline__ double face_coef(const Dev& d, double A, double h_other, double h_m, int m, int kfirst,
                                            int klast, int k) {
  return (m == d.g.lm1 || k < kfirst || k > klast) ? 0.0 : A * fmin(h_other, h_m);
}

struct FaceCol {
  int l, lE, lW, lN, lS, lO, kmx, k1x, lX2;
};

// ------------------------------------------------------------------ cell terms
// The per-thread description of one face column that the cell terms read.
struct CellCol {
  int l, lW, lS, lO, k1x, kmx, mW_first, mW_last, mS_first, mS_last;
  int dE, dW, dN, dS, dX2, dO;
};

template <int IEQ>
__device__ __forceinline__ CellCol cell_col(const Dev& d, const FaceMeta* __restrict__ meta, int t) {
  const bool X = (IEQ == 1);
  const int4 ma = __ldg(&meta[t].a), mb = __ldg(&meta[t].b);
  const int l = ma.x, lE = ma.y, lW = ma.z, lN = ma.w, lS = mb.x, lX2 = mb.y;
  CellCol C;
  C.l = l; C.lW = lW; C.lS = lS; C.kmx = mb.z;
  C.lO = X ? lE : lN;
  const int* k1f = X ? d.s.k1u : d.s.k1v;
  C.k1x = NB(k1f, l);
  // west / south neighbouring faces' diffusion ranges (their first wet layers change per step)
  C.mW_last = mb.w;
  C.mS_last = __ldg(&meta[t].c.x);
  C.mW_first = C.mW_last >= 0 ? NB(k1f, lW) : 0;
  C.mS_first = C.mS_last >= 0 ? NB(k1f, lS) : 0;
  C.dE = lE - l; C.dW = lW - l; C.dN = lN - l; C.dS = lS - l; C.dX2 = lX2 - l; C.dO = C.lO - l;
  return C;
}

// The explicit term ex(k) (advection, Coriolis, horizontal diffusion) and the baroclinic increment
// of wet face layer k of column C, and the thickness of layer k + 1 (loaded for the weights anyway).
template <int IEQ>
__device__ __forceinline__ void mom_cell(const Dev& d, const CellCol& C, int k, double& ex_out, double& hdrho_out,
                                         double& hkp_out) {
  const bool X = (IEQ == 1);
  const int l = C.l, lO = C.lO, k1x = C.k1x, kmx = C.kmx;
  const int dE = C.dE, dW = C.dW, dN = C.dN, dS = C.dS, dX2 = C.dX2, dO = C.dO;
  const double* huv = X ? d.f.hup : d.f.hvp;
  const double* huvpp = X ? d.f.hupp : d.f.hvpp;
  const double* uvpp_h = X ? d.f.uhpp : d.f.vhpp;
  const double* uvp = X ? d.f.up : d.f.vp;
  const double* uvpp = X ? d.f.upp : d.f.vpp;
  const double twodt1 = d.p.twodt * d.tz;
  const double gdt = X ? d.p.gdtdx : d.p.gdtdy;
  const double* __restrict__ vhp = d.f.vhp;
  const double* __restrict__ uhp = d.f.uhp;
  const double* __restrict__ wp = d.f.wp;
  const double* __restrict__ hp3 = d.f.hp;
  const int P = d.g.P;
  const int ik = IX(d, k, l);
  // every input of the explicit term is loaded before the dry-cell test, so a layer costs one
  // memory round trip; the arithmetic below is the reference's, term by term
  const double hk = huv[ik];
  const double hkm = huv[ik - P];
  const double hkp = huv[ik + P];
  const double hpl = hp3[ik], hpo = hp3[ik + dO];
  double cor, uE, uW, vN, vS, wU, wD;
  if (X) {
    const double vE = vhp[ik + dE], vC = vhp[ik], vX = vhp[ik + dX2], vSS = vhp[ik + dS];
    const double uEE = uhp[ik + dE], uC = uhp[ik], uWW = uhp[ik + dW];
    cor = 0.25 * d.p.f * (vE + vC + vX + vSS);
    uE = uEE + uC;
    uW = uC + uWW;
    vN = vE + vC;
    vS = vX + vSS;
    wU = wp[ik + dE] + wp[ik];
    wD = wp[ik + P + dE] + wp[ik + P];
  } else {
    const double uN = uhp[ik + dN], uC = uhp[ik], uX = uhp[ik + dX2], uWW = uhp[ik + dW];
    const double vNN = vhp[ik + dN], vC = vhp[ik], vSS = vhp[ik + dS];
    cor = 0.25 * d.p.f * (uN + uC + uX + uWW);
    uE = uN + uC;
    uW = uX + uWW;
    vN = vNN + vC;
    vS = vC + vSS;
    wU = wp[ik + dN] + wp[ik];
    wD = wp[ik + P + dN] + wp[ik + P];
  }
  const double uc = uvp[ik];
  const double uvE = uvp[ik + dE], uvW = uvp[ik + dW], uvN = uvp[ik + dN], uvS = uvp[ik + dS];
  const double uvU = uvp[ik - P], uvD = uvp[ik + P];
  const double own_pp = uvpp_h[ik];
  double hd = 0.0;
  if (d.p.ihd == 1) {
    const double hppl = huvpp[ik], hppE = huvpp[ik + dE], hppN = huvpp[ik + dN];
    const double hppW = huvpp[ik + dW], hppS = huvpp[ik + dS];
    const double pc = uvpp[ik], pN = uvpp[ik + dN], pS = uvpp[ik + dS], pE = uvpp[ik + dE], pW = uvpp[ik + dW];
    const double ax_l = d.p.Ax0 * fmin(hppE, hppl);
    const double ay_l = d.p.Ay0 * fmin(hppN, hppl);
    const double ax_w = face_coef(d, d.p.Ax0, hppl, hppW, C.lW, C.mW_first, C.mW_last, k);
    const double ay_s = face_coef(d, d.p.Ay0, hppl, hppS, C.lS, C.mS_first, C.mS_last, k);
    hd = (ay_l * (pN - pc) - ay_s * (pc - pS)) * d.p.rdydy + (ax_l * (pE - pc) - ax_w * (pc - pW)) * d.p.rdxdx;
  }
  double ex;
  if (hpl <= ZERO || hpo <= ZERO) {
    ex = own_pp;
  } else {
    const double th_k = (k == k1x) ? 0.0 : hkm * (1.0 / (hkm + hk));
    const double th1_k = (k == k1x) ? 0.0 : 1. - th_k;
    const double th_kp = (k == kmx) ? 0.5 : hk * (1.0 / (hk + hkp));
    const double th1_kp = (k == kmx) ? 0.5 : 1. - th_kp;
    if (k == k1x) wU = 0.0;
    if (k == kmx) wD = 0.0;
    const double scE = uvE + uc, scW = uvW + uc;
    const double scN = uvN + uc, scS = uvS + uc;
    double adv = (uE * scE - uW * scW) * d.p.rfourdx + (vN * scN - vS * scS) * d.p.rfourdy;
    adv = adv + (wU * (th_k * uc + th1_k * uvU) - wD * (th_kp * uvD + th1_kp * uc)) / 2.;
    if (X) ex = own_pp - twodt1 * (adv * d.p.iadv - cor - hd);
    else ex = own_pp - twodt1 * (adv * d.p.iadv + cor - hd);
  }
  // ---- baroclinic increment (:1283-1301 / :1475-1491), bottom layer via bclnc_km
  double hdrho = 0;
  if (d.p.ibc != 0) {
    hdrho = gdt * hk * (d.f.rhop[IX(d, k, lO)] - d.f.rhop[ik]);
    if (k == kmx && kmx > k1x) {
      const int kb = kmx;
      const double eps = 2.220446049250313e-16;
      const double hplus = hk + eps, hminus = hk - eps;
      const double* rh = d.f.rhop;
      const double* hp = d.f.hp;
      bool co, cw;
      double rho_o, rho_w;
      if (hp[IX(d, kb, lO)] > hplus || hp[IX(d, kb, lO)] < hminus) {
        co = true;
        const double dz1 = 0.5 * (hp[IX(d, kb - 1, lO)] + hp[IX(d, kb, lO)]);
        const double dz2 = 0.5 * (hp[IX(d, kb - 1, lO)] + hk);
        rho_o = rh[IX(d, kb - 1, lO)] + (dz2 / dz1) * (rh[IX(d, kb, lO)] - rh[IX(d, kb - 1, lO)]);
      } else { co = false; rho_o = rh[IX(d, kb, lO)]; }
      if (hp[IX(d, kb, l)] > hplus || hp[IX(d, kb, l)] < hminus) {
        cw = true;
        const double dz1 = 0.5 * (hp[IX(d, kb - 1, l)] + hp[IX(d, kb, l)]);
        const double dz2 = 0.5 * (hp[IX(d, kb - 1, l)] + hk);
        rho_w = rh[IX(d, kb - 1, l)] + (dz2 / dz1) * (rh[IX(d, kb, l)] - rh[IX(d, kb - 1, l)]);
      } else { cw = false; rho_w = rh[IX(d, kb, l)]; }
      if (co || cw) hdrho = gdt * hk * (rho_o - rho_w);
    }
  }
  ex_out = ex;
  hdrho_out = hdrho;
  hkp_out = hkp;
}

// ------------------------------------------------------------------ cell kernel
template <int IEQ, int CL>
__global__ void __launch_bounds__(CW * CL, 768 / (CW * CL)) k_mom_cells(Dev d, const FaceMeta* __restrict__ meta, int ncols) {
  const int t = blockIdx.x * CW + threadIdx.x;
  if (t >= ncols) return;
  const CellCol C = cell_col<IEQ>(d, meta, t);
  if (C.k1x + (int)threadIdx.y > C.kmx) return;
  double* agA = (IEQ == 1) ? d.f.agx : d.f.agy;
  double* arA = (IEQ == 1) ? d.f.arx : d.f.ary;
  for (int k = C.k1x + threadIdx.y; k <= C.kmx; k += CL) {
    double ex, hdrho, hkp;
    mom_cell<IEQ>(d, C, k, ex, hdrho, hkp);
    const int ik = IX(d, k, C.l);
    agA[ik] = ex;
    arA[ik] = hdrho;
  }
}

// ------------------------------------------------------------------ column kernel
template <int IEQ, int NT>
__global__ void __launch_bounds__(NT, 768 / NT) k_mom_columns(Dev d, const FaceMeta* __restrict__ meta, int ncols) {
  constexpr int RD = (NT >= 256) ? 3 : 4;   // layers in flight (static shared memory under 48 KB)
  __shared__ double ring[RD][6][NT];        // [slot][input][thread]: a thread's slots are its own
  const int t = blockIdx.x * NT + threadIdx.x;
  if (t >= ncols) return;
  const bool X = (IEQ == 1);
  const int4 ma = __ldg(&meta[t].a), mb = __ldg(&meta[t].b);
  FaceCol F;
  F.l = ma.x; F.lE = ma.y; F.lW = ma.z; F.lN = ma.w; F.lS = mb.x; F.lX2 = mb.y; F.kmx = mb.z;
  F.lO = X ? F.lE : F.lN;
  F.k1x = X ? NB(d.s.k1u, F.l) : NB(d.s.k1v, F.l);
  const int l = F.l, lE = F.lE, lW = F.lW, lN = F.lN, lS = F.lS, lO = F.lO, kmx = F.kmx, k1x = F.k1x, lX2 = F.lX2;
  const int nw = kmx - k1x + 1;
  if (nw < 1) return;
  const int P = d.g.P;
  const double* __restrict__ huv = X ? d.f.hup : d.f.hvp;
  const double* __restrict__ uvpp = X ? d.f.upp : d.f.vpp;
  const double* __restrict__ uvpp_h = X ? d.f.uhpp : d.f.vhpp;
  const double* __restrict__ Av = d.f.Av;
  double* __restrict__ agA = X ? d.f.agx : d.f.agy;
  double* __restrict__ arA = X ? d.f.arx : d.f.ary;
  double* __restrict__ cc = d.scr;
  const double twodt1 = d.p.twodt * d.tz, tz = d.tz, theta = d.p.theta;
  const double gdt = X ? d.p.gdtdx : d.p.gdtdy;
  // depth-mean density (:1277 / :1470)
  double rsum = 0;
#pragma unroll 4
  for (int k = k1x; k <= kmx; ++k) rsum += 1000 + d.f.rhop[IX(d, k, l)];
  const double rhopx = rsum / nw;
  const double ws0 = rhopx * gdt * (d.s.spp[lO - 1] - d.s.spp[l - 1]);
  // wind drag coefficient cdw*rhoair*|Uair - usurf| (:1348-1360 / :1540-1552)
  double cwx;
  {
    const double ua = d.s.uair[l - 1], va = d.s.vair[l - 1];
    if (X) {
      const double usurf = d.f.up[IX(d, k1x, l)];
      const double vsurf = (d.f.vp[IX(d, NB(d.s.k1v, l), l)] + d.f.vp[IX(d, NB(d.s.k1v, lS), lS)] +
                            d.f.vp[IX(d, NB(d.s.k1v, lE), lE)] + d.f.vp[IX(d, NB(d.s.k1v, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((va - vsurf) * (va - vsurf) + (ua - usurf) * (ua - usurf));
    } else {
      const double vsurf = d.f.vp[IX(d, k1x, l)];
      const double usurf = (d.f.up[IX(d, NB(d.s.k1u, l), l)] + d.f.up[IX(d, NB(d.s.k1u, lW), lW)] +
                            d.f.up[IX(d, NB(d.s.k1u, lN), lN)] + d.f.up[IX(d, NB(d.s.k1u, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((ua - usurf) * (ua - usurf) + (va - vsurf) * (va - vsurf));
    }
  }
  // bottom stress (:1364-1369 / :1556-1561)
  double taub;
  {
    const double hkb = huv[IX(d, kmx, l)];
    double q;
    if (X) q = 0.25 * (d.f.vhpp[IX(d, kmx, lE)] + d.f.vhpp[IX(d, kmx, l)] + d.f.vhpp[IX(d, kmx, lS)] +
                       d.f.vhpp[IX(d, kmx, lX2)]);
    else q = 0.25 * (d.f.uhpp[IX(d, kmx, lN)] + d.f.uhpp[IX(d, kmx, lX2)] + d.f.uhpp[IX(d, kmx, lW)] +
                     d.f.uhpp[IX(d, kmx, l)]);
    const double own = uvpp_h[IX(d, kmx, l)];
    taub = d.p.cd * sqrt((own * own) + q * q) / (hkb * hkb);
  }
  const double taus_g = cwx / rhopx * (X ? d.s.uair[l - 1] : d.s.vair[l - 1]);
  const double taus_a = cwx / rhopx / huv[IX(d, k1x, l)];
  // forward sweep of trid with the matmom coefficients.  Iteration k consumes huv, uvpp and Av (both
  // columns) of layer k + 1 and the staged ex / increment of layer k; these six values are copied
  // into this thread's slots of a shared-memory ring by cp.async, RD layers ahead, so the copies of
  // several layers are in flight during the division chain without holding registers.
  double bcl = 0, c1p = 0, d1p = 0, e1p = 0, hdr_prev = 0;
  double hkm = huv[IX(d, k1x - 1, l)], hk = huv[IX(d, k1x, l)];
  double upm = uvpp[IX(d, k1x - 1, l)], upk = uvpp[IX(d, k1x, l)];
  const int dO = (lO - l);   // column offset of the other face column
  const int ik0 = IX(d, k1x, l);
  double avo = Av[ik0 + dO], avl = Av[ik0];   // Av of layer k (both columns); layer k + 1 is carried
  const int tid = threadIdx.x;
  auto issue = [&](int kk, int slot) {   // the six inputs of iteration kk into ring slot `slot`
    const int ikk = IX(d, kk, l);
    cp_async8(&ring[slot][0][tid], &huv[ikk + P]);
    cp_async8(&ring[slot][1][tid], &uvpp[ikk + P]);
    cp_async8(&ring[slot][2][tid], &Av[ikk + P + dO]);
    cp_async8(&ring[slot][3][tid], &Av[ikk + P]);
    cp_async8(&ring[slot][4][tid], &agA[ikk]);
    cp_async8(&ring[slot][5][tid], &arA[ikk]);
  };
#pragma unroll
  for (int j = 0; j < RD; ++j) {   // one commit group per layer (empty past the bottom)
    if (k1x + j <= kmx) issue(k1x + j, j);
    cp_async_commit();
  }
  // reciprocals shared between the coefficients: 1 / hk, 1 / hkm, 1 / (hkm + hk) (the previous
  // layer's 1 / (hk + hkp)), and 1 / rhopx; three divisions a layer instead of ten
  const double rrho = 1.0 / rhopx;
  double rhk = 1.0 / hk, rhkm = 0.0, rkm = 0.0;
  for (int k = k1x, slot = 0; k <= kmx; ++k, slot = (slot + 1 == RD) ? 0 : slot + 1) {
    const int ik = IX(d, k, l);
    cp_async_wait<RD - 1>();   // layer k's group has landed (this thread's own copies)
    const double hkp = ring[slot][0][tid], upp1 = ring[slot][1][tid];
    const double avop = ring[slot][2][tid], avlp = ring[slot][3][tid];
    const double ex = ring[slot][4][tid], hdr = ring[slot][5][tid];
    const double rkp = 1.0 / (hk + hkp), rhkp = 1.0 / hkp;
    const double Avk = (k > k1x) ? 0.5 * (avo + avl) : 0.0;
    const double Avkp = (k < kmx) ? 0.5 * (avop + avlp) : 0.0;
    double vdiff = 0.0;
    if (nw >= 2) {
      const double fk = (k > k1x) ? Avk * (upm - upk) * rkm : 0.0;
      const double fkp = (k < kmx) ? Avkp * (upk - upp1) * rkp : 0.0;
      vdiff = d.p.twodt * (fk - fkp) * 2. * (1. - theta);
    }
    double a1 = 0, a2, a3 = 0;
    if (nw == 1) {
      a2 = 1.0;
    } else {
      if (k < kmx) a3 = -twodt1 * Avkp * (rhkp * rkp) * 2. * theta;
      if (k > k1x) a1 = -twodt1 * Avk * (rhkm * rkm) * 2. * theta;
      a2 = 1.0 - (hkm * rhk) * a1 - (hkp * rhk) * a3;
    }
    if (d.p.ibc != 0) {
      if (k == k1x) bcl = hdr;
      else if (X) { const double aaux = hdr_prev + hdr; bcl = bcl + aaux; }
      else bcl = bcl + hdr_prev + hdr;
    }
    hdr_prev = hdr;
    const double hh = hk * rrho;
    const double vtz = vdiff * tz;
    double gg = ex - hh * (bcl + ws0) * tz + vtz;
    if (k == k1x) { gg = gg + taus_g * twodt1; a2 = a2 + taus_a * twodt1; }
    if (k == kmx) a2 = a2 + taub * twodt1;
    double c1v, d1v, e1v;
    if (k == k1x) {
      const double r = 1.0 / a2;
      c1v = a3 * r; d1v = gg * r; e1v = hh * r;
    } else {
      const double r = 1.0 / (a2 - a1 * c1p);
      c1v = a3 * r;
      d1v = (gg - a1 * d1p) * r;
      e1v = (hh - a1 * e1p) * r;
    }
    cc[ik] = c1v; agA[ik] = d1v; arA[ik] = e1v;
    // refill the slot with layer k + RD (its values are consumed: the stores above depend on them)
    if (k + RD <= kmx) issue(k + RD, slot);
    cp_async_commit();
    c1p = c1v; d1p = d1v; e1p = e1v;
    hkm = hk; hk = hkp;
    upm = upk; upk = upp1;
    avo = avop; avl = avlp;
    rhkm = rhk; rhk = rhkp; rkm = rkp;
  }
  // back substitution, summing the depth totals on the way up
  double d2 = d1p, e2 = e1p;
  double sg = d2, sr = e2;
#pragma unroll 4
  for (int k = kmx - 1; k >= k1x; --k) {
    const int ik = IX(d, k, l);
    const double c = cc[ik];
    d2 = agA[ik] - c * d2;
    e2 = arA[ik] - c * e2;
    agA[ik] = d2; arA[ik] = e2;
    sg += d2; sr += e2;
  }
  if (X) { d.s.eagx[l - 1] = sg; d.s.earx[l - 1] = sr; }
  else { d.s.eagy[l - 1] = sg; d.s.eary[l - 1] = sr; }
}

// ------------------------------------------------------------------ fused kernel
// k_mom_fused (one thread per face column): the cell and the column work of a face column in one
// pass down the column.  At layer k the thread forms the explicit term and the baroclinic increment
// exactly as k_mom_cells does and feeds them straight into the forward sweep of k_mom_columns, so
// neither goes through memory, and every input is read once.  The values that layer k needs and the
// layer above it did not (32 FP64 loads: the layer's own cells and its neighbours, and layer k + 1
// where the sweep or the vertical terms reach down) are copied by cp.async into this thread's slots
// of a shared-memory ring, RD layers ahead; the values shared with the layer above (thickness,
// velocity, wp, upp and Av of layer k, depth and density of layer k - 1 for the bottom-layer
// interpolation) are carried in registers.  Same expressions in the same order as the split
// kernels: the results are bit-identical to theirs.
namespace fz {
enum { HKP, HPL, HPO, A0, A1, A2, A3, B0, B1, B2, WDO, WDL, UVD, UVE, UVW, UVN, UVS, OWN, UPP1,
       HPPL, HPPE, HPPN, HPPW, HPPS, PN, PS, PE, PW, RHO_O, RHO_L, AVO, AVL, NIN };
}

template <int NT, int RD>
constexpr int fused_smem() { return RD * fz::NIN * NT * (int)sizeof(double); }

template <int IEQ, int NT, int RD, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_mom_fused(Dev d, const FaceMeta* __restrict__ meta, int ncols) {
  extern __shared__ double ring[];   // [RD][NIN][NT]: a thread's slots are its own
  const int t = blockIdx.x * NT + threadIdx.x;
  if (t >= ncols) return;
  const bool X = (IEQ == 1);
  const int4 ma = __ldg(&meta[t].a), mb = __ldg(&meta[t].b);
  const int l = ma.x, lE = ma.y, lW = ma.z, lN = ma.w, lS = mb.x, lX2 = mb.y, kmx = mb.z;
  const int lO = X ? lE : lN;
  const int* k1f = X ? d.s.k1u : d.s.k1v;
  const int k1x = NB(k1f, l);
  const int nw = kmx - k1x + 1;
  if (nw < 1) return;
  const int mW_last = mb.w, mS_last = __ldg(&meta[t].c.x);
  const int mW_first = mW_last >= 0 ? NB(k1f, lW) : 0;
  const int mS_first = mS_last >= 0 ? NB(k1f, lS) : 0;
  const double* __restrict__ huv = X ? d.f.hup : d.f.hvp;
  const double* __restrict__ huvpp = X ? d.f.hupp : d.f.hvpp;
  const double* __restrict__ uvpp_h = X ? d.f.uhpp : d.f.vhpp;
  const double* __restrict__ uvp = X ? d.f.up : d.f.vp;
  const double* __restrict__ uvpp = X ? d.f.upp : d.f.vpp;
  const double* __restrict__ vhp = d.f.vhp;
  const double* __restrict__ uhp = d.f.uhp;
  const double* __restrict__ wp = d.f.wp;
  const double* __restrict__ hp3 = d.f.hp;
  const double* __restrict__ rhop = d.f.rhop;
  const double* __restrict__ Av = d.f.Av;
  double* __restrict__ agA = X ? d.f.agx : d.f.agy;
  double* __restrict__ arA = X ? d.f.arx : d.f.ary;
  double* __restrict__ cc = d.scr;
  const double twodt1 = d.p.twodt * d.tz, tz = d.tz, theta = d.p.theta;
  const double gdt = X ? d.p.gdtdx : d.p.gdtdy;
  const bool ihd = d.p.ihd == 1, ibc = d.p.ibc != 0;
  const int P = d.g.P;
  const int dE = lE - l, dW = lW - l, dN = lN - l, dS = lS - l, dX2 = lX2 - l, dO = lO - l;
  const int tid = threadIdx.x;
  auto sp = [&](int s, int i) { return &ring[(s * fz::NIN + i) * NT + tid]; };
  auto issue = [&](int kk, int s) {   // the new inputs of layer kk into ring slot s
    const int ikk = IX(d, kk, l);
    cp_async8(sp(s, fz::HKP), &huv[ikk + P]);
    cp_async8(sp(s, fz::HPL), &hp3[ikk]);
    cp_async8(sp(s, fz::HPO), &hp3[ikk + dO]);
    if (X) {
      cp_async8(sp(s, fz::A0), &vhp[ikk + dE]);
      cp_async8(sp(s, fz::A1), &vhp[ikk]);
      cp_async8(sp(s, fz::A2), &vhp[ikk + dX2]);
      cp_async8(sp(s, fz::A3), &vhp[ikk + dS]);
      cp_async8(sp(s, fz::B0), &uhp[ikk + dE]);
      cp_async8(sp(s, fz::B1), &uhp[ikk]);
      cp_async8(sp(s, fz::B2), &uhp[ikk + dW]);
    } else {
      cp_async8(sp(s, fz::A0), &uhp[ikk + dN]);
      cp_async8(sp(s, fz::A1), &uhp[ikk]);
      cp_async8(sp(s, fz::A2), &uhp[ikk + dX2]);
      cp_async8(sp(s, fz::A3), &uhp[ikk + dW]);
      cp_async8(sp(s, fz::B0), &vhp[ikk + dN]);
      cp_async8(sp(s, fz::B1), &vhp[ikk]);
      cp_async8(sp(s, fz::B2), &vhp[ikk + dS]);
    }
    cp_async8(sp(s, fz::WDO), &wp[ikk + P + dO]);
    cp_async8(sp(s, fz::WDL), &wp[ikk + P]);
    cp_async8(sp(s, fz::UVD), &uvp[ikk + P]);
    cp_async8(sp(s, fz::UVE), &uvp[ikk + dE]);
    cp_async8(sp(s, fz::UVW), &uvp[ikk + dW]);
    cp_async8(sp(s, fz::UVN), &uvp[ikk + dN]);
    cp_async8(sp(s, fz::UVS), &uvp[ikk + dS]);
    cp_async8(sp(s, fz::OWN), &uvpp_h[ikk]);
    cp_async8(sp(s, fz::UPP1), &uvpp[ikk + P]);
    if (ihd) {
      cp_async8(sp(s, fz::HPPL), &huvpp[ikk]);
      cp_async8(sp(s, fz::HPPE), &huvpp[ikk + dE]);
      cp_async8(sp(s, fz::HPPN), &huvpp[ikk + dN]);
      cp_async8(sp(s, fz::HPPW), &huvpp[ikk + dW]);
      cp_async8(sp(s, fz::HPPS), &huvpp[ikk + dS]);
      cp_async8(sp(s, fz::PN), &uvpp[ikk + dN]);
      cp_async8(sp(s, fz::PS), &uvpp[ikk + dS]);
      cp_async8(sp(s, fz::PE), &uvpp[ikk + dE]);
      cp_async8(sp(s, fz::PW), &uvpp[ikk + dW]);
    }
    if (ibc) {
      cp_async8(sp(s, fz::RHO_O), &rhop[ikk + dO]);
      cp_async8(sp(s, fz::RHO_L), &rhop[ikk]);
    }
    cp_async8(sp(s, fz::AVO), &Av[ikk + P + dO]);
    cp_async8(sp(s, fz::AVL), &Av[ikk + P]);
  };
#pragma unroll
  for (int j = 0; j < RD; ++j) {   // one commit group per layer (empty past the bottom)
    if (k1x + j <= kmx) issue(k1x + j, j);
    cp_async_commit();
  }
  // column totals and surface / bottom terms while the first layers are in flight (as k_mom_columns)
  double rsum = 0;
#pragma unroll 4
  for (int k = k1x; k <= kmx; ++k) rsum += 1000 + rhop[IX(d, k, l)];
  const double rhopx = rsum / nw;
  const double ws0 = rhopx * gdt * (d.s.spp[lO - 1] - d.s.spp[l - 1]);
  double cwx;
  {
    const double ua = d.s.uair[l - 1], va = d.s.vair[l - 1];
    if (X) {
      const double usurf = d.f.up[IX(d, k1x, l)];
      const double vsurf = (d.f.vp[IX(d, NB(d.s.k1v, l), l)] + d.f.vp[IX(d, NB(d.s.k1v, lS), lS)] +
                            d.f.vp[IX(d, NB(d.s.k1v, lE), lE)] + d.f.vp[IX(d, NB(d.s.k1v, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((va - vsurf) * (va - vsurf) + (ua - usurf) * (ua - usurf));
    } else {
      const double vsurf = d.f.vp[IX(d, k1x, l)];
      const double usurf = (d.f.up[IX(d, NB(d.s.k1u, l), l)] + d.f.up[IX(d, NB(d.s.k1u, lW), lW)] +
                            d.f.up[IX(d, NB(d.s.k1u, lN), lN)] + d.f.up[IX(d, NB(d.s.k1u, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((ua - usurf) * (ua - usurf) + (va - vsurf) * (va - vsurf));
    }
  }
  double taub;
  {
    const double hkb = huv[IX(d, kmx, l)];
    double q;
    if (X) q = 0.25 * (d.f.vhpp[IX(d, kmx, lE)] + d.f.vhpp[IX(d, kmx, l)] + d.f.vhpp[IX(d, kmx, lS)] +
                       d.f.vhpp[IX(d, kmx, lX2)]);
    else q = 0.25 * (d.f.uhpp[IX(d, kmx, lN)] + d.f.uhpp[IX(d, kmx, lX2)] + d.f.uhpp[IX(d, kmx, lW)] +
                     d.f.uhpp[IX(d, kmx, l)]);
    const double own = uvpp_h[IX(d, kmx, l)];
    taub = d.p.cd * sqrt((own * own) + q * q) / (hkb * hkb);
  }
  const double taus_g = cwx / rhopx * (X ? d.s.uair[l - 1] : d.s.vair[l - 1]);
  const double taus_a = cwx / rhopx / huv[IX(d, k1x, l)];
  // carried values: layer k - 1 and k of the column, as the first iteration sees them
  const int ik0 = IX(d, k1x, l);
  double hkm = huv[ik0 - P], hk = huv[ik0];
  double upm = uvpp[ik0 - P], upk = uvpp[ik0];
  double uvU = uvp[ik0 - P], uc = uvp[ik0];
  double avo = Av[ik0 + dO], avl = Av[ik0];
  double wprev = 0.0;                                       // wp sum of layer k (the layer above's wD)
  double thq_prev = 0.0;                                    // hkm / (hkm + hk) of layer k
  double hpl_prev = 0.0, hpo_prev = 0.0, ro_prev = 0.0, rl_prev = 0.0;
  const double rrho = 1.0 / rhopx;
  double rhk = 1.0 / hk, rhkm = 0.0, rkm = 0.0;
  double bcl = 0, c1p = 0, d1p = 0, e1p = 0, hdr_prev = 0;
  for (int k = k1x, s = 0; k <= kmx; ++k, s = (s + 1 == RD) ? 0 : s + 1) {
    const int ik = IX(d, k, l);
    cp_async_wait<RD - 1>();   // layer k's group has landed (this thread's own copies)
    const double hkp = *sp(s, fz::HKP);
    const double hpl = *sp(s, fz::HPL), hpo = *sp(s, fz::HPO);
    // ---- explicit term (k_mom_cells)
    double cor, uE, uW, vN, vS;
    if (X) {
      const double vE = *sp(s, fz::A0), vC = *sp(s, fz::A1), vX = *sp(s, fz::A2), vSS = *sp(s, fz::A3);
      const double uEE = *sp(s, fz::B0), uC = *sp(s, fz::B1), uWW = *sp(s, fz::B2);
      cor = 0.25 * d.p.f * (vE + vC + vX + vSS);
      uE = uEE + uC;
      uW = uC + uWW;
      vN = vE + vC;
      vS = vX + vSS;
    } else {
      const double uN = *sp(s, fz::A0), uC = *sp(s, fz::A1), uX = *sp(s, fz::A2), uWW = *sp(s, fz::A3);
      const double vNN = *sp(s, fz::B0), vC = *sp(s, fz::B1), vSS = *sp(s, fz::B2);
      cor = 0.25 * d.p.f * (uN + uC + uX + uWW);
      uE = uN + uC;
      uW = uX + uWW;
      vN = vNN + vC;
      vS = vC + vSS;
    }
    const double wDraw = *sp(s, fz::WDO) + *sp(s, fz::WDL);
    double wU = wprev, wD = wDraw;
    const double uvD = *sp(s, fz::UVD);
    const double uvE = *sp(s, fz::UVE), uvW = *sp(s, fz::UVW), uvN = *sp(s, fz::UVN), uvS = *sp(s, fz::UVS);
    const double own_pp = *sp(s, fz::OWN);
    double hd = 0.0;
    if (ihd) {
      const double hppl = *sp(s, fz::HPPL), hppE = *sp(s, fz::HPPE), hppN = *sp(s, fz::HPPN);
      const double hppW = *sp(s, fz::HPPW), hppS = *sp(s, fz::HPPS);
      const double pc = upk, pN = *sp(s, fz::PN), pS = *sp(s, fz::PS), pE = *sp(s, fz::PE), pW = *sp(s, fz::PW);
      const double ax_l = d.p.Ax0 * fmin(hppE, hppl);
      const double ay_l = d.p.Ay0 * fmin(hppN, hppl);
      const double ax_w = face_coef(d, d.p.Ax0, hppl, hppW, lW, mW_first, mW_last, k);
      const double ay_s = face_coef(d, d.p.Ay0, hppl, hppS, lS, mS_first, mS_last, k);
      hd = (ay_l * (pN - pc) - ay_s * (pc - pS)) * d.p.rdydy + (ax_l * (pE - pc) - ax_w * (pc - pW)) * d.p.rdxdx;
    }
    // the interpolation weight hk / (hk + hkp), as the cell kernel forms it (a product with the
    // reciprocal the sweep needs too); it is the next layer's hkm / (hkm + hk), so it is carried down
    const double rkp = 1.0 / (hk + hkp);
    const double thq = hk * rkp;
    double ex;
    if (hpl <= ZERO || hpo <= ZERO) {
      ex = own_pp;
    } else {
      const double th_k = (k == k1x) ? 0.0 : thq_prev;
      const double th1_k = (k == k1x) ? 0.0 : 1. - th_k;
      const double th_kp = (k == kmx) ? 0.5 : thq;
      const double th1_kp = (k == kmx) ? 0.5 : 1. - th_kp;
      if (k == k1x) wU = 0.0;
      if (k == kmx) wD = 0.0;
      const double scE = uvE + uc, scW = uvW + uc;
      const double scN = uvN + uc, scS = uvS + uc;
      double adv = (uE * scE - uW * scW) * d.p.rfourdx + (vN * scN - vS * scS) * d.p.rfourdy;
      adv = adv + (wU * (th_k * uc + th1_k * uvU) - wD * (th_kp * uvD + th1_kp * uc)) / 2.;
      if (X) ex = own_pp - twodt1 * (adv * d.p.iadv - cor - hd);
      else ex = own_pp - twodt1 * (adv * d.p.iadv + cor - hd);
    }
    // ---- baroclinic increment, bottom layer via bclnc_km (layer k - 1 carried)
    double hdr = 0, ro = 0, rl = 0;
    if (ibc) {
      ro = *sp(s, fz::RHO_O);
      rl = *sp(s, fz::RHO_L);
      hdr = gdt * hk * (ro - rl);
      if (k == kmx && kmx > k1x) {
        const double eps = 2.220446049250313e-16;
        const double hplus = hk + eps, hminus = hk - eps;
        bool co, cw;
        double rho_o, rho_w;
        if (hpo > hplus || hpo < hminus) {
          co = true;
          const double dz1 = 0.5 * (hpo_prev + hpo);
          const double dz2 = 0.5 * (hpo_prev + hk);
          rho_o = ro_prev + (dz2 / dz1) * (ro - ro_prev);
        } else { co = false; rho_o = ro; }
        if (hpl > hplus || hpl < hminus) {
          cw = true;
          const double dz1 = 0.5 * (hpl_prev + hpl);
          const double dz2 = 0.5 * (hpl_prev + hk);
          rho_w = rl_prev + (dz2 / dz1) * (rl - rl_prev);
        } else { cw = false; rho_w = rl; }
        if (co || cw) hdr = gdt * hk * (rho_o - rho_w);
      }
    }
    // ---- forward sweep (k_mom_columns)
    const double upp1 = *sp(s, fz::UPP1);
    const double avop = *sp(s, fz::AVO), avlp = *sp(s, fz::AVL);
    const double rhkp = 1.0 / hkp;
    const double Avk = (k > k1x) ? 0.5 * (avo + avl) : 0.0;
    const double Avkp = (k < kmx) ? 0.5 * (avop + avlp) : 0.0;
    double vdiff = 0.0;
    if (nw >= 2) {
      const double fk = (k > k1x) ? Avk * (upm - upk) * rkm : 0.0;
      const double fkp = (k < kmx) ? Avkp * (upk - upp1) * rkp : 0.0;
      vdiff = d.p.twodt * (fk - fkp) * 2. * (1. - theta);
    }
    double a1 = 0, a2, a3 = 0;
    if (nw == 1) {
      a2 = 1.0;
    } else {
      if (k < kmx) a3 = -twodt1 * Avkp * (rhkp * rkp) * 2. * theta;
      if (k > k1x) a1 = -twodt1 * Avk * (rhkm * rkm) * 2. * theta;
      a2 = 1.0 - (hkm * rhk) * a1 - (hkp * rhk) * a3;
    }
    if (ibc) {
      if (k == k1x) bcl = hdr;
      else if (X) { const double aaux = hdr_prev + hdr; bcl = bcl + aaux; }
      else bcl = bcl + hdr_prev + hdr;
    }
    hdr_prev = hdr;
    const double hh = hk * rrho;
    const double vtz = vdiff * tz;
    double gg = ex - hh * (bcl + ws0) * tz + vtz;
    if (k == k1x) { gg = gg + taus_g * twodt1; a2 = a2 + taus_a * twodt1; }
    if (k == kmx) a2 = a2 + taub * twodt1;
    double c1v, d1v, e1v;
    if (k == k1x) {
      const double r = 1.0 / a2;
      c1v = a3 * r; d1v = gg * r; e1v = hh * r;
    } else {
      const double r = 1.0 / (a2 - a1 * c1p);
      c1v = a3 * r;
      d1v = (gg - a1 * d1p) * r;
      e1v = (hh - a1 * e1p) * r;
    }
    cc[ik] = c1v; agA[ik] = d1v; arA[ik] = e1v;
    // refill the slot with layer k + RD (its values are consumed: the stores above depend on them)
    if (k + RD <= kmx) issue(k + RD, s);
    cp_async_commit();
    c1p = c1v; d1p = d1v; e1p = e1v;
    hkm = hk; hk = hkp;
    upm = upk; upk = upp1;
    avo = avop; avl = avlp;
    rhkm = rhk; rhk = rhkp; rkm = rkp;
    uvU = uc; uc = uvD;
    wprev = wDraw;
    thq_prev = thq;
    hpl_prev = hpl; hpo_prev = hpo; ro_prev = ro; rl_prev = rl;
  }
  // back substitution, summing the depth totals on the way up
  double d2 = d1p, e2 = e1p;
  double sg = d2, sr = e2;
#pragma unroll 4
  for (int k = kmx - 1; k >= k1x; --k) {
    const int ik = IX(d, k, l);
    const double c = cc[ik];
    d2 = agA[ik] - c * d2;
    e2 = arA[ik] - c * e2;
    agA[ik] = d2; arA[ik] = e2;
    sg += d2; sr += e2;
  }
  if (X) { d.s.eagx[l - 1] = sg; d.s.earx[l - 1] = sr; }
  else { d.s.eagy[l - 1] = sg; d.s.eary[l - 1] = sr; }
}

// MINB: resident blocks per SM the register budget is sized for (the ring's shared memory allows
// 7 blocks of 64 threads, 3 of 128, 1 of 256)
template <int IEQ, int NT, int RD, int MINB>
void launch_fused(const Dev& d, const FaceMeta* cols, int ncols, cudaStream_t st) {
  k_mom_fused<IEQ, NT, RD, MINB><<<(ncols + NT - 1) / NT, NT, fused_smem<NT, RD>(), st>>>(d, cols, ncols);
}

template <int NT, int RD, int MINB>
int fused_attr() {
  const int b = fused_smem<NT, RD>();
  if (cudaFuncSetAttribute(k_mom_fused<1, NT, RD, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) != cudaSuccess ||
      cudaFuncSetAttribute(k_mom_fused<2, NT, RD, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) != cudaSuccess)
    return -1;
  return 0;
}

}  // namespace

int momentum_init(int km1) {
  (void)km1;   // the fused kernel's ring is sized by its threads, not by the column depth
  if (fused_attr<64, 2, 7>() || fused_attr<128, 2, 3>() || fused_attr<256, 2, 1>()) return -1;
  return 0;
}

template <int IEQ>
void launch_dir(const Dev& d, const FaceMeta* cols, int ncols, const Tune& tu, cudaStream_t st, const ObcDev* obc,
                int nobc) {
  if (tu.mom_cl == 1 && nobc == 0) {   // one pass per column (open boundaries need the split kernels)
    switch (tu.mom_nt) {
      case 64: launch_fused<IEQ, 64, 2, 7>(d, cols, ncols, st); break;
      case 256: launch_fused<IEQ, 256, 2, 1>(d, cols, ncols, st); break;
      default: launch_fused<IEQ, 128, 2, 3>(d, cols, ncols, st); break;
    }
    return;
  }
  const int g1 = (ncols + CW - 1) / CW;
  switch (tu.mom_cl) {
    case 2: k_mom_cells<IEQ, 2><<<g1, dim3(CW, 2), 0, st>>>(d, cols, ncols); break;
    case 4: k_mom_cells<IEQ, 4><<<g1, dim3(CW, 4), 0, st>>>(d, cols, ncols); break;
    default: k_mom_cells<IEQ, 8><<<g1, dim3(CW, 8), 0, st>>>(d, cols, ncols); break;
  }
  // open boundaries: MODexmom4openBCX/Y replace the explicit term of their face columns
  for (int b = 0; b < nobc; ++b) obc_exmom(d, obc[b], IEQ, st);
  switch (tu.mom_nt) {
    case 64: k_mom_columns<IEQ, 64><<<(ncols + 63) / 64, 64, 0, st>>>(d, cols, ncols); break;
    case 256: k_mom_columns<IEQ, 256><<<(ncols + 255) / 256, 256, 0, st>>>(d, cols, ncols); break;
    default: k_mom_columns<IEQ, 128><<<(ncols + 127) / 128, 128, 0, st>>>(d, cols, ncols); break;
  }
}

void launch_momentum(const Dev& d, int ieq, const FaceMeta* cols, int ncols, const Tune& tu, cudaStream_t st,
                     const ObcDev* obc, int nobc) {
  if (ncols <= 0) return;
  if (ieq == 1) launch_dir<1>(d, cols, ncols, tu, st, obc, nobc);
  else launch_dir<2>(d, cols, ncols, tu, st, obc, nobc);
}

}  // namespace si3d
