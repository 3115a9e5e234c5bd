// Momentum stage: exmom + matmom + trid fused into one column kernel per direction.
//
// Reference: exmom (si3d_procedures.f90:578-1173), matmom (:1176-1630), bclnc_km (:1633-1746),
// trid (:3210-3289).  One thread owns one u (v) face column l — the columns whose east (north)
// neighbour is wet, i.e. the reference's id_columnCE (id_columnCN) list — and walks down the
// wet layers k1x..kmx.  Threads of a warp hold 32 consecutive columns, so every per-layer load
// of a layer-major field is a coalesced 256-byte access; the neighbour columns lE/lW (another
// i-strip) are contiguous runs as well.  The explicit term ex(k) is never stored: it is formed in
// registers and fed straight into the tridiagonal assembly and the forward Thomas sweep.  The
// sweep keeps c1 in the layer-major scratch and d1/e1 in agx/arx, which the backward sweep
// overwrites with the solution (the reference's ag/ar) — so the only 3-D outputs are agx/arx.
#include "common.cuh"
#include "kernels.h"

namespace si3d {

namespace {

// Horizontal-diffusion coefficient of a neighbouring face column m at layer k
// (haxpp/haypp as rebuilt by exmom each call, :623-681 / :962-1018): zero outside that
// column's wet face layers or when its face is closed.
__device__ __forceinline__ double face_coef(const Dev& d, const double* hpp3, double A, int m, int kfirst,
                                            int klast, int other, int k) {
  if (m == d.g.lm1 || k < kfirst || k > klast) return 0.0;
  return A * fmin(hpp3[IX(d, k, other)], hpp3[IX(d, k, m)]);
}

template <int IEQ>
__global__ void __launch_bounds__(128) k_momentum(Dev d, const int* __restrict__ cols, int ncols) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncols) return;
  const int l = cols[t];
  const Grid& g = d.g;
  const int lm1 = g.lm1;
  const bool X = (IEQ == 1);
  const int lE = NB(g.lEC, l), lW = NB(g.lWC, l), lN = NB(g.lNC, l), lS = NB(g.lSC, l);
  const int lO = X ? lE : lN;                 // the column across the face
  const int kmx = min(NB(g.kmz, lO), NB(g.kmz, l));
  const int k1x = X ? NB(d.s.k1u, l) : NB(d.s.k1v, l);
  const int nw = kmx - k1x + 1;
  if (nw < 1) return;   // the reference CYCLEs and keeps agx/eagx from the previous call

  // face-aligned 3-D fields
  const double* huv = X ? d.f.hup : d.f.hvp;     // hup / hvp
  const double* huvpp = X ? d.f.hupp : d.f.hvpp;
  const double* uvpp_h = X ? d.f.uhpp : d.f.vhpp;  // uhpp / vhpp (flux, own direction)
  const double* uvp = X ? d.f.up : d.f.vp;
  const double* uvpp = X ? d.f.upp : d.f.vpp;
  double* agA = X ? d.f.agx : d.f.agy;
  double* arA = X ? d.f.arx : d.f.ary;
  double* c1s = d.scr;
  const double twodt1 = d.p.twodt * d.tz, tz = d.tz, theta = d.p.theta;
  const double gdt = X ? d.p.gdtdx : d.p.gdtdy;

  // neighbour face columns whose diffusion coefficients enter the stencil
  int mW_first = 0, mW_last = -1, mS_first = 0, mS_last = -1;
  if (X) {
    if (lW != lm1) { mW_first = NB(d.s.k1u, lW); mW_last = min(NB(g.kmz, l), NB(g.kmz, lW)); }
    if (lS != lm1 && NB(g.lEC, lS) != lm1) {
      mS_first = NB(d.s.k1u, lS); mS_last = min(NB(g.kmz, NB(g.lEC, lS)), NB(g.kmz, lS));
    }
  } else {
    if (lS != lm1) { mS_first = NB(d.s.k1v, lS); mS_last = min(NB(g.kmz, l), NB(g.kmz, lS)); }
    if (lW != lm1 && NB(g.lNC, lW) != lm1) {
      mW_first = NB(d.s.k1v, lW); mW_last = min(NB(g.kmz, NB(g.lNC, lW)), NB(g.kmz, lW));
    }
  }
  const int lX2 = X ? NB(g.lSC, lE) : NB(g.lWC, lN);   // lSC(lEC(l)) / lWC(lNC(l))

  // pass 1: depth-mean density of the column (:1277 / :1470)
  double rsum = 0;
  for (int k = k1x; k <= kmx; ++k) rsum += 1000 + d.f.rhop[IX(d, k, l)];
  const double rhopx = rsum / nw;
  const double ws0 = rhopx * gdt * (d.s.spp[lO - 1] - d.s.spp[l - 1]);

  // wind stress at the surface face (:1348-1360 / :1540-1552)
  double taus_g, taus_a;
  {
    const double ua = d.s.uair[l - 1], va = d.s.vair[l - 1];
    double cwx;
    if (X) {
      const double usurf = d.f.up[IX(d, k1x, l)];
      const double vsurf = (d.f.vp[IX(d, NB(d.s.k1v, l), l)] + d.f.vp[IX(d, NB(d.s.k1v, lS), lS)] +
                            d.f.vp[IX(d, NB(d.s.k1v, lE), lE)] + d.f.vp[IX(d, NB(d.s.k1v, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((va - vsurf) * (va - vsurf) + (ua - usurf) * (ua - usurf));
      taus_g = cwx / rhopx * ua;
    } else {
      const double vsurf = d.f.vp[IX(d, k1x, l)];
      const double usurf = (d.f.up[IX(d, NB(d.s.k1u, l), l)] + d.f.up[IX(d, NB(d.s.k1u, lW), lW)] +
                            d.f.up[IX(d, NB(d.s.k1u, lN), lN)] + d.f.up[IX(d, NB(d.s.k1u, lX2), lX2)]) / 4.;
      cwx = d.s.cdw[l - 1] * RHOAIR * sqrt((ua - usurf) * (ua - usurf) + (va - vsurf) * (va - vsurf));
      taus_g = cwx / rhopx * va;
    }
    taus_a = cwx / rhopx / huv[IX(d, k1x, l)];
  }
  // bottom stress at the deepest face (:1364-1369 / :1556-1561)
  double taub;
  {
    double q;
    if (X) q = 0.25 * (d.f.vhpp[IX(d, kmx, lE)] + d.f.vhpp[IX(d, kmx, l)] + d.f.vhpp[IX(d, kmx, lS)] +
                       d.f.vhpp[IX(d, kmx, lX2)]);
    else q = 0.25 * (d.f.uhpp[IX(d, kmx, lN)] + d.f.uhpp[IX(d, kmx, lX2)] + d.f.uhpp[IX(d, kmx, lW)] +
                     d.f.uhpp[IX(d, kmx, l)]);
    const double own = uvpp_h[IX(d, kmx, l)];
    const double hb = huv[IX(d, kmx, l)];
    taub = d.p.cd * sqrt((own * own) + q * q) / (hb * hb);
  }
  // bottom-layer baroclinic term on a horizontal plane (bclnc_km)
  double hdrho_bottom = 0;
  bool bottom_mod = false;
  if (d.p.ibc != 0 && kmx > k1x) {
    const int kb = kmx;
    const double eps = 2.220446049250313e-16;
    const double hb = huv[IX(d, kb, l)];
    const double hplus = hb + eps, hminus = hb - eps;
    const double* rh = d.f.rhop;
    const double* hp = d.f.hp;
    bool co, cw;
    double rho_o, rho_w;
    if (hp[IX(d, kb, lO)] > hplus || hp[IX(d, kb, lO)] < hminus) {
      co = true;
      const double dz1 = 0.5 * (hp[IX(d, kb - 1, lO)] + hp[IX(d, kb, lO)]);
      const double dz2 = 0.5 * (hp[IX(d, kb - 1, lO)] + hb);
      rho_o = rh[IX(d, kb - 1, lO)] + (dz2 / dz1) * (rh[IX(d, kb, lO)] - rh[IX(d, kb - 1, lO)]);
    } else { co = false; rho_o = rh[IX(d, kb, lO)]; }
    if (hp[IX(d, kb, l)] > hplus || hp[IX(d, kb, l)] < hminus) {
      cw = true;
      const double dz1 = 0.5 * (hp[IX(d, kb - 1, l)] + hp[IX(d, kb, l)]);
      const double dz2 = 0.5 * (hp[IX(d, kb - 1, l)] + hb);
      rho_w = rh[IX(d, kb - 1, l)] + (dz2 / dz1) * (rh[IX(d, kb, l)] - rh[IX(d, kb - 1, l)]);
    } else { cw = false; rho_w = rh[IX(d, kb, l)]; }
    if (co || cw) { bottom_mod = true; hdrho_bottom = gdt * hb * (rho_o - rho_w); }
  }

  // pass 2: march down the face column building ex, gg, hh, aa and the forward sweep
  double bcl = 0, hdrho_prev = 0, c1_prev = 0, d1_prev = 0, e1_prev = 0;
  for (int k = k1x; k <= kmx; ++k) {
    const size_t ik = IX(d, k, l);
    const double hk = huv[ik];
    const double hkm = huv[IX(d, k - 1, l)];
    const double hkp = huv[IX(d, k + 1, l)];
    // ---- explicit term (exmom)
    double ex;
    const double hpl = d.f.hp[ik], hpo = d.f.hp[IX(d, k, lO)];
    if (hpl <= ZERO || hpo <= ZERO) {
      ex = uvpp_h[ik];
    } else {
      const double th_k = (k == k1x) ? 0.0 : hkm / (hkm + hk);
      const double th1_k = (k == k1x) ? 0.0 : 1. - th_k;
      const double th_kp = (k == kmx) ? 0.5 : hk / (hk + hkp);
      const double th1_kp = (k == kmx) ? 0.5 : 1. - th_kp;
      double cor, uE, uW, vN, vS, wU, wD;
      if (X) {
        const double* vhp = d.f.vhp;
        const double* uhp = d.f.uhp;
        cor = 0.25 * d.p.f * (vhp[IX(d, k, lE)] + vhp[ik] + vhp[IX(d, k, lX2)] + vhp[IX(d, k, lS)]);
        uE = uhp[IX(d, k, lE)] + uhp[ik];
        uW = uhp[ik] + uhp[IX(d, k, lW)];
        vN = vhp[IX(d, k, lE)] + vhp[ik];
        vS = vhp[IX(d, k, lX2)] + vhp[IX(d, k, lS)];
        wU = d.f.wp[IX(d, k, lE)] + d.f.wp[ik];
        wD = d.f.wp[IX(d, k + 1, lE)] + d.f.wp[IX(d, k + 1, l)];
      } else {
        const double* vhp = d.f.vhp;
        const double* uhp = d.f.uhp;
        cor = 0.25 * d.p.f * (uhp[IX(d, k, lN)] + uhp[ik] + uhp[IX(d, k, lX2)] + uhp[IX(d, k, lW)]);
        uE = uhp[IX(d, k, lN)] + uhp[ik];
        uW = uhp[IX(d, k, lX2)] + uhp[IX(d, k, lW)];
        vN = vhp[IX(d, k, lN)] + vhp[ik];
        vS = vhp[ik] + vhp[IX(d, k, lS)];
        wU = d.f.wp[IX(d, k, lN)] + d.f.wp[ik];
        wD = d.f.wp[IX(d, k + 1, lN)] + d.f.wp[IX(d, k + 1, l)];
      }
      if (k == k1x) wU = 0.0;
      if (k == kmx) wD = 0.0;
      const double uc = uvp[ik];
      const double scE = uvp[IX(d, k, lE)] + uc, scW = uvp[IX(d, k, lW)] + uc;
      const double scN = uvp[IX(d, k, lN)] + uc, scS = uvp[IX(d, k, lS)] + uc;
      double adv = (uE * scE - uW * scW) / d.p.fourdx + (vN * scN - vS * scS) / d.p.fourdy;
      adv = adv + (wU * (th_k * uc + th1_k * uvp[IX(d, k - 1, l)]) -
                   wD * (th_kp * uvp[IX(d, k + 1, l)] + th1_kp * uc)) / 2.;
      double hd = 0.0;
      if (d.p.ihd == 1) {
        const double hppl = huvpp[ik];
        double ax_l, ay_l, ax_w, ay_s;
        if (X) {
          ax_l = d.p.Ax0 * fmin(huvpp[IX(d, k, lE)], hppl);
          ay_l = d.p.Ay0 * fmin(huvpp[IX(d, k, lN)], hppl);
          ax_w = face_coef(d, huvpp, d.p.Ax0, lW, mW_first, mW_last, l, k);
          ay_s = face_coef(d, huvpp, d.p.Ay0, lS, mS_first, mS_last, l, k);
        } else {
          ay_l = d.p.Ay0 * fmin(huvpp[IX(d, k, lN)], hppl);
          ax_l = d.p.Ax0 * fmin(huvpp[IX(d, k, lE)], hppl);
          ay_s = face_coef(d, huvpp, d.p.Ay0, lS, mS_first, mS_last, l, k);
          ax_w = face_coef(d, huvpp, d.p.Ax0, lW, mW_first, mW_last, l, k);
        }
        const double pc = uvpp[ik];
        hd = (ay_l * (uvpp[IX(d, k, lN)] - pc) - ay_s * (pc - uvpp[IX(d, k, lS)])) / d.p.dydy +
             (ax_l * (uvpp[IX(d, k, lE)] - pc) - ax_w * (pc - uvpp[IX(d, k, lW)])) / d.p.dxdx;
      }
      if (X) ex = uvpp_h[ik] - twodt1 * (adv * d.p.iadv - cor - hd);
      else ex = uvpp_h[ik] - twodt1 * (adv * d.p.iadv + cor - hd);
    }
    // ---- baroclinic cumulative sum (:1283-1301 / :1475-1491)
    double hdrho = 0;
    if (d.p.ibc != 0) {
      hdrho = gdt * hk * (d.f.rhop[IX(d, k, lO)] - d.f.rhop[ik]);
      if (k == kmx && bottom_mod) hdrho = hdrho_bottom;
      if (k == k1x) bcl = hdrho;
      else if (X) { const double aaux = hdrho_prev + hdrho; bcl = bcl + aaux; }
      else bcl = bcl + hdrho_prev + hdrho;
      hdrho_prev = hdrho;
    }
    // ---- explicit vertical diffusion (:1304-1317)
    const double Avk = (k > k1x) ? 0.5 * (d.f.Av[IX(d, k, lO)] + d.f.Av[ik]) : 0.0;
    const double Avkp = (k < kmx) ? 0.5 * (d.f.Av[IX(d, k + 1, lO)] + d.f.Av[IX(d, k + 1, l)]) : 0.0;
    double vdiff = 0.0;
    if (nw >= 2) {
      const double fk = (k > k1x) ? Avk * (uvpp[IX(d, k - 1, l)] - uvpp[ik]) / (hkm + hk) : 0.0;
      const double fkp = (k < kmx) ? Avkp * (uvpp[ik] - uvpp[IX(d, k + 1, l)]) / (hk + hkp) : 0.0;
      vdiff = d.p.twodt * (fk - fkp) * 2. * (1. - theta);
    }
    const double hh = hk / rhopx;
    double gg = ex - hh * (bcl + ws0) * tz + vdiff * tz;
    double a1 = 0, a2, a3 = 0;
    if (nw == 1) {
      a2 = 1.0;
    } else {
      if (k < kmx) a3 = -twodt1 * Avkp / (hkp * (hk + hkp)) * 2. * theta;
      if (k > k1x) a1 = -twodt1 * Avk / (hkm * (hkm + hk)) * 2. * theta;
      a2 = 1.0 - (hkm / hk) * a1 - (hkp / hk) * a3;
    }
    if (k == k1x) { gg = gg + taus_g * twodt1; a2 = a2 + taus_a * twodt1; }
    if (k == kmx) a2 = a2 + taub * twodt1;
    // ---- forward sweep of trid
    double c1v, d1v, e1v;
    if (k == k1x) {
      c1v = a3 / a2; d1v = gg / a2; e1v = hh / a2;
    } else {
      const double den = a2 - a1 * c1_prev;
      c1v = a3 / den;
      d1v = (gg - a1 * d1_prev) / den;
      e1v = (hh - a1 * e1_prev) / den;
    }
    c1s[ik] = c1v; agA[ik] = d1v; arA[ik] = e1v;
    c1_prev = c1v; d1_prev = d1v; e1_prev = e1v;
  }
  // pass 3: backward sweep and depth sums (:1424-1428)
  double d2 = d1_prev, e2 = e1_prev;
  double sg = 0, sr = 0;
  for (int k = kmx - 1; k >= k1x; --k) {
    const size_t ik = IX(d, k, l);
    const double c = c1s[ik];
    d2 = agA[ik] - c * d2;
    e2 = arA[ik] - c * e2;
    agA[ik] = d2; arA[ik] = e2;
  }
  for (int k = k1x; k <= kmx; ++k) sg += agA[IX(d, k, l)];
  for (int k = k1x; k <= kmx; ++k) sr += arA[IX(d, k, l)];
  if (X) { d.s.eagx[l - 1] = sg; d.s.earx[l - 1] = sr; }
  else { d.s.eagy[l - 1] = sg; d.s.eary[l - 1] = sr; }
}

}  // namespace

void launch_momentum(const Dev& d, int ieq, const int* cols, int ncols, cudaStream_t st) {
  if (ncols <= 0) return;
  const int B = 128, G = (ncols + B - 1) / B;
  if (ieq == 1) k_momentum<1><<<G, B, 0, st>>>(d, cols, ncols);
  else k_momentum<2><<<G, B, 0, st>>>(d, cols, ncols);
}

}  // namespace si3d
