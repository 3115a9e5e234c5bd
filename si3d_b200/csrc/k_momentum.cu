// Momentum stage: exmom + matmom + trid fused into one kernel per direction.
//
// Reference: exmom (si3d_procedures.f90:578-1173), matmom (:1176-1630), bclnc_km (:1633-1746),
// trid (:3210-3289).  The work items are the u (v) face columns l whose east (north) neighbour is
// wet — the reference's id_columnCE (id_columnCN) list.
//
// One block owns a tile of MC = 16 consecutive face columns and runs two phases:
//   phase 1 (all 256 threads, cell-parallel): thread (sub, c) handles column c at layers
//     k1x+sub, k1x+sub+16, ...; it forms the explicit term ex(k) and every per-cell input of the
//     tridiagonal system (a1, a3, the diagonal before the boundary terms, vdiff*tz, the baroclinic
//     increment, the face thickness, 1000+rhop) and stages them in shared memory.  Layer-major
//     fields make each access a 128-byte run of 16 consecutive columns; the 16 layers in flight per
//     column give the memory-level parallelism a one-thread-per-column walk lacks.
//   phase 2 (one thread per column): the sequential parts — the depth-mean density, the
//     baroclinic prefix sum, the boundary terms and the Thomas forward/backward sweeps of trid —
//     from shared memory, in the reference's exact operation order.
// Only agx/arx (ag/ar) and eagx/earx are written to HBM; ex is never stored.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace si3d {

namespace {

constexpr int MC = 16;       // face columns per block
constexpr int MT = 256;      // threads per block
constexpr int NARR = 8;      // staged per-cell arrays
enum { A_EX, A_VTZ, A_HDR, A_HK, A_A1, A_A2, A_A3, A_RHO };

// Horizontal-diffusion coefficient of a neighbouring face column m at layer k
// (haxpp/haypp as rebuilt by exmom each call, :623-681 / :962-1018): zero outside that
// column's wet face layers or when its face is closed.
__device__ __forceinline__ double face_coef(const Dev& d, const double* hpp3, double A, int m, int kfirst,
                                            int klast, int other, int k) {
  if (m == d.g.lm1 || k < kfirst || k > klast) return 0.0;
  return A * fmin(hpp3[IX(d, k, other)], hpp3[IX(d, k, m)]);
}

template <int IEQ>
__global__ void __launch_bounds__(MT, 3) k_momentum(Dev d, const int* __restrict__ cols, int ncols) {
  extern __shared__ double sm[];
  __shared__ double s_cw[MC], s_taub[MC];
  const int km1 = d.g.km1;
  auto S = [&](int a, int k, int c) -> double& { return sm[((size_t)a * km1 + (k - 1)) * MC + c]; };

  const int c = threadIdx.x % MC, sub = threadIdx.x / MC;
  const int t = blockIdx.x * MC + c;
  const bool active = t < ncols;
  const Grid& g = d.g;
  const int lm1 = g.lm1;
  const bool X = (IEQ == 1);
  int l = 1, lE = 1, lW = 1, lN = 1, lS = 1, lO = 1, kmx = 0, k1x = 1, lX2 = 1;
  if (active) {
    l = cols[t];
    lE = NB(g.lEC, l); lW = NB(g.lWC, l); lN = NB(g.lNC, l); lS = NB(g.lSC, l);
    lO = X ? lE : lN;
    kmx = min(NB(g.kmz, lO), NB(g.kmz, l));
    k1x = X ? NB(d.s.k1u, l) : NB(d.s.k1v, l);
    lX2 = X ? NB(g.lSC, lE) : NB(g.lWC, lN);   // lSC(lEC(l)) / lWC(lNC(l))
  }
  const int nw = kmx - k1x + 1;

  const double* huv = X ? d.f.hup : d.f.hvp;
  const double* huvpp = X ? d.f.hupp : d.f.hvpp;
  const double* uvpp_h = X ? d.f.uhpp : d.f.vhpp;
  const double* uvp = X ? d.f.up : d.f.vp;
  const double* uvpp = X ? d.f.upp : d.f.vpp;
  const double twodt1 = d.p.twodt * d.tz, tz = d.tz, theta = d.p.theta;
  const double gdt = X ? d.p.gdtdx : d.p.gdtdy;

  // ---------------------------------------------------------------- phase 1 (cell-parallel)
  if (active && nw >= 1) {
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
    // bottom-layer baroclinic term on a horizontal plane (bclnc_km), used by the kmx thread
    for (int k = k1x + sub; k <= kmx; k += MT / MC) {
      const int ik = IX(d, k, l);
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
        const double* vhp = d.f.vhp;
        const double* uhp = d.f.uhp;
        if (X) {
          cor = 0.25 * d.p.f * (vhp[IX(d, k, lE)] + vhp[ik] + vhp[IX(d, k, lX2)] + vhp[IX(d, k, lS)]);
          uE = uhp[IX(d, k, lE)] + uhp[ik];
          uW = uhp[ik] + uhp[IX(d, k, lW)];
          vN = vhp[IX(d, k, lE)] + vhp[ik];
          vS = vhp[IX(d, k, lX2)] + vhp[IX(d, k, lS)];
          wU = d.f.wp[IX(d, k, lE)] + d.f.wp[ik];
          wD = d.f.wp[IX(d, k + 1, lE)] + d.f.wp[IX(d, k + 1, l)];
        } else {
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
          const double ax_l = d.p.Ax0 * fmin(huvpp[IX(d, k, lE)], hppl);
          const double ay_l = d.p.Ay0 * fmin(huvpp[IX(d, k, lN)], hppl);
          const double ax_w = face_coef(d, huvpp, d.p.Ax0, lW, mW_first, mW_last, l, k);
          const double ay_s = face_coef(d, huvpp, d.p.Ay0, lS, mS_first, mS_last, l, k);
          const double pc = uvpp[ik];
          hd = (ay_l * (uvpp[IX(d, k, lN)] - pc) - ay_s * (pc - uvpp[IX(d, k, lS)])) / d.p.dydy +
               (ax_l * (uvpp[IX(d, k, lE)] - pc) - ax_w * (pc - uvpp[IX(d, k, lW)])) / d.p.dxdx;
        }
        if (X) ex = uvpp_h[ik] - twodt1 * (adv * d.p.iadv - cor - hd);
        else ex = uvpp_h[ik] - twodt1 * (adv * d.p.iadv + cor - hd);
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
      // ---- explicit vertical diffusion (:1304-1317) and the tridiagonal coefficients
      const double Avk = (k > k1x) ? 0.5 * (d.f.Av[IX(d, k, lO)] + d.f.Av[ik]) : 0.0;
      const double Avkp = (k < kmx) ? 0.5 * (d.f.Av[IX(d, k + 1, lO)] + d.f.Av[IX(d, k + 1, l)]) : 0.0;
      double vdiff = 0.0;
      if (nw >= 2) {
        const double fk = (k > k1x) ? Avk * (uvpp[IX(d, k - 1, l)] - uvpp[ik]) / (hkm + hk) : 0.0;
        const double fkp = (k < kmx) ? Avkp * (uvpp[ik] - uvpp[IX(d, k + 1, l)]) / (hk + hkp) : 0.0;
        vdiff = d.p.twodt * (fk - fkp) * 2. * (1. - theta);
      }
      double a1 = 0, a2, a3 = 0;
      if (nw == 1) {
        a2 = 1.0;
      } else {
        if (k < kmx) a3 = -twodt1 * Avkp / (hkp * (hk + hkp)) * 2. * theta;
        if (k > k1x) a1 = -twodt1 * Avk / (hkm * (hkm + hk)) * 2. * theta;
        a2 = 1.0 - (hkm / hk) * a1 - (hkp / hk) * a3;
      }
      S(A_EX, k, c) = ex;
      S(A_VTZ, k, c) = vdiff * tz;
      S(A_HDR, k, c) = hdrho;
      S(A_HK, k, c) = hk;
      S(A_A1, k, c) = a1;
      S(A_A2, k, c) = a2;
      S(A_A3, k, c) = a3;
      S(A_RHO, k, c) = 1000 + d.f.rhop[ik];
      // per-column boundary terms that do not depend on the depth-mean density
      if (k == k1x) {   // wind drag coefficient cdw*rhoair*|Uair - usurf| (:1348-1360 / :1540-1552)
        const double ua = d.s.uair[l - 1], va = d.s.vair[l - 1];
        if (X) {
          const double usurf = d.f.up[IX(d, k1x, l)];
          const double vsurf = (d.f.vp[IX(d, NB(d.s.k1v, l), l)] + d.f.vp[IX(d, NB(d.s.k1v, lS), lS)] +
                                d.f.vp[IX(d, NB(d.s.k1v, lE), lE)] + d.f.vp[IX(d, NB(d.s.k1v, lX2), lX2)]) / 4.;
          s_cw[c] = d.s.cdw[l - 1] * RHOAIR * sqrt((va - vsurf) * (va - vsurf) + (ua - usurf) * (ua - usurf));
        } else {
          const double vsurf = d.f.vp[IX(d, k1x, l)];
          const double usurf = (d.f.up[IX(d, NB(d.s.k1u, l), l)] + d.f.up[IX(d, NB(d.s.k1u, lW), lW)] +
                                d.f.up[IX(d, NB(d.s.k1u, lN), lN)] + d.f.up[IX(d, NB(d.s.k1u, lX2), lX2)]) / 4.;
          s_cw[c] = d.s.cdw[l - 1] * RHOAIR * sqrt((ua - usurf) * (ua - usurf) + (va - vsurf) * (va - vsurf));
        }
      }
      if (k == kmx) {   // bottom stress (:1364-1369 / :1556-1561)
        double q;
        if (X) q = 0.25 * (d.f.vhpp[IX(d, kmx, lE)] + d.f.vhpp[IX(d, kmx, l)] + d.f.vhpp[IX(d, kmx, lS)] +
                           d.f.vhpp[IX(d, kmx, lX2)]);
        else q = 0.25 * (d.f.uhpp[IX(d, kmx, lN)] + d.f.uhpp[IX(d, kmx, lX2)] + d.f.uhpp[IX(d, kmx, lW)] +
                         d.f.uhpp[IX(d, kmx, l)]);
        const double own = uvpp_h[ik];
        s_taub[c] = d.p.cd * sqrt((own * own) + q * q) / (hk * hk);
      }
    }
  }
  __syncthreads();
  // ---------------------------------------------------------------- phase 2 (per column)
  if (sub != 0 || !active || nw < 1) return;
  double rsum = 0;
  for (int k = k1x; k <= kmx; ++k) rsum += S(A_RHO, k, c);
  const double rhopx = rsum / nw;
  const double ws0 = rhopx * gdt * (d.s.spp[lO - 1] - d.s.spp[l - 1]);
  const double cwx = s_cw[c];
  const double taus_g = cwx / rhopx * (X ? d.s.uair[l - 1] : d.s.vair[l - 1]);
  const double taus_a = cwx / rhopx / S(A_HK, k1x, c);
  const double taub = s_taub[c];
  double bcl = 0, c1p = 0, d1p = 0, e1p = 0;
  for (int k = k1x; k <= kmx; ++k) {
    if (d.p.ibc != 0) {
      const double hdr = S(A_HDR, k, c);
      if (k == k1x) bcl = hdr;
      else if (X) { const double aaux = S(A_HDR, k - 1, c) + hdr; bcl = bcl + aaux; }
      else bcl = bcl + S(A_HDR, k - 1, c) + hdr;
    }
    const double hh = S(A_HK, k, c) / rhopx;
    double gg = S(A_EX, k, c) - hh * (bcl + ws0) * tz + S(A_VTZ, k, c);
    double a2 = S(A_A2, k, c);
    const double a1 = S(A_A1, k, c), a3 = S(A_A3, k, c);
    if (k == k1x) { gg = gg + taus_g * twodt1; a2 = a2 + taus_a * twodt1; }
    if (k == kmx) a2 = a2 + taub * twodt1;
    double c1v, d1v, e1v;
    if (k == k1x) {
      c1v = a3 / a2; d1v = gg / a2; e1v = hh / a2;
    } else {
      const double den = a2 - a1 * c1p;
      c1v = a3 / den;
      d1v = (gg - a1 * d1p) / den;
      e1v = (hh - a1 * e1p) / den;
    }
    S(A_A3, k, c) = c1v; S(A_EX, k, c) = d1v; S(A_VTZ, k, c) = e1v;
    c1p = c1v; d1p = d1v; e1p = e1v;
  }
  double* agA = X ? d.f.agx : d.f.agy;
  double* arA = X ? d.f.arx : d.f.ary;
  double d2 = d1p, e2 = e1p;
  agA[IX(d, kmx, l)] = d2; arA[IX(d, kmx, l)] = e2;
  S(A_EX, kmx, c) = d2; S(A_VTZ, kmx, c) = e2;
  for (int k = kmx - 1; k >= k1x; --k) {
    const double cc = S(A_A3, k, c);
    d2 = S(A_EX, k, c) - cc * d2;
    e2 = S(A_VTZ, k, c) - cc * e2;
    S(A_EX, k, c) = d2; S(A_VTZ, k, c) = e2;
    agA[IX(d, k, l)] = d2; arA[IX(d, k, l)] = e2;
  }
  double sg = 0, sr = 0;
  for (int k = k1x; k <= kmx; ++k) sg += S(A_EX, k, c);
  for (int k = k1x; k <= kmx; ++k) sr += S(A_VTZ, k, c);
  if (X) { d.s.eagx[l - 1] = sg; d.s.earx[l - 1] = sr; }
  else { d.s.eagy[l - 1] = sg; d.s.eary[l - 1] = sr; }
}

}  // namespace

// The dynamic shared-memory limit is a property of the kernel, shared by every handle: it only ever
// grows, to the largest tile any handle has needed (handles with different layer counts coexist).
int momentum_init(int km1) {
  static std::mutex mu;
  static int granted = 0;
  const int smem = (int)((size_t)NARR * km1 * MC * sizeof(double));
  std::lock_guard<std::mutex> lk(mu);
  if (smem <= granted) return 0;
  if (cudaFuncSetAttribute(k_momentum<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_momentum<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
  granted = smem;
  return 0;
}

void launch_momentum(const Dev& d, int ieq, const int* cols, int ncols, cudaStream_t st) {
  if (ncols <= 0) return;
  const size_t smem = (size_t)NARR * d.g.km1 * MC * sizeof(double);
  const int G = (ncols + MC - 1) / MC;
  if (ieq == 1) k_momentum<1><<<G, MT, smem, st>>>(d, cols, ncols);
  else k_momentum<2><<<G, MT, smem, st>>>(d, cols, ncols);
}

}  // namespace si3d
