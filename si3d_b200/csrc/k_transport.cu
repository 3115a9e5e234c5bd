// Column kernels after the zeta solve and the leapfrog-trapezoidal bookkeeping.
//
// slayer_h (si3d_procedures.f90:2070-2175), vel + continuity(1) (:2430-2567, :2653-2707),
// exsal (:2827-3076) + imsal/trid1 (:3079-3207, :3292-3352), vel2/layer_h (:2570-2631,
// :2181-2231), settrap (:3418-3618), settrap2 (:3944-4087), save (:3621-3941) with layer_hp2
// (:2238-2292), TopLayerIndexp2 (:2368-2427), continuity(2) and densty_s.
//
// Every kernel gives one thread one water column and walks the layers; a warp covers 32
// consecutive columns so each per-layer access of a layer-major field is coalesced.  Arrays that
// the reference keeps across calls with partial rewrites (the thread-private flux arrays Bth2,
// Bth3, Bth4, and uh/vh/h above the surface) are kept as persistent device fields and written
// exactly where the reference writes them.
#include "common.cuh"
#include "kernels.h"

namespace si3d {

namespace {


constexpr int TB = 128;
constexpr int BK_TRIP = 1;   // layers a lane handles per trip of the bookkeeping passes

__device__ __forceinline__ bool ewet(const Dev& d, int l) { return NB(d.g.lEC, l) != d.g.lm1; }
__device__ __forceinline__ bool nwet(const Dev& d, int l) { return NB(d.g.lNC, l) != d.g.lm1; }

// Deepest level of column l whose values can change.  Below kmz+1 the reference keeps
// h = hp = hpp = 0, wp = 0 and sal/salp/salpp/rhop at their initial values, and below the face
// depth min(kmz(l), kmz(lE)) it keeps hu = hup = hupp = uh-derived fields = 0 (a closed face keeps
// them 0 everywhere); its full-column loops rewrite those levels with identical values, so the
// loops below stop at these limits and the state stays bit-identical.
__device__ __forceinline__ int zlim(const Dev& d, int l) { return NB(d.g.kmz, l) + 1; }
__device__ __forceinline__ int ulim(const Dev& d, int l) {
  return ewet(d, l) ? min(NB(d.g.kmz, l), NB(d.g.kmz, NB(d.g.lEC, l))) : 0;
}
__device__ __forceinline__ int vlim(const Dev& d, int l) {
  return nwet(d, l) ? min(NB(d.g.kmz, l), NB(d.g.kmz, NB(d.g.lNC, l))) : 0;
}

// ------------------------------------------------------------- slayer_h
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_slayer_h(Dev d) {
  double* __restrict__ f_h = d.f.h;
  double* __restrict__ f_hp = d.f.hp;
  double* __restrict__ f_hu = d.f.hu;
  double* __restrict__ f_hup = d.f.hup;
  double* __restrict__ f_hv = d.f.hv;
  double* __restrict__ f_hvp = d.f.hvp;
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int ty = threadIdx.y;
  const int km1 = d.g.km1;
  const int kz = d.s.k1z[l - 1], ku = d.s.k1u[l - 1], kv = d.s.k1v[l - 1];
  double* __restrict__ h = f_h; double* __restrict__ hu = f_hu; double* __restrict__ hv = f_hv;
  const double* __restrict__ hp = f_hp; const double* __restrict__ hup = f_hup; const double* __restrict__ hvp = f_hvp;
  const int zL = zlim(d, l), uL = ulim(d, l), vL = vlim(d, l);
  #pragma unroll 4
  for (int k = 1 + ty; k <= min(kz - 1, zL); k += CLN) h[IX(d, k, l)] = hp[IX(d, k, l)];
  #pragma unroll 4
  for (int k = 1 + ty; k <= min(ku - 1, uL); k += CLN) hu[IX(d, k, l)] = hup[IX(d, k, l)];
  #pragma unroll 4
  for (int k = 1 + ty; k <= min(kv - 1, vL); k += CLN) hv[IX(d, k, l)] = hvp[IX(d, k, l)];
  #pragma unroll 4
  for (int k = kz + 2 + ty; k <= zL; k += CLN) h[IX(d, k, l)] = hp[IX(d, k, l)];
  #pragma unroll 4
  for (int k = ku + 1 + ty; k <= uL; k += CLN) hu[IX(d, k, l)] = hup[IX(d, k, l)];
  #pragma unroll 4
  for (int k = kv + 2 + ty; k <= vL; k += CLN) hv[IX(d, k, l)] = hvp[IX(d, k, l)];
  // the copies above leave out the surface layers written below, so the lanes never overlap
  if (ty != 0) return;
  // Surface layers.  A column whose surface index has reached the bottom level (every layer
  // dry) is left untouched: the reference would read zlevel past km1 there.
  const double sl = d.s.s[l - 1];
  int k = kz;
  if (k < km1) {
    double haux = fmin(zl(d, k + 1), d.g.hhs[l - 1]) + sl;
    if (haux <= HMIN) {
      h[IX(d, k, l)] = ZERO;
      k = k + 1;
      if (k < km1) {
        haux = fmin(zl(d, k + 1), d.g.hhs[l - 1]) + sl;
        h[IX(d, k, l)] = (haux <= HMIN) ? ZERO : haux;
      }
    } else h[IX(d, k, l)] = haux;
  }
  if (ewet(d, l)) {
    if (ku < km1) {
      const double sm = fmax(sl, d.s.s[NB(d.g.lEC, l) - 1]);
      const double haux = fmin(zl(d, ku + 1), d.g.hhu[l - 1]) + sm;
      // on drying the reference recomputes the same layer (k is reset to k1u, :2136)
      hu[IX(d, ku, l)] = (haux <= HMIN) ? ZERO : haux;
    }
  }  // a closed east face keeps hu = hup = 0 (the reference's copy of hup(k1u:k1u+1) is a no-op)
  if (nwet(d, l)) {
    const double sm = fmax(sl, d.s.s[NB(d.g.lNC, l) - 1]);
    k = kv;
    if (k < km1) {
      double haux = fmin(zl(d, k + 1), d.g.hhv[l - 1]) + sm;
      if (haux <= HMIN) {
        hv[IX(d, k, l)] = ZERO;
        k = k + 1;
        if (k < km1) {
          haux = fmin(zl(d, k + 1), d.g.hhv[l - 1]) + sm;
          hv[IX(d, k, l)] = (haux <= HMIN) ? ZERO : haux;
        }
      } else hv[IX(d, k, l)] = haux;
    }
  }  // a closed north face keeps hv = hvp = 0
}

// ------------------------------------------------------------- vel (uh, vh, k1u, k1v)
template <int IEQ, int CLN>
__global__ void __launch_bounds__(32 * CLN) k_vel_uv(Dev d, const int* __restrict__ cols, int ncols) {
  double* __restrict__ f_agx = d.f.agx;
  double* __restrict__ f_agy = d.f.agy;
  double* __restrict__ f_arx = d.f.arx;
  double* __restrict__ f_ary = d.f.ary;
  double* __restrict__ f_hu = d.f.hu;
  double* __restrict__ f_hv = d.f.hv;
  double* __restrict__ f_uh = d.f.uh;
  double* __restrict__ f_vh = d.f.vh;
  const int t = blockIdx.x * 32 + threadIdx.x, ty = threadIdx.y;
  const bool act = t < ncols;
  const bool X = IEQ == 1;
  int l = 0, k0 = 0;
  int* k1 = X ? d.s.k1u : d.s.k1v;
  double* uv = X ? f_uh : f_vh;
  if (act) {
    l = cols[t];
    const int lO = X ? NB(d.g.lEC, l) : NB(d.g.lNC, l);
    const int kmx = min(NB(d.g.kmz, lO), NB(d.g.kmz, l));
    k0 = k1[l - 1];
    const double gth = (X ? d.p.gdtdx : d.p.gdtdy) * d.tz;
    const double c = gth * 1000. * (d.s.s[lO - 1] - d.s.s[l - 1]);
    const double* ag = X ? f_agx : f_agy;
    const double* ar = X ? f_arx : f_ary;
#pragma unroll 4
    for (int k = k0 + ty; k <= kmx; k += CLN) uv[IX(d, k, l)] = ag[IX(d, k, l)] - c * ar[IX(d, k, l)];
  }
  __syncthreads();   // the surface correction reads layers written by other lanes
  if (!act || ty != 0) return;
  const double* huv = X ? f_hu : f_hv;
  // (a face column with every layer dry, k0 = km1, is never reached: the reference would write
  //  past the last level there)
  if (k0 < d.g.km1 && huv[IX(d, k0, l)] <= ZERO) {
    uv[IX(d, k0 + 1, l)] = uv[IX(d, k0, l)] + uv[IX(d, k0 + 1, l)];
    uv[IX(d, k0, l)] = 0.0;
    k1[l - 1] = k0 + 1;
  }
}

// continuity(1) at the end of vel and continuity(2) after settrap, settrap2 and save
// (si3d_procedures.f90:2653-2707): wp from the horizontal fluxes, summed from the column bottom up.
// Block = 32 consecutive columns x CLN layer lanes.  The lanes form every layer's x and y flux
// differences, divided by the grid constant as the reference divides, into shared memory (one
// memory round trip per layer for all of them, every load of a layer issued first); then the first
// warp runs the bottom-up sum of its 32 columns in the reference's order, w = (w - tx) - ty per
// layer, so wp is bit-identical to the reference's one-thread loop.  CONT1: the fluxes are
// uh + uhpp over 2 dx (2 dy), and k1z moves down one level where the top cell has dried.
// Dynamic shared memory: two planes of (km1 + 1) levels x 32 columns.
template <int CLN, bool CONT1>
__global__ void __launch_bounds__(32 * CLN) k_cont(Dev d) {
  extern __shared__ double s_term[];
  const int cx = threadIdx.x, ty = threadIdx.y;
  const int l = blockIdx.x * 32 + cx + 1;
  const bool act = l <= d.g.lm;
  const int kms = act ? NB(d.g.kmz, l) : 0, k1s = act ? d.s.k1z[l - 1] : 1;
  const bool wet = act && k1s <= kms;
  double* __restrict__ wp = d.f.wp;
  double* s_x = s_term;
  double* s_y = s_term + (d.g.km1 + 1) * 32;
  if (wet) {
    const int lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l);
    for (int k = 1 + ty; k < k1s; k += CLN) wp[IX(d, k, l)] = 0.0;   // wp below kms is never non-zero
    if (CONT1) {
      const double* __restrict__ uh = d.f.uh;
      const double* __restrict__ vh = d.f.vh;
      const double* __restrict__ uhpp = d.f.uhpp;
      const double* __restrict__ vhpp = d.f.vhpp;
      for (int k = d.g.k1 + ty; k <= kms; k += CLN) {
        const int ik = IX(d, k, l), iw = IX(d, k, lW), is = IX(d, k, lS);
        const double a0 = uh[ik], a1 = uh[iw], a2 = uhpp[ik], a3 = uhpp[iw];
        const double b0 = vh[ik], b1 = vh[is], b2 = vhpp[ik], b3 = vhpp[is];
        s_x[k * 32 + cx] = (a0 - a1 + a2 - a3) / d.p.twodx;
        s_y[k * 32 + cx] = (b0 - b1 + b2 - b3) / d.p.twody;
      }
    } else {
      const double* __restrict__ uhp = d.f.uhp;
      const double* __restrict__ vhp = d.f.vhp;
      for (int k = d.g.k1 + ty; k <= kms; k += CLN) {
        const int ik = IX(d, k, l);
        const double a0 = uhp[ik], a1 = uhp[IX(d, k, lW)], b0 = vhp[ik], b1 = vhp[IX(d, k, lS)];
        s_x[k * 32 + cx] = (a0 - a1) / d.p.dx;
        s_y[k * 32 + cx] = (b0 - b1) / d.p.dy;
      }
    }
  }
  __syncthreads();
  if (ty != 0 || !act) return;
  if (wet) {
    double w = 0.0;
#pragma unroll 4
    for (int k = kms; k > k1s; --k) {
      w = w - s_x[k * 32 + cx] - s_y[k * 32 + cx];
      wp[IX(d, k, l)] = w;
    }
    // level k1s: its own term, then the dry levels above it folded in (the reference stores the
    // first sum and overwrites it with the second)
    double ws = w - s_x[k1s * 32 + cx] - s_y[k1s * 32 + cx];
    for (int k = d.g.k1; k <= k1s - 1; ++k) ws = ws - s_x[k * 32 + cx] - s_y[k * 32 + cx];
    wp[IX(d, k1s, l)] = ws;
  }
  if (CONT1 && d.f.h[IX(d, k1s, l)] <= ZERO) d.s.k1z[l - 1] = min(k1s + 1, d.g.km1);
}

// ------------------------------------------------------------- exsal fluxes

// Cell-parallel kernels use blocks of 32 consecutive columns x CLN layer lanes: a warp reads one
// layer of 32 consecutive columns (coalesced) and each thread takes layers k0 + lane, k0 + lane + CLN...

// exsal's three limited fluxes per cell (:2895-3013) of the scalar `sp` (salpp), into the
// persistent Bth2/Bth4/Bth3 fields.
// Every value a layer may need is loaded before any test (all addresses are valid: neighbours are
// real columns or the dry column lm1, and layer k - 2 is clamped to 1), so a layer costs one memory
// round trip; the tests then only select among loaded values, in the reference's arithmetic (with
// products by the reciprocals of dx and dy where the reference divides by them, here and in the
// right-hand side below).
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_exsal_flux(Dev d, const double* __restrict__ sp) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  if (k1s + (int)threadIdx.y > kms) return;
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const int lEE = NB(d.g.lEC, lE), lNN = NB(d.g.lNC, lN);
  const int P = d.g.P;
  const double twodt1 = d.p.twodt * d.tz;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ hp = d.f.hp;
  const double* __restrict__ hup = d.f.hup;
  const double* __restrict__ hvp = d.f.hvp;
  const double* __restrict__ uhpp = d.f.uhpp;
  const double* __restrict__ uh = d.f.uh;
  const double* __restrict__ vhpp = d.f.vhpp;
  const double* __restrict__ vh = d.f.vh;
  const double* __restrict__ wp = d.f.wp;
  double* __restrict__ B2 = d.f.Bth2;
  double* __restrict__ B3 = d.f.Bth3;
  double* __restrict__ B4 = d.f.Bth4;
  const int dE = lE - l, dW = lW - l, dN = lN - l, dS = lS - l, dEE = lEE - l, dNN = lNN - l;
  for (int k = k1s + threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const int ik2 = IX(d, k - 2 < 1 ? 1 : k - 2, l);
    // ---- all loads of this layer
    const double hu = hup[ik], hv = hvp[ik], hpu = hp[ik - P], hpk = hp[ik];
    const double uo = uhpp[ik], un = uh[ik], vo = vhpp[ik], vn = vh[ik], wk = wp[ik];
    const double s2 = sp[ik], sE = sp[ik + dE], sW = sp[ik + dW], sEE = sp[ik + dEE];
    const double sN = sp[ik + dN], sS = sp[ik + dS], sNN = sp[ik + dNN];
    const double sU = sp[ik - P], sUU = sp[ik2], sD = sp[ik + P];
    const double hW = hpp[ik + dW], hEE = hpp[ik + dEE], hS = hpp[ik + dS], hNN = hpp[ik + dNN];
    const double hUU = hpp[ik2], hD = hpp[ik + P];
    // EW
    if (hu > ZERO) {
      const double vel = (uo + un) / 2.;
      const double s3 = sE;
      const double s1 = (hW <= ZERO) ? s2 : sW;
      const double s4 = (hEE <= ZERO) ? s3 : sEE;
      const double C_f = superbee(s1, s2, s3, s4, vel, 0.0);
      B2[ik] = vel / 2. * (s3 + s2) - ((1. - C_f) * fabs(vel) + vel * vel * twodt1 * d.p.rdx * C_f) * (s3 - s2) / 2.;
    } else B2[ik] = 0.0;
    // NS
    if (hv > ZERO) {
      const double vel = (vo + vn) / 2.;
      const double s3 = sN;
      const double s1 = (hS <= ZERO) ? s2 : sS;
      const double s4 = (hNN <= ZERO) ? s3 : sNN;
      const double C_f = superbee(s1, s2, s3, s4, vel, 0.0);
      B4[ik] = vel / 2. * (s3 + s2) - ((1. - C_f) * fabs(vel) + vel * vel * twodt1 * d.p.rdy * C_f) * (s3 - s2) / 2.;
    } else B4[ik] = 0.0;
    // UD (hp(1, l) is never positive, so k-2 >= 1 whenever this branch is taken)
    if (hpu > ZERO) {
      double vel = wk;
      if (k == k1s) vel = 0.0;
      const double s3 = sU;
      const double s4 = (k - 2 < 1 || hUU <= ZERO) ? s3 : sUU;
      const double s1 = (hD <= ZERO) ? s2 : sD;
      const double C_f = superbee(s1, s2, s3, s4, vel, 1.0);
      const double delz = (hpk + hpu) / 2.;
      B3[ik] = vel / 2. * (s3 + s2) - ((1. - C_f) * fabs(vel) + vel * vel * twodt1 / delz * C_f) * (s3 - s2) / 2.;
    } else B3[ik] = 0.0;
  }
}

// exsal's divergence Bex plus the heat source (imsal's right-hand side ds, :3059-3065, :3113) per
// cell, staged in sal (which imsal then overwrites with the solution in place).  The horizontal-
// diffusion coefficients Bhaxpp/Bhaypp of a column m at layer k (:2867-2877) are A * hupp (hvpp)
// inside m's wet layers [k1, kmz(m)] and zero elsewhere or for the dry column; as in the flux kernel
// every value is loaded before the tests select among them.
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_exsal_rhs(Dev d) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  if (k1s + (int)threadIdx.y > kms) return;
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const int lm1 = d.g.lm1, k1 = d.g.k1;
  const int kmW = NB(d.g.kmz, lW), kmS = NB(d.g.kmz, lS);
  const int P = d.g.P;
  const double twodt1 = d.p.twodt * d.tz;
  const double* __restrict__ sp = d.f.salpp;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ B2 = d.f.Bth2;
  const double* __restrict__ B3 = d.f.Bth3;
  const double* __restrict__ B4 = d.f.Bth4;
  const double* __restrict__ hupp = d.f.hupp;
  const double* __restrict__ hvpp = d.f.hvpp;
  const double* __restrict__ heat = d.f.HeatSource;
  double* __restrict__ sal = d.f.sal;
  const bool ihd = d.p.ihd > 0;
  const int dE = lE - l, dW = lW - l, dN = lN - l, dS = lS - l;
  for (int k = k1s + threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const double spc = sp[ik], hc = hpp[ik], b2 = B2[ik], b2W = B2[ik + dW], b4 = B4[ik], b4S = B4[ik + dS];
    const double b3 = B3[ik], b3D = B3[ik + P], hs = heat[ik];
    double sE = 0, sW = 0, sN = 0, sS = 0, axl = 0, axW = 0, ayl = 0, ayS = 0;
    if (ihd) {
      sE = sp[ik + dE]; sW = sp[ik + dW]; sN = sp[ik + dN]; sS = sp[ik + dS];
      axl = hupp[ik]; axW = hupp[ik + dW]; ayl = hvpp[ik]; ayS = hvpp[ik + dS];
    }
    double v = hc * spc / twodt1 - (b2 - b2W) * d.p.rdx - (b4 - b4S) * d.p.rdy - (b3 - b3D);
    if (ihd) {
      const bool inl = k >= k1 && k <= kms;
      const double bxl = inl ? d.p.Ax0 * axl : 0.0;
      const double bxW = (lW != lm1 && k >= k1 && k <= kmW) ? d.p.Ax0 * axW : 0.0;
      const double byl = inl ? d.p.Ay0 * ayl : 0.0;
      const double byS = (lS != lm1 && k >= k1 && k <= kmS) ? d.p.Ay0 * ayS : 0.0;
      const double hd = (bxl * (sE - spc) - bxW * (spc - sW)) * d.p.rdxdx + (byl * (sN - spc) - byS * (spc - sS)) * d.p.rdydy;
      v = v + hd;
    }
    sal[ik] = v + hs;
  }
}

// imsal's vertical-diffusion tridiagonal solve per column (trid1), right-hand side read from sal.
template <int NTB>
__global__ void __launch_bounds__(NTB) k_imsal(Dev d) {
  constexpr int RD = 4;                // layers in flight in the forward sweep
  __shared__ double ring[RD][3][NTB];  // [slot][input][thread]: a thread's slots are its own
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  const int nw = kms - k1s + 1;
  if (nw < 1) return;
  const int P = d.g.P;
  const double twodt1 = d.p.twodt * d.tz;
  const double* __restrict__ sp = d.f.salpp;
  const double* __restrict__ h = d.f.h;
  const double* __restrict__ Dv = d.f.Dv;
  double* __restrict__ sal = d.f.sal;
  double* __restrict__ esc = d.scr;
  // layer thickness at time n with the surface corrections (:3128-3132)
  const double hpp_k1 = d.f.hpp[IX(d, k1s, l)];
  auto hn = [&](int k) -> double {
    if (k == k1s) return twodt1 * d.f.wp[IX(d, k1s, l)] + hpp_k1;
    if (k == k1s + 1 && hpp_k1 <= ZERO) return d.f.hpp[IX(d, k1s + 1, l)];
    return h[IX(d, k, l)];
  };
  if (nw == 1) {
    const double a2 = hn(k1s) / twodt1;
    const double ds = sal[IX(d, k1s, l)];
    double v = ds / a2;
    if (h[IX(d, k1s, l)] < 1.E-2) v = sp[IX(d, k1s, l)];
    sal[IX(d, k1s, l)] = v;
    return;
  }
  // trid1 forward sweep: e in scratch, f in sal.  Iteration k reads sal(k), Dv(k + 1) and h(k + 1);
  // these are copied into this thread's slots of a shared-memory ring by cp.async, RD layers ahead.
  // 1 / (hn(k) + hn(k+1)) is shared with the next layer's a1, so a layer takes two divisions.
  const double rt = 1.0 / twodt1;
  const int tid = threadIdx.x;
  auto issue = [&](int kk, int slot) {
    const int ikk = IX(d, kk, l);
    cp_async8(&ring[slot][0][tid], &sal[ikk]);
    cp_async8(&ring[slot][1][tid], &Dv[ikk + P]);
    cp_async8(&ring[slot][2][tid], &h[ikk + P]);
  };
#pragma unroll
  for (int j = 0; j < RD; ++j) {   // one commit group per layer (empty past the bottom)
    if (k1s + j <= kms) issue(k1s + j, j);
    cp_async_commit();
  }
  const double hn1 = hn(k1s + 1);  // the second layer's thickness carries the surface correction
  double hn_k = hn(k1s), e_prev = 0, f_prev = 0, rkm = 0.0, dvk = Dv[IX(d, k1s, l)];
  int ik = IX(d, k1s, l);
  for (int k = k1s, slot = 0; k <= kms; ++k, ik += P, slot = (slot + 1 == RD) ? 0 : slot + 1) {
    cp_async_wait<RD - 1>();     // layer k's group has landed (this thread's own copies)
    const double ds = ring[slot][0][tid], dvkp = ring[slot][1][tid];
    const double hn_kp = (k < kms) ? ((k == k1s) ? hn1 : ring[slot][2][tid]) : 0.0;
    const double rkp = (k < kms) ? 1.0 / (hn_k + hn_kp) : 0.0;
    const double a3 = (k < kms) ? -dvkp * rkp * 2. : 0.0;
    double a1 = 0.0;
    if (k > k1s) a1 = -dvk * rkm * 2.;
    const double a2 = hn_k * rt - a1 - a3;
    const int kk = k - k1s + 1;
    if (kk == 1) {
      const double r = 1.0 / a2;
      e_prev = -a3 * r;
      f_prev = ds * r;
      esc[ik] = e_prev;
      sal[ik] = f_prev;
    } else {
      const double r = 1.0 / (a2 + a1 * e_prev);
      const double f = (ds - a1 * f_prev) * r;
      sal[ik] = f;
      if (kk < nw) {
        const double e = -a3 * r;
        esc[ik] = e;
        e_prev = e; f_prev = f;
      }
    }
    // refill the slot with layer k + RD (its values are consumed: the stores above depend on them)
    if (k + RD <= kms) issue(k + RD, slot);
    cp_async_commit();
    hn_k = hn_kp;
    rkm = rkp;
    dvk = dvkp;
  }
  double nxt = sal[IX(d, kms, l)];
#pragma unroll 4
  for (int k = kms - 1; k >= k1s; --k) {
    nxt = esc[IX(d, k, l)] * nxt + sal[IX(d, k, l)];
    sal[IX(d, k, l)] = nxt;
  }
  const double top = sal[IX(d, k1s, l)];
  for (int k = d.g.k1; k <= k1s - 1; ++k) sal[IX(d, k, l)] = top;
  sal[IX(d, kms + 1, l)] = sal[IX(d, kms, l)];
}

// ------------------------------------------------------------- vel2 (layer_h + wetting)
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_vel2(Dev d) {
  double* __restrict__ f_h = d.f.h;
  double* __restrict__ f_hu = d.f.hu;
  double* __restrict__ f_hv = d.f.hv;
  double* __restrict__ f_uh = d.f.uh;
  double* __restrict__ f_vh = d.f.vh;
  const int l = blockIdx.x * 32 + threadIdx.x + 1, ty = threadIdx.y;
  const bool act = l <= d.g.lm;
  if (act) {
    const int kms = NB(d.g.kmz, l);
    const double sl = d.s.s[l - 1];
#pragma unroll 4
    for (int k = d.g.k1 + ty; k <= kms; k += CLN) {
      double v = fmin(zl(d, k + 1), d.g.hhs[l - 1]) - fmax(zl(d, k), -sl);
      if (v <= HMIN) v = ZERO;
      f_h[IX(d, k, l)] = v;
    }
    if (ewet(d, l)) {
      const int lE = NB(d.g.lEC, l);
      const int kmx = min(kms, NB(d.g.kmz, lE));
      const double sm = fmax(sl, d.s.s[lE - 1]);
  #pragma unroll 4
      for (int k = d.g.k1 + ty; k <= kmx; k += CLN) {
        double v = fmin(zl(d, k + 1), d.g.hhu[l - 1]) - fmax(zl(d, k), -sm);
        if (v <= HMIN) v = ZERO;
        f_hu[IX(d, k, l)] = v;
      }
    }
    if (nwet(d, l)) {
      const int lN = NB(d.g.lNC, l);
      const int kmy = min(kms, NB(d.g.kmz, lN));
      const double sm = fmax(sl, d.s.s[lN - 1]);
  #pragma unroll 4
      for (int k = d.g.k1 + ty; k <= kmy; k += CLN) {
        double v = fmin(zl(d, k + 1), d.g.hhv[l - 1]) - fmax(zl(d, k), -sm);
        if (v <= HMIN) v = ZERO;
        f_hv[IX(d, k, l)] = v;
      }
    }
  }
  __syncthreads();   // the surface corrections read layers written by other lanes
  if (!act || ty != 0) return;
  if (ewet(d, l)) {
    const int k = d.s.k1u[l - 1];
    const double hkm = f_hu[IX(d, k - 1, l)];
    if (hkm > ZERO) {
      const double hk = f_hu[IX(d, k, l)];
      const double ut = f_uh[IX(d, k, l)] / (hk + hkm);
      f_uh[IX(d, k, l)] = ut * hk;
      f_uh[IX(d, k - 1, l)] = ut * hkm;
    }
  }
  if (nwet(d, l)) {
    const int k = d.s.k1v[l - 1];
    const double hkm = f_hv[IX(d, k - 1, l)];
    if (hkm > ZERO) {
      const double hk = f_hv[IX(d, k, l)];
      const double vt = f_vh[IX(d, k, l)] / (hk + hkm);
      f_vh[IX(d, k, l)] = vt * hk;
      f_vh[IX(d, k - 1, l)] = vt * hkm;
    }
  }
}

// ------------------------------------------------------------- settrap / settrap2 / save
// zeta at n+1/2 (settrap: spp <- sp first; settrap2: recompute only)
__global__ void k_half_zeta(Dev d, int rotate) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  if (rotate) d.s.spp[l - 1] = d.s.sp[l - 1];
  d.s.sp[l - 1] = 0.5 * (d.s.s[l - 1] + d.s.spp[l - 1]);
}

// Bookkeeping kernels are cell-parallel: block = 32 consecutive columns x CLN layer lanes, a lane
// taking layers k0 + lane, k0 + lane + CLN, ...  Every routine of a call (the pp rotation, the
// thicknesses, the scalar with its density, both velocities) is one pass over the layers in which a
// cell's loads are all issued before any of its arithmetic, one trip ahead (walk_layers).  The
// expressions are the reference's, so the state is bit-identical to the per-routine loops.

// The layer walk of a lane: layers k0, k0 + CLN, ... up to ke, BK_TRIP of them per trip.  `load`
// fills one layer's inputs (its addresses clamped inside the column), `apply` does nothing above ke.
// The next trip's loads are issued before this trip's arithmetic and stores, so a lane keeps a
// memory round trip in flight while it evaluates the equation of state (measured at 2000x1000x60:
// settrap 1.79 -> 1.67 ms against the same walk without the prefetch; two layers per trip with the
// prefetch need 150 registers and are slower).
template <int CLN, typename In, typename Load, typename Apply>
__device__ __forceinline__ void walk_layers(int k0, int ke, Load& load, Apply& apply) {
  constexpr int STEP = BK_TRIP * CLN;
  if (k0 > ke) return;
  In v[BK_TRIP];
#pragma unroll
  for (int t = 0; t < BK_TRIP; ++t) load(k0 + t * CLN, v[t]);
  for (int k = k0;; k += STEP) {
    const bool more = k + STEP <= ke;
    In w[BK_TRIP];
    if (more) {
#pragma unroll
      for (int t = 0; t < BK_TRIP; ++t) load(k + STEP + t * CLN, w[t]);
    }
#pragma unroll
    for (int t = 0; t < BK_TRIP; ++t) apply(k + t * CLN, v[t]);
    if (!more) break;
#pragma unroll
    for (int t = 0; t < BK_TRIP; ++t) v[t] = w[t];
  }
}

// Values of one cell (k, l) that settrap / settrap2 read.
struct HalfIn {
  double hp, hup, hvp, sal, salq, uh, uhq, up, vh, vhq, vp;   // q: salp/uhp/vhp (rotate) or the pp level
};

// settrap / settrap2 body after the zeta update (layer_hp2, TopLayerIndexp2, scalars at n+1/2 with
// densty_s, velocities at n+1/2) with settrap's rotation n -> n-1 of h, s, u, v (ROT).  The first
// wet layer of each column (TopLayerIndexp2) is the minimum over the lanes, reduced in shared
// memory; the surface corrections at the new k1u/k1v run after a block barrier, once every layer's
// average is in place.
template <int CLN, bool ROT>
__global__ void __launch_bounds__(32 * CLN) k_half_level(Dev d) {
  double* __restrict__ f_hp = d.f.hp;
  double* __restrict__ f_hpp = d.f.hpp;
  double* __restrict__ f_hu = d.f.hu;
  double* __restrict__ f_hup = d.f.hup;
  double* __restrict__ f_hupp = d.f.hupp;
  double* __restrict__ f_hv = d.f.hv;
  double* __restrict__ f_hvp = d.f.hvp;
  double* __restrict__ f_hvpp = d.f.hvpp;
  double* __restrict__ f_rhop = d.f.rhop;
  double* __restrict__ f_sal = d.f.sal;
  double* __restrict__ f_salp = d.f.salp;
  double* __restrict__ f_salpp = d.f.salpp;
  double* __restrict__ f_uh = d.f.uh;
  double* __restrict__ f_uhp = d.f.uhp;
  double* __restrict__ f_uhpp = d.f.uhpp;
  double* __restrict__ f_up = d.f.up;
  double* __restrict__ f_upp = d.f.upp;
  double* __restrict__ f_vh = d.f.vh;
  double* __restrict__ f_vhp = d.f.vhp;
  double* __restrict__ f_vhpp = d.f.vhpp;
  double* __restrict__ f_vp = d.f.vp;
  double* __restrict__ f_vpp = d.f.vpp;
  __shared__ int s_first[3][CLN][32];
  const int cx = threadIdx.x, ty = threadIdx.y;
  const int l = blockIdx.x * 32 + cx + 1;
  const bool act = l <= d.g.lm;
  const int k1 = d.g.k1, km1 = d.g.km1;
  bool ew = false, nw = false;
  int fz = km1, fu = km1, fv = km1;
  if (act) {
    const int kms = NB(d.g.kmz, l);
    ew = ewet(d, l);
    nw = nwet(d, l);
    const int lE = NB(d.g.lEC, l), lN = NB(d.g.lNC, l);
    const int kmx = ew ? min(kms, NB(d.g.kmz, lE)) : 0;
    const int kmy = nw ? min(kms, NB(d.g.kmz, lN)) : 0;
    const double spl = d.s.sp[l - 1];
    const double hhs = d.g.hhs[l - 1], hhu = d.g.hhu[l - 1], hhv = d.g.hhv[l - 1];
    const double smx = fmax(spl, d.s.sp[lE - 1]), smy = fmax(spl, d.s.sp[lN - 1]);
    // settrap also rotates hp, hup, hvp over levels 1 .. kmz + 1 (1 .. kmx, 1 .. kmy)
    const int kb = ROT ? 1 : k1, ke = ROT ? kms + 1 : kms;
    auto load = [&](int k, HalfIn& v) {
      const int ik = IX(d, min(k, ke), l);   // clamped: every address is inside the column
      v.hp = f_hp[ik]; v.hup = f_hup[ik]; v.hvp = f_hvp[ik];
      v.sal = f_sal[ik]; v.salq = ROT ? f_salp[ik] : f_salpp[ik];
      v.uh = f_uh[ik]; v.uhq = ROT ? f_uhp[ik] : f_uhpp[ik]; v.up = f_up[ik];
      v.vh = f_vh[ik]; v.vhq = ROT ? f_vhp[ik] : f_vhpp[ik]; v.vp = f_vp[ik];
    };
    auto apply = [&](int k, const HalfIn& v) {
      if (k > ke) return;
      const int ik = IX(d, k, l);
      const bool zin = k >= k1 && k <= kms;
      const bool uin = ew && k >= k1 && k <= kmx;
      const bool vin = nw && k >= k1 && k <= kmy;
      if (ROT) {
        f_hpp[ik] = v.hp;
        if (ew && k <= kmx) f_hupp[ik] = v.hup;
        if (nw && k <= kmy) f_hvpp[ik] = v.hvp;
      }
      if (zin) {
        double h = fmin(zl(d, k + 1), hhs) - fmax(zl(d, k), -spl);
        if (h <= HMIN) h = ZERO;
        f_hp[ik] = h;
        if (h > ZERO && k < fz) fz = k;
        // scalar at n+1/2 (salpp <- salp first in settrap)
        if (ROT) f_salpp[ik] = v.salq;
        const double sp = (v.sal + v.salq) / 2.;
        f_salp[ik] = sp;
        f_rhop[ik] = densty_s(sp, 0.00004, zmid(d, k, h)) - 1000.;
      }
      if (uin) {
        double h = fmin(zl(d, k + 1), hhu) - fmax(zl(d, k), -smx);
        if (h <= HMIN) h = ZERO;
        f_hup[ik] = h;
        if (h > ZERO && k < fu) fu = k;
        if (ROT) { f_uhpp[ik] = v.uhq; f_upp[ik] = v.up; }
        if (h > ZERO) { const double a = 0.5 * (v.uh + v.uhq); f_uhp[ik] = a; f_up[ik] = a / h; }
        else { f_uhp[ik] = 0.0; f_up[ik] = 0.0; }
      }
      if (vin) {
        double h = fmin(zl(d, k + 1), hhv) - fmax(zl(d, k), -smy);
        if (h <= HMIN) h = ZERO;
        f_hvp[ik] = h;
        if (h > ZERO && k < fv) fv = k;
        if (ROT) { f_vhpp[ik] = v.vhq; f_vpp[ik] = v.vp; }
        if (h > ZERO) { const double a = 0.5 * (v.vh + v.vhq); f_vhp[ik] = a; f_vp[ik] = a / h; }
        else { f_vhp[ik] = 0.0; f_vp[ik] = 0.0; }
      }
    };
    walk_layers<CLN, HalfIn>(kb + ty, ke, load, apply);
  }
  s_first[0][ty][cx] = fz; s_first[1][ty][cx] = fu; s_first[2][ty][cx] = fv;
  __syncthreads();
  if (act && ty == 0) {
    int kz = km1, ku = km1, kv = km1;
#pragma unroll
    for (int q = 0; q < CLN; ++q) {
      kz = min(kz, s_first[0][q][cx]); ku = min(ku, s_first[1][q][cx]); kv = min(kv, s_first[2][q][cx]);
    }
    d.s.k1z[l - 1] = kz; d.s.k1u[l - 1] = ku; d.s.k1v[l - 1] = kv;
  }
  if (!act || ty != 0) return;
  // surface corrections at the first wet face layer (:3503-3516 / :4033-4046)
  if (ew) {
    const int k = d.s.k1u[l - 1];
    const int ik = IX(d, k, l);
    if (f_hu[IX(d, k - 1, l)] > ZERO) {
      f_uhp[ik] = f_uhp[ik] + f_uh[IX(d, k - 1, l)] / 2.;
      f_up[ik] = f_uhp[ik] / f_hup[ik];
    }
    if (f_hupp[IX(d, k - 1, l)] > ZERO) {
      f_uhp[ik] = f_uhp[ik] + f_uhpp[IX(d, k - 1, l)] / 2.;
      f_up[ik] = f_uhp[ik] / f_hup[ik];
    }
  }
  if (nw) {
    const int k = d.s.k1v[l - 1];
    const int ik = IX(d, k, l);
    if (f_hv[IX(d, k - 1, l)] > ZERO) {
      f_vhp[ik] = f_vhp[ik] + f_vh[IX(d, k - 1, l)] / 2.;
      f_vp[ik] = f_vhp[ik] / f_hvp[ik];
    }
    if (f_hvpp[IX(d, k - 1, l)] > ZERO) {
      f_vhp[ik] = f_vhp[ik] + f_vhpp[IX(d, k - 1, l)] / 2.;
      f_vp[ik] = f_vhp[ik] / f_hvp[ik];
    }
  }
}

// Values of one cell (k, l) that save reads.
struct SaveIn {
  double h, hp, hu, hup, hv, hvp, sal, salp, uh, uhp, up, vh, vhp, vp;
};

// save (istep = 2 after a trapezoidal step, 1 after a leapfrog step, which also rotates n -> n-1):
// one pass over levels 1 .. kmz + 1 like k_half_level; the new first wet layers are reduced over
// the lanes in shared memory.
template <int CLN, bool ROT>
__global__ void __launch_bounds__(32 * CLN) k_save(Dev d) {
  double* __restrict__ f_h = d.f.h;
  double* __restrict__ f_hp = d.f.hp;
  double* __restrict__ f_hpp = d.f.hpp;
  double* __restrict__ f_hu = d.f.hu;
  double* __restrict__ f_hup = d.f.hup;
  double* __restrict__ f_hupp = d.f.hupp;
  double* __restrict__ f_hv = d.f.hv;
  double* __restrict__ f_hvp = d.f.hvp;
  double* __restrict__ f_hvpp = d.f.hvpp;
  double* __restrict__ f_rhop = d.f.rhop;
  double* __restrict__ f_sal = d.f.sal;
  double* __restrict__ f_salp = d.f.salp;
  double* __restrict__ f_salpp = d.f.salpp;
  double* __restrict__ f_uh = d.f.uh;
  double* __restrict__ f_uhp = d.f.uhp;
  double* __restrict__ f_uhpp = d.f.uhpp;
  double* __restrict__ f_up = d.f.up;
  double* __restrict__ f_upp = d.f.upp;
  double* __restrict__ f_vh = d.f.vh;
  double* __restrict__ f_vhp = d.f.vhp;
  double* __restrict__ f_vhpp = d.f.vhpp;
  double* __restrict__ f_vp = d.f.vp;
  double* __restrict__ f_vpp = d.f.vpp;
  __shared__ int s_first[3][CLN][32];
  const int cx = threadIdx.x, ty = threadIdx.y;
  const int l = blockIdx.x * 32 + cx + 1;
  const bool act = l <= d.g.lm;
  const int k1 = d.g.k1, km1 = d.g.km1;
  int fz = km1, fu = km1, fv = km1;
  if (act) {
    if (ty == 0) {
      if (ROT) d.s.spp[l - 1] = d.s.sp[l - 1];
      d.s.sp[l - 1] = d.s.s[l - 1];
    }
    const int kms = NB(d.g.kmz, l);
    const int zL = zlim(d, l), uL = ulim(d, l), vL = vlim(d, l);
    const int ksal = min(d.g.km, zL);
    auto load = [&](int k, SaveIn& v) {
      const int ik = IX(d, min(k, zL), l);   // clamped: every address is inside the column
      v.h = f_h[ik]; v.hp = f_hp[ik]; v.hu = f_hu[ik]; v.hup = f_hup[ik]; v.hv = f_hv[ik]; v.hvp = f_hvp[ik];
      v.sal = f_sal[ik]; v.salp = f_salp[ik];
      v.uh = f_uh[ik]; v.uhp = f_uhp[ik]; v.up = f_up[ik];
      v.vh = f_vh[ik]; v.vhp = f_vhp[ik]; v.vp = f_vp[ik];
    };
    auto apply = [&](int k, const SaveIn& v) {
      if (k > zL) return;
      const int ik = IX(d, k, l);
      if (ROT) f_hpp[ik] = v.hp;
      f_hp[ik] = v.h;
      if (k >= k1 && k <= kms && v.h > ZERO && k < fz) fz = k;
      if (k <= uL) {
        if (ROT) f_hupp[ik] = v.hup;
        f_hup[ik] = v.hu;
        if (k >= k1 && v.hu > ZERO && k < fu) fu = k;
      }
      if (k <= vL) {
        if (ROT) f_hvpp[ik] = v.hvp;
        f_hvp[ik] = v.hv;
        if (k >= k1 && v.hv > ZERO && k < fv) fv = k;
      }
      if (k >= k1 && k <= ksal) {
        const double z = zmid(d, k, v.h);
        if (ROT) f_salpp[ik] = v.salp;
        f_salp[ik] = v.sal;
        f_rhop[ik] = densty_s(v.sal, 0.00004, z) - 1000.;
      }
      if (k >= k1 && k <= uL) {
        if (ROT) { f_uhpp[ik] = v.uhp; f_upp[ik] = v.up; }
        if (v.hu > ZERO) { f_uhp[ik] = v.uh; f_up[ik] = v.uh / v.hu; }
        else { f_uhp[ik] = 0.0; f_up[ik] = 0.0; }
      }
      if (k >= k1 && k <= vL) {
        if (ROT) { f_vhpp[ik] = v.vhp; f_vpp[ik] = v.vp; }
        if (v.hv > ZERO) { f_vhp[ik] = v.vh; f_vp[ik] = v.vh / v.hv; }
        else { f_vhp[ik] = 0.0; f_vp[ik] = 0.0; }
      }
    };
    walk_layers<CLN, SaveIn>(1 + ty, zL, load, apply);
  }
  s_first[0][ty][cx] = fz; s_first[1][ty][cx] = fu; s_first[2][ty][cx] = fv;
  __syncthreads();
  if (act && ty == 0) {
    int kz = km1, ku = km1, kv = km1;
#pragma unroll
    for (int q = 0; q < CLN; ++q) {
      kz = min(kz, s_first[0][q][cx]); ku = min(ku, s_first[1][q][cx]); kv = min(kv, s_first[2][q][cx]);
    }
    d.s.k1z[l - 1] = kz; d.s.k1u[l - 1] = ku; d.s.k1v[l - 1] = kv;
  }
}

// Initial density anomaly on every column incl. the sentinel (si3d_procedures.f90:363-373)
__global__ void k_density_init(Dev d) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm1) return;
  for (int k = d.g.k1; k <= d.g.km1; ++k) {
    const int ik = IX(d, k, l);
    d.f.rhop[ik] = densty_s(d.f.salp[ik], 0.00004, zmid(d, k, d.f.hp[ik])) - 1000.;
  }
}

// Batched two-right-hand-side Thomas solver (trid) for the C-ABI unit entry point.
__global__ void k_column_tridiag(int n, int nsys, const double* a, const double* b, const double* c,
                                 const double* g, const double* r, double* ag, double* ar, double* c1) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  // element k of system s at k*nsys + s (layer-major, coalesced); the host transposes
  double cp = 0, dp = 0, ep = 0;
  for (int k = 0; k < n; ++k) {
    const size_t i = (size_t)k * nsys + s;
    double cv, dv, ev;
    if (k == 0) { cv = c[i] / b[i]; dv = g[i] / b[i]; ev = r[i] / b[i]; }
    else {
      const double den = b[i] - a[i] * cp;
      cv = c[i] / den; dv = (g[i] - a[i] * dp) / den; ev = (r[i] - a[i] * ep) / den;
    }
    c1[i] = cv; ag[i] = dv; ar[i] = ev;
    cp = cv; dp = dv; ep = ev;
  }
  for (int k = n - 2; k >= 0; --k) {
    const size_t i = (size_t)k * nsys + s;
    dp = ag[i] - c1[i] * dp;
    ep = ar[i] - c1[i] * ep;
    ag[i] = dp; ar[i] = ep;
  }
}

}  // namespace

static inline int grid_of(int n) { return (n + TB - 1) / TB; }

constexpr int BK_LANES = 4;   // layer lanes of the copy kernels (slayer_h, vel_uv, vel2)
constexpr int HALF_LANES = 2;   // layer lanes of k_half_level and k_save
constexpr int CONT_LANES = 8;   // layer lanes of the continuity kernels (4 and 16 measured slower)

// Shared memory of a continuity block: two planes of km1 + 1 levels x 32 columns.
static size_t cont_smem(int km1) { return 2 * (size_t)(km1 + 1) * 32 * sizeof(double); }

template <bool CONT1>
static void launch_cont(const Dev& d, cudaStream_t st) {
  k_cont<CONT_LANES, CONT1><<<(d.g.lm + 31) / 32, dim3(32, CONT_LANES), cont_smem(d.g.km1), st>>>(d);
}

// Columns deeper than 95 levels need more than the default 48 KB of dynamic shared memory in the
// continuity kernels: the limit is raised once, to what SI3D_MAXK levels need, so handles of
// different depths never lower it for one another.
int transport_init(int km1) {
  if (cont_smem(km1) <= 48 * 1024) return 0;
  const int mx = (int)cont_smem(SI3D_MAXK);
  if (cudaFuncSetAttribute(k_cont<CONT_LANES, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
      cudaFuncSetAttribute(k_cont<CONT_LANES, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess)
    return -1;
  return 0;
}

void launch_slayer_h(const Dev& d, cudaStream_t st) {
  k_slayer_h<BK_LANES><<<(d.g.lm + 31) / 32, dim3(32, BK_LANES), 0, st>>>(d);
}

void launch_vel(const Dev& d, const int* ce, int nce, const int* cn, int ncn, cudaStream_t st) {
  if (nce > 0) k_vel_uv<1, BK_LANES><<<(nce + 31) / 32, dim3(32, BK_LANES), 0, st>>>(d, ce, nce);
  if (ncn > 0) k_vel_uv<2, BK_LANES><<<(ncn + 31) / 32, dim3(32, BK_LANES), 0, st>>>(d, cn, ncn);
  launch_cont<true>(d, st);
}

void launch_exsal_imsal(const Dev& d, const Tune& tu, cudaStream_t st) {
  const int cg = (d.g.lm + 31) / 32;
  const double* sp = d.f.salpp;
  switch (tu.sal_cl) {
    case 2: k_exsal_flux<2><<<cg, dim3(32, 2), 0, st>>>(d, sp); k_exsal_rhs<2><<<cg, dim3(32, 2), 0, st>>>(d); break;
    case 4: k_exsal_flux<4><<<cg, dim3(32, 4), 0, st>>>(d, sp); k_exsal_rhs<4><<<cg, dim3(32, 4), 0, st>>>(d); break;
    default: k_exsal_flux<8><<<cg, dim3(32, 8), 0, st>>>(d, sp); k_exsal_rhs<8><<<cg, dim3(32, 8), 0, st>>>(d); break;
  }
  switch (tu.sal_nt) {
    case 64: k_imsal<64><<<(d.g.lm + 63) / 64, 64, 0, st>>>(d); break;
    case 256: k_imsal<256><<<(d.g.lm + 255) / 256, 256, 0, st>>>(d); break;
    default: k_imsal<128><<<(d.g.lm + 127) / 128, 128, 0, st>>>(d); break;
  }
}

void launch_vel2(const Dev& d, cudaStream_t st) {
  k_vel2<BK_LANES><<<(d.g.lm + 31) / 32, dim3(32, BK_LANES), 0, st>>>(d);
}

void launch_settrap(const Dev& d, cudaStream_t st) {
  k_half_zeta<<<grid_of(d.g.lm), TB, 0, st>>>(d, 1);
  k_half_level<HALF_LANES, true><<<(d.g.lm + 31) / 32, dim3(32, HALF_LANES), 0, st>>>(d);
  launch_cont<false>(d, st);
}

void launch_settrap2(const Dev& d, cudaStream_t st) {
  k_half_zeta<<<grid_of(d.g.lm), TB, 0, st>>>(d, 0);
  k_half_level<HALF_LANES, false><<<(d.g.lm + 31) / 32, dim3(32, HALF_LANES), 0, st>>>(d);
  launch_cont<false>(d, st);
}

void launch_save(const Dev& d, int istep, cudaStream_t st) {
  if (istep == 1) k_save<HALF_LANES, true><<<(d.g.lm + 31) / 32, dim3(32, HALF_LANES), 0, st>>>(d);
  else k_save<HALF_LANES, false><<<(d.g.lm + 31) / 32, dim3(32, HALF_LANES), 0, st>>>(d);
  launch_cont<false>(d, st);
}

void launch_density_init(const Dev& d, cudaStream_t st) { k_density_init<<<grid_of(d.g.lm1), TB, 0, st>>>(d); }

void launch_column_tridiag(int n, int nsys, const double* a, const double* b, const double* c, const double* g,
                           const double* r, double* ag, double* ar, double* scratch, cudaStream_t st) {
  k_column_tridiag<<<grid_of(nsys), TB, 0, st>>>(n, nsys, a, b, c, g, r, ag, ar, scratch);
}

}  // namespace si3d
