// Non-active (conservative) tracers: exTracer (si3d_procedures.f90:4090-4356) and ImTracer
// (:4359-4487) with sourcesink = 0 (srcsnk00, si3d_ecomod.f90:24-34), for all ntr tracers of a
// basin in two launches instead of 2 ntr.
//
// The reference advances the tracers one after another, each through the thread-private flux
// arrays Bth2/Bth3/Bth4 that exsal uses too.  A cell's right-hand side needs six face fluxes: its
// own east, north and upper faces, and the west, south and lower faces, which are the east face
// of the west column, the north face of the south column and the upper face of the layer below.
// Here every cell computes all six in registers, so no flux array is written per tracer: the
// velocities and thicknesses of a cell are loaded once and serve the tracers of its group, and
// each tracer costs a gather of tracerpp (neighbours mostly from L1/L2) and one store.  A
// neighbour face that the reference does not rewrite in this call (the west column is not wet at
// this layer, or the face below the bottom layer) keeps what an earlier routine left in the
// persistent flux arrays, so it is read from them, as the reference reads it; after the tracers
// the caller rewrites the persistent arrays with the last tracer's fluxes (exsal's flux kernel on
// that tracer), which is the state the reference leaves behind.
//
// The vertical solve shares one factorisation between the tracers of a group: the matrix of
// ImTracer depends on the layer thicknesses and Dv only, so a column's forward sweep computes the
// coefficients and the elimination factors once and carries kTracerGroup right-hand sides.
#include "kernels.h"

namespace si3d {
namespace {

constexpr int TR_LANES = 4;       // layer lanes per column in the right-hand-side kernel
constexpr int TR_RHS_GROUP = 4;   // tracers per block of the right-hand-side kernel
constexpr int TR_COL_NT = 64;     // threads (columns) per block of the column kernel

// One limited flux (:4172-4184): superbee C_f, then the Lax-Wendroff-corrected upwind flux.
__device__ __forceinline__ double lflux(double vel, double s1, double s2, double s3, double s4, double cf0,
                                        double twodt1, double len) {
  const double C_f = superbee(s1, s2, s3, s4, vel, cf0);
  return vel / 2. * (s3 + s2) - ((1. - C_f) * fabs(vel) + vel * vel * twodt1 / len * C_f) * (s3 - s2) / 2.;
}

// exTracer's Bex (:4317-4340) per wet cell and tracer, with ImTracer's sourcesink added (+ 0.0),
// stored in the tracer field (the column kernel then solves in place).
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_tracer_rhs(Dev d, const double* __restrict__ cpp, double* tr, int ntr,
                                                      long long stride) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  if (k1s + (int)threadIdx.y > kms) return;
  const int t0 = blockIdx.y * TR_RHS_GROUP, t1 = min(ntr, t0 + TR_RHS_GROUP);
  const int lm1 = d.g.lm1, P = d.g.P, k1 = d.g.k1, km1 = d.g.km1;
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const int lEE = NB(d.g.lEC, lE), lNN = NB(d.g.lNC, lN);
  // the west face is the east face of lW and takes its stencil from lW's own neighbours (the dry
  // column lm1 maps to itself); the south face likewise from lS's
  const int lWW = NB(d.g.lWC, lW), lWE = NB(d.g.lEC, lW), lWEE = NB(d.g.lEC, lWE);
  const int lSS = NB(d.g.lSC, lS), lSN = NB(d.g.lNC, lS), lSNN = NB(d.g.lNC, lSN);
  const bool wetW = lW != lm1, wetS = lS != lm1;
  const int k1W = d.s.k1z[lW - 1], kmW = NB(d.g.kmz, lW);
  const int k1S = d.s.k1z[lS - 1], kmS = NB(d.g.kmz, lS);
  const int dE = lE - l, dW = lW - l, dN = lN - l, dS = lS - l, dEE = lEE - l, dNN = lNN - l;
  const int dWW = lWW - l, dWE = lWE - l, dWEE = lWEE - l, dSS = lSS - l, dSN = lSN - l, dSNN = lSNN - l;
  const double twodt1 = d.p.twodt * d.tz;
  const double dx = d.p.dx, dy = d.p.dy;
  const bool ihd = d.p.ihd > 0;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ hp = d.f.hp;
  const double* __restrict__ hup = d.f.hup;
  const double* __restrict__ hvp = d.f.hvp;
  const double* __restrict__ uhpp = d.f.uhpp;
  const double* __restrict__ uh = d.f.uh;
  const double* __restrict__ vhpp = d.f.vhpp;
  const double* __restrict__ vh = d.f.vh;
  const double* __restrict__ wp = d.f.wp;
  const double* __restrict__ B2 = d.f.Bth2;
  const double* __restrict__ B3 = d.f.Bth3;
  const double* __restrict__ B4 = d.f.Bth4;
  for (int k = k1s + threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const int ikUU = IX(d, k - 2 < 1 ? 1 : k - 2, l);
    const int ikDD = IX(d, k + 2 > km1 ? km1 : k + 2, l);
    // ---- what the tracers of the group share
    const double huE = hup[ik], huW = hup[ik + dW], hvN = hvp[ik], hvS = hvp[ik + dS];
    const double velE = (uhpp[ik] + uh[ik]) / 2., velW = (uhpp[ik + dW] + uh[ik + dW]) / 2.;
    const double velN = (vhpp[ik] + vh[ik]) / 2., velS = (vhpp[ik + dS] + vh[ik + dS]) / 2.;
    const double hpU = hp[ik - P], hpC = hp[ik], hpD = hp[ik + P];
    const double velU = (k == k1s) ? 0.0 : wp[ik], velD = wp[ik + P];
    const double gW = hpp[ik + dW], gEE = hpp[ik + dEE], gWW = hpp[ik + dWW], gWEE = hpp[ik + dWEE];
    const double gS = hpp[ik + dS], gNN = hpp[ik + dNN], gSS = hpp[ik + dSS], gSNN = hpp[ik + dSNN];
    const double gUU = hpp[ikUU], gU = hpp[ik - P], gC = hpp[ik], gD = hpp[ik + P], gDD = hpp[ikDD];
    // faces the reference rewrites in this call; the others keep the persistent values
    const bool fW = wetW && k >= k1W && k <= kmW, fS = wetS && k >= k1S && k <= kmS, fD = k < kms;
    const double b2W = fW ? 0.0 : B2[ik + dW], b4S = fS ? 0.0 : B4[ik + dS], b3D = fD ? 0.0 : B3[ik + P];
    // horizontal-diffusion coefficients Bhaxpp/Bhaypp (:4121-4124): A * hupp (hvpp) inside a
    // column's wet layers [k1, kmz], zero elsewhere and for the dry column
    double bxl = 0.0, bxW = 0.0, byl = 0.0, byS = 0.0;
    if (ihd) {
      bxl = d.p.Ax0 * d.f.hupp[ik];
      byl = d.p.Ay0 * d.f.hvpp[ik];
      if (wetW && k >= k1 && k <= kmW) bxW = d.p.Ax0 * d.f.hupp[ik + dW];
      if (wetS && k >= k1 && k <= kmS) byS = d.p.Ay0 * d.f.hvpp[ik + dS];
    }
    for (int t = t0; t < t1; ++t) {
      const double* __restrict__ c = cpp + t * stride;
      const double cC = c[ik], cE = c[ik + dE], cW = c[ik + dW], cN = c[ik + dN], cS = c[ik + dS];
      const double cEE = c[ik + dEE], cNN = c[ik + dNN], cWW = c[ik + dWW], cSS = c[ik + dSS];
      const double cWE = c[ik + dWE], cWEE = c[ik + dWEE], cSN = c[ik + dSN], cSNN = c[ik + dSNN];
      const double cU = c[ik - P], cUU = c[ikUU], cD = c[ik + P], cDD = c[ikDD];
      // EW (:4151-4184), NS (:4203-4232), UD (:4235-4313), each face as the reference's loop
      // over its owning cell computes it
      const double fE = (huE > ZERO) ? lflux(velE, (gW <= ZERO) ? cC : cW, cC, cE, (gEE <= ZERO) ? cE : cEE, 0.0,
                                             twodt1, dx)
                                     : 0.0;
      const double fWv = !fW ? b2W
                             : (huW > ZERO) ? lflux(velW, (gWW <= ZERO) ? cW : cWW, cW, cWE,
                                                    (gWEE <= ZERO) ? cWE : cWEE, 0.0, twodt1, dx)
                                            : 0.0;
      const double fN = (hvN > ZERO) ? lflux(velN, (gS <= ZERO) ? cC : cS, cC, cN, (gNN <= ZERO) ? cN : cNN, 0.0,
                                             twodt1, dy)
                                     : 0.0;
      const double fSv = !fS ? b4S
                             : (hvS > ZERO) ? lflux(velS, (gSS <= ZERO) ? cS : cSS, cS, cSN,
                                                    (gSNN <= ZERO) ? cSN : cSNN, 0.0, twodt1, dy)
                                            : 0.0;
      // hp(1, l) is never positive, so k - 2 >= 1 whenever the upper face carries a flux
      const double fU = (hpU > ZERO) ? lflux(velU, (gD <= ZERO) ? cC : cD, cC, cU,
                                             (k - 2 < 1 || gUU <= ZERO) ? cU : cUU, 1.0, twodt1, (hpC + hpU) / 2.)
                                     : 0.0;
      const double fDv = !fD ? b3D
                             : (hpC > ZERO) ? lflux(velD, (gDD <= ZERO) ? cD : cDD, cD, cC, (gU <= ZERO) ? cC : cU,
                                                    1.0, twodt1, (hpD + hpC) / 2.)
                                            : 0.0;
      double v = gC * cC / twodt1 - (fE - fWv) / dx - (fN - fSv) / dy - (fU - fDv);
      if (ihd) {
        const double hd = (bxl * (cE - cC) - bxW * (cC - cW)) / d.p.dxdx + (byl * (cN - cC) - byS * (cC - cS)) / d.p.dydy;
        v = v + hd;
      }
      tr[t * stride + ik] = v + 0.0;
    }
  }
}

__device__ __forceinline__ double clip0(double v) { return (v < 0.0) ? 0.0 : v; }

// ImTracer per column for a group of tracers: the trid1 sweep with one factorisation, the copies
// above the surface, the sediment layer kms + 1 and the clipping of negative values (:4464-4482).
// `cur` holds the values that layers without a solve keep.
template <int NT>
__global__ void __launch_bounds__(NT) k_tracer_col(Dev d, const double* __restrict__ cpp, double* tr, const double* cur,
                                                   int ntr, long long stride, double* __restrict__ scr) {
  const int l = blockIdx.x * NT + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int t0 = blockIdx.y * kTracerGroup;
  const int nt = min(kTracerGroup, ntr - t0);
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1], nw = kms - k1s + 1, k1 = d.g.k1, P = d.g.P;
  const double twodt1 = d.p.twodt * d.tz;
  const double* __restrict__ h = d.f.h;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ Dv = d.f.Dv;
  double* trg = tr + t0 * stride;
  const double* curg = cur + t0 * stride;
  const double* __restrict__ cppg = cpp + t0 * stride;
  double* __restrict__ esc = scr + (long long)blockIdx.y * d.g.km1 * P;
  if (nw >= 2) {
    const double hpp_k1 = hpp[IX(d, k1s, l)];
    auto hn = [&](int k) -> double {   // thickness at time n with the surface corrections (:4404-4408)
      if (k == k1s) return twodt1 * d.f.wp[IX(d, k1s, l)] + hpp_k1;
      if (k == k1s + 1 && hpp_k1 <= ZERO) return hpp[IX(d, k1s + 1, l)];
      return h[IX(d, k, l)];
    };
    double f[kTracerGroup];
    double hn_k = hn(k1s), e_prev = 0.0, a1 = 0.0;
    for (int k = k1s; k <= kms; ++k) {
      const int ik = IX(d, k, l);
      double a3 = 0.0, hn_kp = 0.0;
      if (k < kms) {
        hn_kp = hn(k + 1);
        a3 = -Dv[ik + P] / (hn_k + hn_kp) * 2.;
      }
      const double a2 = hn_k / twodt1 - a1 - a3;
      const double r = 1.0 / ((k == k1s) ? a2 : a2 + a1 * e_prev);
      if (k < kms) {
        e_prev = -a3 * r;
        esc[ik] = e_prev;
      }
#pragma unroll
      for (int j = 0; j < kTracerGroup; ++j) {
        if (j < nt) {
          const double ds = trg[j * stride + ik];
          f[j] = (k == k1s) ? ds * r : (ds - a1 * f[j]) * r;
          trg[j * stride + ik] = f[j];
        }
      }
      a1 = a3;   // the lower diagonal of layer k + 1 is the upper diagonal of layer k
      hn_k = hn_kp;
    }
    // back substitution on the unclipped values; the stores are clipped
    const int ikm = IX(d, kms, l);
#pragma unroll
    for (int j = 0; j < kTracerGroup; ++j)
      if (j < nt) trg[j * stride + ikm] = clip0(f[j]);
    for (int k = kms - 1; k >= k1s; --k) {
      const int ik = IX(d, k, l);
      const double e = esc[ik];
#pragma unroll
      for (int j = 0; j < kTracerGroup; ++j) {
        if (j < nt) {
          f[j] = e * f[j] + trg[j * stride + ik];
          trg[j * stride + ik] = clip0(f[j]);
        }
      }
    }
    for (int k = k1 - 1; k <= k1s - 1; ++k) {
      const int ik = IX(d, k, l);
#pragma unroll
      for (int j = 0; j < kTracerGroup; ++j)
        if (j < nt) trg[j * stride + ik] = clip0(f[j]);
    }
  } else if (nw == 1) {
    const int ik = IX(d, k1s, l);
    const double a2 = (twodt1 * d.f.wp[ik] + hpp[ik]) / twodt1;
    for (int j = 0; j < nt; ++j) trg[j * stride + ik] = clip0(trg[j * stride + ik] / a2);
    for (int k = k1 - 1; k <= k1s - 1; ++k)
      for (int j = 0; j < nt; ++j) trg[j * stride + IX(d, k, l)] = clip0(curg[j * stride + IX(d, k, l)]);
  } else {
    for (int k = k1 - 1; k <= kms; ++k)
      for (int j = 0; j < nt; ++j) trg[j * stride + IX(d, k, l)] = clip0(curg[j * stride + IX(d, k, l)]);
  }
  // sediment layer (:4468-4471): Bex(kms + 1) = hpp tracerpp / twodt1, solved with hn = hpp
  const int iks = IX(d, kms + 1, l);
  const double hs = hpp[iks];
  const double a2s = hs / twodt1;
  for (int j = 0; j < nt; ++j) trg[j * stride + iks] = clip0((hs * cppg[j * stride + iks] / twodt1 + 0.0) / a2s);
}

}  // namespace

void launch_tracers(const Dev& d, const double* cpp, double* tr, const double* cur, int ntr, long long stride,
                    double* scr, cudaStream_t st) {
  if (ntr <= 0) return;
  const dim3 g1((d.g.lm + 31) / 32, (ntr + TR_RHS_GROUP - 1) / TR_RHS_GROUP);
  k_tracer_rhs<TR_LANES><<<g1, dim3(32, TR_LANES), 0, st>>>(d, cpp, tr, ntr, stride);
  const dim3 g2((d.g.lm + TR_COL_NT - 1) / TR_COL_NT, (ntr + kTracerGroup - 1) / kTracerGroup);
  k_tracer_col<TR_COL_NT><<<g2, TR_COL_NT, 0, st>>>(d, cpp, tr, cur, ntr, stride, scr);
}

}  // namespace si3d
