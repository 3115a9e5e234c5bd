// Non-active (conservative) tracers: exTracer (si3d_procedures.f90:4090-4356) and ImTracer
// (:4359-4487) with sourcesink = 0 (srcsnk00, si3d_ecomod.f90:24-34), for all ntr tracers of a
// basin in 2 ceil(ntr / kTracerFluxGroup) + 1 launches instead of 2 ntr.
//
// The reference advances the tracers one after another through the thread-private flux arrays
// Bth2/Bth3/Bth4 that exsal uses too.  Here a group of tracers at a time:
//   k_tracer_flux  each wet cell's own three face fluxes (east, north, upper) for every tracer of
//                  the group: the velocities, thicknesses and limiter directions are loaded and
//                  derived once per cell and serve the whole group, and each face is computed once
//                  (the FP64 work of the limiter is what bounds this kernel).  The fluxes go to a
//                  scratch field per tracer, except the last tracer's, which go straight into
//                  Bth2/Bth4/Bth3: that is the state the reference's last exTracer leaves there.
//   k_tracer_rhs   Bex per cell and tracer from its six faces.  A neighbour face that the
//                  reference does not rewrite in this call (the west column not wet at this layer,
//                  the face below the bottom layer) keeps what an earlier routine left in the
//                  persistent arrays, and is read from them, as the reference reads it; the
//                  persistent arrays are written in this call only at faces that are rewritten.
// and then for all tracers
//   k_tracer_col   ImTracer per column: the matrix depends on layer thicknesses and Dv only, so
//                  one forward sweep computes the coefficients and elimination factors once and
//                  carries kTracerGroup right-hand sides.
#include <algorithm>

#include "kernels.h"

namespace si3d {
namespace {

constexpr int TR_LANES = 4;       // layer lanes per column in the flux and right-hand-side kernels
constexpr int TR_COL_NT = 64;     // threads (columns) per block of the column kernel

// One face of exTracer's flux loops (:4151-4313) with the per-face quantities precomputed: the
// superbee limiter reads the far value on the upwind side (s1 when the velocity is positive, s4
// otherwise: ratio (s2 - s1) / (s3 - s2) or (s4 - s3) / (s3 - s2), gamma1 = -SIGN(1, vel)), then the
// Lax-Wendroff-corrected upwind flux with hv = vel / 2, av = |vel| and vvc = vel * vel * twodt1 / len
// (len = dx, dy or delz, the division taken once per face).
struct Face {
  double hv, av, vvc;
  bool down;
};
__device__ __forceinline__ Face face_of(double vel, double ctl) {
  return Face{vel / 2., fabs(vel), vel * vel * ctl, copysign(1.0, vel) > 0};
}
__device__ __forceinline__ double face_flux(const Face& F, double far, double s2, double s3, double cf0) {
  double C_f = cf0;
  if (s3 - s2 != 0) {
    const double ratio = F.down ? (s2 - far) / (s3 - s2) : (far - s3) / (s3 - s2);
    C_f = fmax(fmax(0., fmin(1., 2. * ratio)), fmin(2., ratio));
  }
  return F.hv * (s3 + s2) - ((1. - C_f) * F.av + F.vvc * C_f) * (s3 - s2) / 2.;
}

// exTracer's three flux loops for the tracers t0 .. t0 + nt - 1, each cell its own faces.  Tracer
// `last` (the last of all) writes into Bth2/Bth4/Bth3, the others into fx (face f of group member j
// at fx + (3 j + f) * stride).
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_tracer_flux(Dev d, const double* __restrict__ cpp, int t0, int nt,
                                                       int last, double* __restrict__ fx, long long stride) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  if (k1s + (int)threadIdx.y > kms) return;
  const int P = d.g.P;
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const int lEE = NB(d.g.lEC, lE), lNN = NB(d.g.lNC, lN);
  const int dEo = lE - l, dWo = lW - l, dNo = lN - l, dSo = lS - l, dEEo = lEE - l, dNNo = lNN - l;
  const double twodt1 = d.p.twodt * d.tz;
  const double ctx = twodt1 / d.p.dx, cty = twodt1 / d.p.dy;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ hp = d.f.hp;
  for (int k = k1s + threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const int ikUU = IX(d, k - 2 < 1 ? 1 : k - 2, l);
    // ---- per cell, for the whole group: which faces carry a flux, their velocities and the
    // upwind far cell of each (the dry test of the far cell decides between it and its neighbour)
    const bool wE = d.f.hup[ik] > ZERO, wN = d.f.hvp[ik] > ZERO;
    const double hpU = hp[ik - P], hpC = hp[ik];
    const bool wU = hpU > ZERO;
    const Face FE = face_of((d.f.uhpp[ik] + d.f.uh[ik]) / 2., ctx);
    const Face FN = face_of((d.f.vhpp[ik] + d.f.vh[ik]) / 2., cty);
    // hp(1, l) is never positive, so k - 2 >= 1 whenever the upper face carries a flux
    const Face FU = face_of((k == k1s) ? 0.0 : d.f.wp[ik], twodt1 / ((hpC + hpU) / 2.));
    // far cells: E face s1 = (k, lW) or s4 = (k, lEE); N face (k, lS) or (k, lNN); U face
    // s1 = (k + 1, l) or s4 = (k - 2, l)
    const int oE = FE.down ? dWo : dEEo, oN = FN.down ? dSo : dNNo, oU = FU.down ? P : ikUU - ik;
    const bool dryE = hpp[ik + oE] <= ZERO, dryN = hpp[ik + oN] <= ZERO;
    const bool dryU = FU.down ? hpp[ik + P] <= ZERO : (k - 2 < 1 || hpp[ikUU] <= ZERO);
    for (int j = 0; j < nt; ++j) {
      const double* __restrict__ c = cpp + (t0 + j) * stride;
      const double cC = c[ik];
      double fE = 0.0, fN = 0.0, fU = 0.0;
      if (wE) {
        const double cE = c[ik + dEo];
        const double far = dryE ? (FE.down ? cC : cE) : c[ik + oE];
        fE = face_flux(FE, far, cC, cE, 0.0);
      }
      if (wN) {
        const double cN = c[ik + dNo];
        const double far = dryN ? (FN.down ? cC : cN) : c[ik + oN];
        fN = face_flux(FN, far, cC, cN, 0.0);
      }
      if (wU) {
        const double cU = c[ik - P];
        const double far = dryU ? (FU.down ? cC : cU) : c[ik + oU];
        fU = face_flux(FU, far, cC, cU, 1.0);
      }
      if (t0 + j == last) {
        d.f.Bth2[ik] = fE;
        d.f.Bth4[ik] = fN;
        d.f.Bth3[ik] = fU;
      } else {
        fx[(3 * j + 0) * stride + ik] = fE;
        fx[(3 * j + 1) * stride + ik] = fN;
        fx[(3 * j + 2) * stride + ik] = fU;
      }
    }
  }
}

// exTracer's Bex (:4317-4340) per wet cell and tracer of the group, with ImTracer's sourcesink
// added (+ 0.0), stored in the tracer field (the column kernel then solves in place).  Divisions by
// grid constants are multiplications by their reciprocals, so values differ from the reference's
// operation order in the last bits.
template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_tracer_rhs(Dev d, const double* __restrict__ cpp, double* __restrict__ tr,
                                                      int t0, int nt, int last, const double* __restrict__ fx,
                                                      long long stride) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1];
  if (k1s + (int)threadIdx.y > kms) return;
  const int lm1 = d.g.lm1, P = d.g.P, k1 = d.g.k1;
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const bool wetW = lW != lm1, wetS = lS != lm1;
  const int k1W = d.s.k1z[lW - 1], kmW = NB(d.g.kmz, lW);
  const int k1S = d.s.k1z[lS - 1], kmS = NB(d.g.kmz, lS);
  const int dE = lE - l, dW = lW - l, dN = lN - l, dS = lS - l;
  const double twodt1 = d.p.twodt * d.tz;
  const double rt = 1.0 / twodt1, rdx = 1.0 / d.p.dx, rdy = 1.0 / d.p.dy;
  const double rdxdx = 1.0 / d.p.dxdx, rdydy = 1.0 / d.p.dydy;
  const bool ihd = d.p.ihd > 0;
  const double* __restrict__ B2 = d.f.Bth2;
  const double* __restrict__ B3 = d.f.Bth3;
  const double* __restrict__ B4 = d.f.Bth4;
  for (int k = k1s + threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const double gC = d.f.hpp[ik];
    // faces the reference rewrites in this call; the others keep the persistent values
    const bool fW = wetW && k >= k1W && k <= kmW, fS = wetS && k >= k1S && k <= kmS, fD = k < kms;
    // horizontal-diffusion coefficients Bhaxpp/Bhaypp (:4121-4124): A * hupp (hvpp) inside a
    // column's wet layers [k1, kmz], zero elsewhere and for the dry column
    double bxl = 0.0, bxW = 0.0, byl = 0.0, byS = 0.0;
    if (ihd) {
      bxl = d.p.Ax0 * d.f.hupp[ik];
      byl = d.p.Ay0 * d.f.hvpp[ik];
      if (wetW && k >= k1 && k <= kmW) bxW = d.p.Ax0 * d.f.hupp[ik + dW];
      if (wetS && k >= k1 && k <= kmS) byS = d.p.Ay0 * d.f.hvpp[ik + dS];
    }
    for (int j = 0; j < nt; ++j) {
      const double* __restrict__ c = cpp + (t0 + j) * stride;
      const bool own = t0 + j == last;
      const double* __restrict__ f2 = own ? B2 : fx + (3 * j + 0) * stride;
      const double* __restrict__ f4 = own ? B4 : fx + (3 * j + 1) * stride;
      const double* __restrict__ f3 = own ? B3 : fx + (3 * j + 2) * stride;
      const double fE = f2[ik], fN = f4[ik], fU = f3[ik];
      const double fWv = fW ? f2[ik + dW] : B2[ik + dW];
      const double fSv = fS ? f4[ik + dS] : B4[ik + dS];
      const double fDv = fD ? f3[ik + P] : B3[ik + P];
      const double cC = c[ik];
      double v = gC * cC * rt - (fE - fWv) * rdx - (fN - fSv) * rdy - (fU - fDv);
      if (ihd) {
        const double cE = c[ik + dE], cW = c[ik + dW], cN = c[ik + dN], cS = c[ik + dS];
        const double hd = (bxl * (cE - cC) - bxW * (cC - cW)) * rdxdx + (byl * (cN - cC) - byS * (cC - cS)) * rdydy;
        v = v + hd;
      }
      tr[(t0 + j) * stride + ik] = v + 0.0;
    }
  }
}

__device__ __forceinline__ double clip0(double v) { return (v < 0.0) ? 0.0 : v; }

// ImTracer per column for a group of tracers: the trid1 sweep with one factorisation, the copies
// above the surface, the sediment layer kms + 1 and the clipping of negative values (:4464-4482).
// Layers without a solve keep their tracer values: from tracerpp when keep_pp (the two are equal
// then), else from the tracer field itself.  The forward sweep stages each layer's right-hand
// sides, Dv and h through a shared-memory ring filled by cp.async RD layers ahead; the backward
// sweep loads four layers' factors and values before it stores any of them.
template <int NT>
__global__ void __launch_bounds__(NT) k_tracer_col(Dev d, const double* __restrict__ cpp, double* __restrict__ tr,
                                                   int keep_pp, int ntr, long long stride, double* __restrict__ scr) {
  constexpr int RD = 4;
  constexpr int NV = kTracerGroup + 2;
  __shared__ double ring[RD][NV][NT];   // [slot][value][thread]: a thread's slots are its own
  const int l = blockIdx.x * NT + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int tid = threadIdx.x;
  const int t0 = blockIdx.y * kTracerGroup;
  const int nt = min(kTracerGroup, ntr - t0);
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1], nw = kms - k1s + 1, k1 = d.g.k1, P = d.g.P;
  const double twodt1 = d.p.twodt * d.tz;
  const double* __restrict__ h = d.f.h;
  const double* __restrict__ hpp = d.f.hpp;
  const double* __restrict__ Dv = d.f.Dv;
  double* __restrict__ trg = tr + t0 * stride;
  const double* __restrict__ cppg = cpp + t0 * stride;
  double* __restrict__ esc = scr + (long long)blockIdx.y * d.g.km1 * P;
  if (nw >= 2) {
    const double hpp_k1 = hpp[IX(d, k1s, l)];
    // thickness at time n with the surface corrections (:4404-4408); the second layer's is the
    // only one the ring does not hold
    const double hn_top = twodt1 * d.f.wp[IX(d, k1s, l)] + hpp_k1;
    const double hn1 = (hpp_k1 <= ZERO) ? hpp[IX(d, k1s + 1, l)] : h[IX(d, k1s + 1, l)];
    auto issue = [&](int kk, int slot) {
      const int ikk = IX(d, kk, l);
      for (int j = 0; j < nt; ++j) cp_async8(&ring[slot][j][tid], &trg[j * stride + ikk]);
      cp_async8(&ring[slot][kTracerGroup][tid], &Dv[ikk + P]);
      cp_async8(&ring[slot][kTracerGroup + 1][tid], &h[ikk + P]);
    };
#pragma unroll
    for (int j = 0; j < RD; ++j) {   // one commit group per layer (empty past the bottom)
      if (k1s + j <= kms) issue(k1s + j, j);
      cp_async_commit();
    }
    double f[kTracerGroup];
    double hn_k = hn_top, e_prev = 0.0, a1 = 0.0;
    int ik = IX(d, k1s, l);
    for (int k = k1s, slot = 0; k <= kms; ++k, ik += P, slot = (slot + 1 == RD) ? 0 : slot + 1) {
      cp_async_wait<RD - 1>();   // layer k's group has landed (this thread's own copies)
      double a3 = 0.0, hn_kp = 0.0;
      if (k < kms) {
        hn_kp = (k == k1s) ? hn1 : ring[slot][kTracerGroup + 1][tid];
        a3 = -ring[slot][kTracerGroup][tid] / (hn_k + hn_kp) * 2.;
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
          const double ds = ring[slot][j][tid];
          f[j] = (k == k1s) ? ds * r : (ds - a1 * f[j]) * r;
          trg[j * stride + ik] = f[j];
        }
      }
      // refill the slot with layer k + RD (its values are consumed: the stores above use them)
      if (k + RD <= kms) issue(k + RD, slot);
      cp_async_commit();
      a1 = a3;   // the lower diagonal of layer k + 1 is the upper diagonal of layer k
      hn_k = hn_kp;
    }
    cp_async_wait<0>();
    // back substitution on the unclipped values; the stores are clipped
    const int ikm = IX(d, kms, l);
#pragma unroll
    for (int j = 0; j < kTracerGroup; ++j)
      if (j < nt) trg[j * stride + ikm] = clip0(f[j]);
    int k = kms - 1;
    for (; k - 3 >= k1s; k -= 4) {
      double e4[4], v4[4][kTracerGroup];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ikq = IX(d, k - q, l);
        e4[q] = esc[ikq];
#pragma unroll
        for (int j = 0; j < kTracerGroup; ++j) v4[q][j] = (j < nt) ? trg[j * stride + ikq] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ikq = IX(d, k - q, l);
#pragma unroll
        for (int j = 0; j < kTracerGroup; ++j) {
          if (j < nt) {
            f[j] = e4[q] * f[j] + v4[q][j];
            trg[j * stride + ikq] = clip0(f[j]);
          }
        }
      }
    }
    for (; k >= k1s; --k) {
      const int ikq = IX(d, k, l);
      const double e = esc[ikq];
#pragma unroll
      for (int j = 0; j < kTracerGroup; ++j) {
        if (j < nt) {
          f[j] = e * f[j] + trg[j * stride + ikq];
          trg[j * stride + ikq] = clip0(f[j]);
        }
      }
    }
    for (int kk = k1 - 1; kk <= k1s - 1; ++kk) {
      const int ikq = IX(d, kk, l);
#pragma unroll
      for (int j = 0; j < kTracerGroup; ++j)
        if (j < nt) trg[j * stride + ikq] = clip0(f[j]);
    }
  } else {
    // one wet layer: its solve (:4412-4416); above it (and in a dry column, every layer down to
    // kms) the values stay, clipped
    const int top = nw == 1 ? k1s - 1 : kms;
    if (nw == 1) {
      const int ik = IX(d, k1s, l);
      const double a2 = (twodt1 * d.f.wp[ik] + hpp[ik]) / twodt1;
      for (int j = 0; j < nt; ++j) trg[j * stride + ik] = clip0(trg[j * stride + ik] / a2);
    }
    for (int k = k1 - 1; k <= top; ++k) {
      const int ik = IX(d, k, l);
      for (int j = 0; j < nt; ++j) trg[j * stride + ik] = clip0(keep_pp ? cppg[j * stride + ik] : trg[j * stride + ik]);
    }
  }
  // sediment layer (:4468-4471): Bex(kms + 1) = hpp tracerpp / twodt1, solved with hn = hpp
  const int iks = IX(d, kms + 1, l);
  const double hs = hpp[iks];
  const double a2s = hs / twodt1;
  for (int j = 0; j < nt; ++j) trg[j * stride + iks] = clip0((hs * cppg[j * stride + iks] / twodt1 + 0.0) / a2s);
}

}  // namespace

void launch_tracers(const Dev& d, const double* cpp, double* tr, bool keep_pp, int ntr, long long stride,
                    double* fx, double* scr, cudaStream_t st) {
  if (ntr <= 0) return;
  const dim3 gc((d.g.lm + 31) / 32), bc(32, TR_LANES);
  for (int t0 = 0; t0 < ntr; t0 += kTracerFluxGroup) {
    const int nt = std::min(kTracerFluxGroup, ntr - t0);
    k_tracer_flux<TR_LANES><<<gc, bc, 0, st>>>(d, cpp, t0, nt, ntr - 1, fx, stride);
    k_tracer_rhs<TR_LANES><<<gc, bc, 0, st>>>(d, cpp, tr, t0, nt, ntr - 1, fx, stride);
  }
  const dim3 g2((d.g.lm + TR_COL_NT - 1) / TR_COL_NT, (ntr + kTracerGroup - 1) / kTracerGroup);
  k_tracer_col<TR_COL_NT><<<g2, TR_COL_NT, 0, st>>>(d, cpp, tr, keep_pp ? 1 : 0, ntr, stride, scr);
}

}  // namespace si3d
