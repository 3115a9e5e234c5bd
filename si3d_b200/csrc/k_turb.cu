// Mellor-Yamada 2.5 closure (iturb = 1): UpdateMixingCoefficients CASE(1:) (si3d_mixing.f90:33-298)
// with SolveTKEandLengthScale (:301-551) and tridT (:554-612), and the time levels of q2 and q2l
// (settrap_2EqTVars :727-771, settrap2_2EqTVars :775-816, save_2EqTvars :819-889).
//
// Two kernels, in FP64 and in the reference's operation order.  k_turb_cells (block = 32
// consecutive columns x CLN layer lanes) forms, cell by cell, the shear and buoyancy production from
// the eddy coefficients of time n, then the eddy coefficients of time n+1 from q2 and q2l of time n
// (a cell's production reads only its own coefficients, so they are replaced as soon as they are
// used): independent cells, so thousands of loads are in flight.  k_turb_column (one thread per
// wet column) then sums the distances from the bottom, applies the surface and out-of-column
// limits to the coefficients and solves the two tridiagonal systems for q2 and q2l over the layers
// k1s .. kms + 1 (the same off-diagonals) as tridT does (divisions, not reciprocals), both systems
// in one forward and one backward pass, each pass loading its next layer before the current
// layer's arithmetic.  Per-layer quantities the sweeps
// reuse (limited length scale, production terms, distance from the bottom, elimination factors) go
// to four scratch fields.
#include "kernels.h"

namespace si3d {
namespace {

constexpr double kKappaS = .41, kRhoAir = 1.3;
constexpr double kAvMol = 1.3e-6, kDvMol = 1.4e-7, kQ2Min = 2.e-6, kQ2lMin = 6.80236723501E-009;
constexpr double kGhMax = 2.9E-2, kGhMin = -2.8E-1;
constexpr double A_1 = 0.92, A_2 = 0.74, B_1 = 16.6, B_2 = 10.1, E_1 = 1.80, E_2 = 1.33, E_3 = 0.25, C_2 = 0.70,
                 C_3 = 0.20, Sq = 0.20;

struct TurbConst {
  double t1, t2, t3, t4, t5, b1_23;
};

template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_turb_cells(Dev d, TurbConst T, double* __restrict__ sxl,
                                                      double* __restrict__ ssp, double* __restrict__ sbp) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1], P = d.g.P;
  if (kms - k1s + 1 <= 1) return;
  const int lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l), dW = lW - l, dS = lS - l;
  const double* __restrict__ hp = d.f.hp;
  const double* __restrict__ rhop = d.f.rhop;
  const double* __restrict__ up = d.f.up;
  const double* __restrict__ vp = d.f.vp;
  const double* __restrict__ q2p = d.f.q2p;
  const double* __restrict__ q2lp = d.f.q2lp;
  double* __restrict__ Av = d.f.Av;
  double* __restrict__ Dv = d.f.Dv;
  // ---- production at time n, then the eddy coefficients (:253-277) in place of the old ones
  for (int k = k1s + 1 + (int)threadIdx.y; k <= kms; k += CLN) {
    const int ik = IX(d, k, l);
    const double hpk = hp[ik], hpu = hp[ik - P];
    const double deltaz = 0.5 * (hpu + hpk);
    const double rhoavg = 0.5 * (rhop[ik - P] + rhop[ik]) + 1000.;
    const double drhodz = (rhop[ik - P] - rhop[ik]) / deltaz;
    const double N2 = -G_GRAV / rhoavg * drhodz;
    const double dudz = 0.5 * (up[ik - P] + up[ik - P + dW] - up[ik] - up[ik + dW]) / deltaz;
    const double dvdz = 0.5 * (vp[ik - P] + vp[ik - P + dS] - vp[ik] - vp[ik + dS]) / deltaz;
    const double qp = q2p[ik], qlp = q2lp[ik];
    double xl = qlp / qp;
    if (N2 > 0.0) xl = fmin(xl, 0.53 * sqrt(qp / N2));
    sxl[ik] = xl;
    ssp[ik] = Av[ik] * (dudz * dudz + dvdz * dvdz);
    sbp[ik] = -Dv[ik] * (N2);
    const double n2 = -G_GRAV * drhodz / rhoavg;
    double x = qlp / qp;
    if (n2 > 0.0) x = fmin(x, 0.53 * sqrt(qp / n2));
    double Gh = -n2 * (x * x) / qp;
    Gh = fmax(kGhMin, fmin(kGhMax, Gh));
    const double Sh = T.t1 / (1. - Gh * T.t2);
    const double Sm = (T.t3 + Sh * Gh * T.t4) / (1. - T.t5 * Gh);
    const double Rt = sqrt(qp) * x;
    Av[ik] = Rt * Sm + kAvMol;
    Dv[ik] = Rt * Sh + kDvMol;
  }
}

__global__ void k_turb_column(Dev d, TurbConst T, double* __restrict__ sxl, double* __restrict__ ssp,
                              double* __restrict__ sbp, double* __restrict__ szb, double* __restrict__ se) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1], k1 = d.g.k1, km1 = d.g.km1, P = d.g.P;
  if (kms - k1s + 1 <= 1) return;
  const int lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l), dW = lW - l, dS = lS - l;
  const double twodt1 = d.p.twodt * d.tz;   // twodt / istep
  const double* __restrict__ hp = d.f.hp;
  const double* __restrict__ up = d.f.up;
  const double* __restrict__ vp = d.f.vp;
  const double* __restrict__ q2p = d.f.q2p;
  const double* __restrict__ q2pp = d.f.q2pp;
  const double* __restrict__ q2lp = d.f.q2lp;
  const double* __restrict__ q2lpp = d.f.q2lpp;
  double* __restrict__ q2 = d.f.q2;
  double* __restrict__ q2l = d.f.q2l;
  double* __restrict__ Av = d.f.Av;
  double* __restrict__ Dv = d.f.Dv;
  // ---- distances from the bottom (summed from the bottom up, as the reference does)
  {
    double z0 = 0.0;
    for (int k = kms; k >= k1s + 1; --k) { z0 = z0 + hp[IX(d, k, l)]; szb[IX(d, k, l)] = z0; }
  }
  if (hp[IX(d, k1s, l)] < 1.E-2) {
    const int ik = IX(d, k1s + 1, l);
    Av[ik] = fmax(Av[ik], 1.E-4);
    Dv[ik] = fmax(Dv[ik], 1.E-4);
  }
  for (int k = 1; k <= k1s; ++k) { Av[IX(d, k, l)] = 0.0; Dv[IX(d, k, l)] = 0.0; }
  for (int k = kms + 1; k <= km1; ++k) { Av[IX(d, k, l)] = 0.0; Dv[IX(d, k, l)] = 0.0; }
  // ---- boundary values: bottom and surface friction velocities squared
  const int ikb = IX(d, kms, l);
  const double ub = 0.5 * (d.f.u[ikb] + d.f.u[ikb + dW]), vb = 0.5 * (d.f.v[ikb] + d.f.v[ikb + dS]);
  const double ustar_b = d.p.cd * (ub * ub + vb * vb);
  const double usurf = 0.5 * (up[IX(d, d.s.k1u[l - 1], l)] + up[IX(d, d.s.k1u[lW - 1], lW)]);
  const double vsurf = 0.5 * (vp[IX(d, d.s.k1v[l - 1], l)] + vp[IX(d, d.s.k1v[lS - 1], lS)]);
  const double du = d.s.uair[l - 1] - usurf, dv = d.s.vair[l - 1] - vsurf;
  const double ustar_s = d.s.cdw[l - 1] * kRhoAir * (du * du + dv * dv) / 1000.;
  const double r3 = 3. / twodt1;
  // ---- the two systems over k1s .. kms + 1 (n = nw + 1 unknowns) in one pass: tridT's forward sweep
  // of each, with the elimination factors in scratch (q2's in se, q2l's in ssp, whose value at a
  // layer is dead once the layer is loaded) and the forward values in place, then both backward
  // sweeps.  The systems share the off-diagonals and most inputs; each keeps its own arithmetic.
  {
    double e0 = 0.0, f0 = 0.0, e1 = 0.0, f1 = 0.0;
    double zt = 0.0;
    // dcoeff(k1s) = Sq 0.5 (xl(k1s) + xl(k1s + 1)) sqrt(0.5 (q2p(k1s) + q2p(k1s + 1))), xl(k1s) = 0
    double dco_prev = Sq * 0.50 * (0.0 + sxl[IX(d, k1s + 1, l)]) *
                      sqrt(0.50 * (q2p[IX(d, k1s, l)] + q2p[IX(d, k1s + 1, l)]));
    // the interior layers' inputs, loaded one layer ahead of the arithmetic that uses them
    struct In { double hpk, hpu, xl, xln, qp, qpn, SP, BP, q2o, q2lo, q2loo, zb; };
    auto load = [&](int k) -> In {
      const int ik = IX(d, k, l);
      In v;
      v.hpk = hp[ik]; v.hpu = hp[ik - P]; v.xl = sxl[ik]; v.xln = (k < kms) ? sxl[ik + P] : 0.0;
      v.qp = q2p[ik]; v.qpn = q2p[ik + P]; v.SP = ssp[ik]; v.BP = sbp[ik];
      v.q2o = q2pp[ik]; v.q2lo = q2lp[ik]; v.q2loo = q2lpp[ik]; v.zb = szb[ik];
      return v;
    };
    In nxt = load(k1s + 1);
    for (int k = k1s; k <= kms + 1; ++k) {
      const int ik = IX(d, k, l);
      double a1 = 0.0, a3 = 0.0, a20 = r3, a21 = r3, ds0, ds1;
      if (k == k1s) {
        ds0 = 3. * T.b1_23 * ustar_s / twodt1;
        ds1 = 0.0;
      } else if (k == kms + 1) {
        ds0 = 3. * T.b1_23 * ustar_b / twodt1;
        ds1 = 0.0;
      } else {
        const In v = nxt;
        if (k + 1 <= kms) nxt = load(k + 1);
        const double hpk = v.hpk, hpu = v.hpu, xl = v.xl, qp = v.qp;
        const double dco = Sq * 0.50 * (xl + v.xln) * sqrt(0.50 * (qp + v.qpn));
        a3 = -dco / (hpk * 0.50 * (hpk + hpu));
        a1 = -dco_prev / (hpu * 0.50 * (hpk + hpu));
        dco_prev = dco;
        zt = zt + hpu;   // distance from the surface to the top of layer k
        const double SP = v.SP, BP = v.BP;
        // q2
        a20 = r3 - a1 - a3 + 2. * (sqrt(qp) / (B_1 * xl));
        ds0 = 4. * qp / twodt1 - v.q2o / twodt1;
        if (BP >= 0.0) ds0 = ds0 + 2. * (SP + BP);
        else { ds0 = ds0 + 2. * (SP); a20 = a20 - BP * 2. / qp; }
        // q2l
        const double wa = xl / (kKappaS * v.zb), wb = xl / (kKappaS * zt);
        a21 = r3 - a1 - a3 + sqrt(qp) / (B_1 * xl) * (1. + E_2 * (wa * wa) + E_3 * (wb * wb));
        if (BP >= 0) ds1 = xl * (E_1 * SP + E_1 * BP);
        else { ds1 = xl * (E_1 * SP); a21 = a21 - E_1 * BP / qp; }
        ds1 = ds1 + 4 * v.q2lo / twodt1 - v.q2loo / twodt1;
      }
      if (k == k1s) {
        e0 = -a3 / a20;
        f0 = ds0 / a20;
        e1 = -a3 / a21;
        f1 = ds1 / a21;
      } else {
        const double den0 = a20 + a1 * e0;
        f0 = (ds0 - a1 * f0) / den0;
        e0 = -a3 / den0;
        const double den1 = a21 + a1 * e1;
        f1 = (ds1 - a1 * f1) / den1;
        e1 = -a3 / den1;
      }
      se[ik] = e0;
      q2[ik] = f0;
      ssp[ik] = e1;
      q2l[ik] = f1;
    }
    double x0 = f0, x1 = f1;
    q2[IX(d, kms + 1, l)] = fmax(kQ2Min, x0);
    q2l[IX(d, kms + 1, l)] = fmax(kQ2lMin, x1);
    // backward sweeps, the next layer's factors and forward values loaded ahead
    double en0 = se[IX(d, kms, l)], fn0 = q2[IX(d, kms, l)];
    double en1 = ssp[IX(d, kms, l)], fn1 = q2l[IX(d, kms, l)];
    for (int k = kms; k >= k1s; --k) {
      const int ik = IX(d, k, l);
      const double ea = en0, fa = fn0, eb = en1, fb = fn1;
      if (k - 1 >= k1s) { en0 = se[ik - P]; fn0 = q2[ik - P]; en1 = ssp[ik - P]; fn1 = q2l[ik - P]; }
      x0 = ea * x0 + fa;
      q2[ik] = fmax(kQ2Min, x0);
      x1 = eb * x1 + fb;
      q2l[ik] = fmax(kQ2lMin, x1);
    }
    const double top0 = q2[IX(d, k1s, l)], top1 = q2l[IX(d, k1s, l)];
    for (int k = k1; k <= k1s - 1; ++k) { q2[IX(d, k, l)] = top0; q2l[IX(d, k, l)] = top1; }
  }
}

// settrap_2EqTVars (mode 1) and settrap2_2EqTVars (mode 2): the half level n+1/2 of q2 and q2l.
__global__ void k_turb_half(Dev d, int mode) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int kms = NB(d.g.kmz, l), k1s = d.s.k1z[l - 1], P = d.g.P;
  for (int k = d.g.k1; k <= kms; ++k) {
    const int ik = IX(d, k, l);
    if (mode == 1) { d.f.q2pp[ik] = d.f.q2p[ik]; d.f.q2lpp[ik] = d.f.q2lp[ik]; }
    d.f.q2p[ik] = 0.5 * (d.f.q2[ik] + d.f.q2pp[ik]);
    d.f.q2lp[ik] = 0.5 * (d.f.q2l[ik] + d.f.q2lpp[ik]);
  }
  if (k1s + 2 <= d.g.km1 && d.f.hpp[IX(d, k1s, l)] <= ZERO) {
    const int ik = IX(d, k1s + 1, l);
    d.f.q2lp[ik] = d.f.q2lp[ik + P];
    d.f.q2p[ik] = d.f.q2p[ik + P];
  }
}

// save_2EqTvars: the new time level becomes the current one (every layer and the dry column), and
// save's u = up, v = vp (:3695, :3843) that the bottom friction of the next step reads.
__global__ void k_turb_save(Dev d, int istep) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm1) return;
  const int km1 = d.g.km1, P = d.g.P;
  for (int k = 1; k <= km1; ++k) {
    const int ik = IX(d, k, l);
    if (istep == 1) { d.f.q2pp[ik] = d.f.q2p[ik]; d.f.q2lpp[ik] = d.f.q2lp[ik]; }
    d.f.q2p[ik] = d.f.q2[ik];
    d.f.q2lp[ik] = d.f.q2l[ik];
  }
  if (l > d.g.lm) return;
  for (int k = d.g.k1; k <= d.g.km; ++k) {
    const int ik = IX(d, k, l);
    d.f.u[ik] = d.f.up[ik];
    d.f.v[ik] = d.f.vp[ik];
  }
  const int k1s = d.s.k1z[l - 1];
  if ((istep == 1 || km1 - k1s > 1) && k1s + 2 <= km1 && d.f.hpp[IX(d, k1s, l)] <= ZERO) {
    const int ik = IX(d, k1s + 1, l);
    d.f.q2lp[ik] = d.f.q2lp[ik + P];
    d.f.q2p[ik] = d.f.q2p[ik + P];
  }
}

}  // namespace

void launch_turbulence(const Dev& d, double* scr4, cudaStream_t st) {
  TurbConst T;
  T.t1 = A_2 * (1. - 6. * A_1 / B_1);
  T.t2 = 3. * A_2 * (6. * A_1 + B_2 * (1. - C_3));
  T.t3 = pow(B_1, -1. / 3.);
  T.t4 = 9. * A_1 * (2. * A_1 + A_2 * (1. - C_2));
  T.t5 = 9. * A_1 * A_2;
  T.b1_23 = pow(B_1, 2. / 3.);
  const long long n3 = (long long)d.g.km1 * d.g.P;
  k_turb_cells<4><<<(d.g.lm + 31) / 32, dim3(32, 4), 0, st>>>(d, T, scr4, scr4 + n3, scr4 + 2 * n3);
  k_turb_column<<<(d.g.lm + 63) / 64, 64, 0, st>>>(d, T, scr4, scr4 + n3, scr4 + 2 * n3, scr4 + 3 * n3, d.scr);
}

void launch_turb_half(const Dev& d, int mode, cudaStream_t st) {
  k_turb_half<<<(d.g.lm + 127) / 128, 128, 0, st>>>(d, mode);
}

void launch_turb_save(const Dev& d, int istep, cudaStream_t st) {
  k_turb_save<<<(d.g.lm1 + 127) / 128, 128, 0, st>>>(d, istep);
}

}  // namespace si3d
