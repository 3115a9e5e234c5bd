// Oracle time loop and per-timestep routines — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
//
// FP64 restatement of si3d.f90:324-458 and of every routine `fd` calls on the hot path
// (si3d_procedures.f90).  The single-thread (num_threads = 1) semantics of the OpenMP code are
// followed: every `lhi..lhf` / `lhiW..lhf` loop covers l = 1..lm, every `*CE` loop covers the
// columns whose east neighbour is wet and every `*CN` loop the columns whose north neighbour is
// wet (ConfigThreads, si3d_procedures.f90:4490-4745); the thread-private B* arrays are the
// persistent arrays Bth2/Bth3/Bth4/Bex/... with their Bend+1 sentinel mapped to column lm1.
#include <algorithm>
#include <cmath>

#include "oracle.hpp"

#include <cstdlib>
#include <thread>
#include <vector>

namespace orc {

// Columns l = 1..lm in contiguous static chunks on SI3D_ORACLE_THREADS threads (default 1).  Like the
// reference's OpenMP strip partition, every column's work only writes that column, so the results
// do not depend on the thread count.
static int oracle_threads() {
  static const int n = [] {
    const char* e = std::getenv("SI3D_ORACLE_THREADS");
    const int v = e ? std::atoi(e) : 1;
    return v < 1 ? 1 : v;
  }();
  return n;
}

template <class F>
static void par_cols(int lm, F&& body) {
  const int nt = std::min(oracle_threads(), lm);
  if (nt <= 1) {
    for (int l = 1; l <= lm; ++l) body(l);
    return;
  }
  std::vector<std::thread> ts;
  ts.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    const int a = 1 + (int)((long long)lm * t / nt), b = (int)((long long)lm * (t + 1) / nt);
    ts.emplace_back([&body, a, b] { for (int l = a; l <= b; ++l) body(l); });
  }
  for (auto& th : ts) th.join();
}

namespace {
constexpr real ZERO = 0.0, HMIN = 0.0, g = 9.806, rhoair = 1.3;
const real pi = 3.1415926535897932;
}  // namespace

// densty_s (si3d_utils.f90:3863-3949).  salinity**(3/2) is integer division in the
// reference, i.e. salinity**1 (kept).  Powers are written as products.
real densty_s(real t, real s, real z) {
  const real t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  real densw = 999.842594 + 6.793952e-2 * t - 9.095290e-3 * t2 + 1.001685e-4 * t3 - 1.120083e-6 * t4 +
               6.536332e-9 * t5;
  real densws = densw + s * (0.824493 - 4.0899e-3 * t + 7.6438e-5 * t2 - 8.2467e-7 * t3 + 5.3875e-9 * t4) +
                s * (-5.72466e-3 + 1.0227e-4 * t - 1.6546e-6 * t2) + 4.8314e-4 * (s * s);
  real rhoguess = densws, delta = 1, rho = 0;
  int iter = 0;
  const int maxiter = 10000;
  while (delta > 1e-6 && iter < maxiter) {
    real pressureh = rhoguess * 9.806 * z;
    real pressure = 1e-5 * pressureh;
    real kw = 19652.21 + 148.4206 * t - 2.327105 * t2 + 1.360477e-2 * t3 - 5.155288e-5 * t4;
    real ks = kw + s * (54.6746 - 0.603459 * t + 1.09987e-2 * t2 - 6.1670e-5 * t3) +
              s * (7.944e-2 + 1.6483e-2 * t - 5.3009e-4 * t2);
    real k = ks + pressure * (3.239908 + 1.43713e-3 * t + 1.16092e-4 * t2 - 5.77905e-7 * t3) +
             pressure * s * (2.2838e-3 - 1.0981e-5 * t - 1.6078e-6 * t2) + 1.91075e-4 * pressure * s +
             (pressure * pressure) * (8.50935e-5 - 6.12293e-6 * t + 5.2787e-8 * t2) +
             (pressure * pressure) * s * (-9.9348e-7 + 2.0816e-8 * t + 9.1697e-10 * t2);
    rho = densws / (1 - pressure / k);
    delta = std::fabs(rho - rhoguess);
    rhoguess = rho;
    iter++;
  }
  return rho;
}

// trid (si3d_procedures.f90:3210-3289): Thomas algorithm with two right-hand sides sharing
// one factorisation.  aa is (3, km1) column-major, 1-based in k; n = km - k1 + 1.
void trid(const real* aa, const real* gv, const real* rv, real* ag, real* ar, int k1, int km, int n) {
  std::vector<real> a(n + 1), b(n + 1), c(n + 1), d(n + 1), e(n + 1), c1(n + 1), d1(n + 1), e1(n + 1),
      d2(n + 1), e2(n + 1);
  int k = 0;
  for (int kk = k1; kk <= km; ++kk) {
    ++k;
    a[k] = aa[3 * (kk - 1) + 0]; b[k] = aa[3 * (kk - 1) + 1]; c[k] = aa[3 * (kk - 1) + 2];
    d[k] = gv[kk - 1]; e[k] = rv[kk - 1];
  }
  c1[1] = c[1] / b[1]; d1[1] = d[1] / b[1]; e1[1] = e[1] / b[1];
  for (k = 2; k <= n; ++k) {
    c1[k] = c[k] / (b[k] - a[k] * c1[k - 1]);
    d1[k] = (d[k] - a[k] * d1[k - 1]) / (b[k] - a[k] * c1[k - 1]);
    e1[k] = (e[k] - a[k] * e1[k - 1]) / (b[k] - a[k] * c1[k - 1]);
  }
  d2[n] = d1[n]; e2[n] = e1[n];
  for (k = n - 1; k >= 1; --k) { d2[k] = d1[k] - c1[k] * d2[k + 1]; e2[k] = e1[k] - c1[k] * e2[k + 1]; }
  k = 0;
  for (int kk = k1; kk <= km; ++kk) { ++k; ag[kk - 1] = d2[k]; ar[kk - 1] = e2[k]; }
}

// trid1 (si3d_procedures.f90:3292-3352); sal is 1-based 1..n on return (sal[0..n-1]).
void trid1(const real* aa, const real* dsal, real* sal, int k1, int km, int n) {
  std::vector<real> a(n + 1), b(n + 1), c(n + 1), d(n + 1), e(n + 1), f(n + 1);
  int k = 0;
  for (int kk = k1; kk <= km; ++kk) {
    ++k;
    a[k] = aa[3 * (kk - 1) + 0]; b[k] = aa[3 * (kk - 1) + 1]; c[k] = aa[3 * (kk - 1) + 2]; d[k] = dsal[kk - 1];
  }
  e[1] = -c[1] / b[1];
  f[1] = d[1] / b[1];
  for (k = 2; k <= n - 1; ++k) {
    e[k] = -c[k] / (b[k] + a[k] * e[k - 1]);
    f[k] = (d[k] - a[k] * f[k - 1]) / (b[k] + a[k] * e[k - 1]);
  }
  sal[n - 1] = (d[n] - a[n] * f[n - 1]) / (b[n] + a[n] * e[n - 1]);
  for (k = n - 1; k >= 1; --k) sal[k - 1] = e[k] * sal[k] + f[k];
}

namespace {

// surfbc CASE(0) (si3d_boundaryconditions.f90:4508-4514), or the per-column override.
void surfbc(Model& m) {
  par_cols(m.lm, [&](int l) {
    if (m.wind_override) { m.uair(l) = m.uair_ovr[l - 1]; m.vair(l) = m.vair_ovr[l - 1]; }
    else { m.uair(l) = -m.in.wa * std::sin(pi * m.in.phi / 180.); m.vair(l) = -m.in.wa * std::cos(pi * m.in.phi / 180.); }
    m.cdw(l) = m.in.cw;
  });
}

// Coefficients haxpp/haypp/th/th1 as computed at the top of exmom (si3d_procedures.f90:623-681
// for x, 962-1018 for y); each is fully rewritten on every call, so they are recomputed here.
struct ExCoef { F3 haxpp, haypp, th, th1; };

void exmom(Model& m, int ieq, ExCoef& C) {
  const int km1 = m.km1, lm1 = m.lm1;
  const real twodt1 = m.twodt * m.tz;
  const Inp& p = m.in;
  F3 &haxpp = C.haxpp, &haypp = C.haypp, &th = C.th, &th1 = C.th1;
  if (ieq == 1) {
    for (int k = 1; k <= km1; ++k) { haxpp(k, lm1) = 0.0; haypp(k, lm1) = 0.0; }
    par_cols(m.lm, [&](int l) {
      int kmx = std::min(m.kmz(m.lEC(l)), m.kmz(l)), k1x = m.k1u(l);
      for (int k = 1; k <= k1x - 1 && k <= km1; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
      for (int k = kmx + 1; k <= km1; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
      int i = m.l2i(l), j = m.l2j(l);
      if (!m.mask2d(i + 1, j)) {
        for (int k = k1x; k <= kmx; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
        return;
      }
      if (p.ihd == 1)
        for (int k = k1x; k <= kmx; ++k) {
          haxpp(k, l) = p.Ax0 * std::min(m.hupp(k, m.lEC(l)), m.hupp(k, l));
          haypp(k, l) = p.Ay0 * std::min(m.hupp(k, m.lNC(l)), m.hupp(k, l));
        }
      for (int k = k1x; k <= kmx; ++k) {
        th(k, l) = m.hup(k - 1, l) / (m.hup(k - 1, l) + m.hup(k, l));
        th1(k, l) = 1. - th(k, l);
      }
      th(k1x, l) = 0.0; th1(k1x, l) = 0.0;
      th(kmx + 1, l) = 0.5; th1(kmx + 1, l) = 0.5;
    });
    par_cols(m.lm, [&](int l) {
      int kmx = std::min(m.kmz(m.lEC(l)), m.kmz(l)), k1x = m.k1u(l);
      for (int k = 1; k <= k1x - 1 && k <= km1; ++k) m.ex(k, l) = 0.0;
      for (int k = kmx + 1; k <= km1; ++k) m.ex(k, l) = 0.0;
      int i = m.l2i(l), j = m.l2j(l);
      if (!m.mask2d(i + 1, j)) { for (int k = k1x; k <= kmx; ++k) m.ex(k, l) = 0.0; return; }
      const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l), lSE = m.lSC(lE);
      for (int k = k1x; k <= kmx; ++k) {
        if (m.hp(k, l) <= ZERO || m.hp(k, lE) <= ZERO) { m.ex(k, l) = m.uhpp(k, l); return; }
        real corx = 0.25 * p.f * (m.vhp(k, lE) + m.vhp(k, l) + m.vhp(k, lSE) + m.vhp(k, lS));
        real uE = m.uhp(k, lE) + m.uhp(k, l);
        real uW = m.uhp(k, l) + m.uhp(k, lW);
        real vN = m.vhp(k, lE) + m.vhp(k, l);
        real vS = m.vhp(k, lSE) + m.vhp(k, lS);
        real wU = m.wp(k, lE) + m.wp(k, l); if (k == k1x) wU = 0.0;
        real wD = m.wp(k + 1, lE) + m.wp(k + 1, l); if (k == kmx) wD = 0.0;
        real advx = 0;
        if (p.itrmom == 1) {
          real scE = m.up(k, lE) + m.up(k, l), scW = m.up(k, lW) + m.up(k, l);
          real scN = m.up(k, lN) + m.up(k, l), scS = m.up(k, lS) + m.up(k, l);
          advx = (uE * scE - uW * scW) / m.fourdx + (vN * scN - vS * scS) / m.fourdy;
          advx = advx + (wU * (th(k, l) * m.up(k, l) + th1(k, l) * m.up(k - 1, l)) -
                         wD * (th(k + 1, l) * m.up(k + 1, l) + th1(k + 1, l) * m.up(k, l))) / 2.;
        }
        real hdx = 0.0;
        if (p.ihd == 1)
          hdx = (haypp(k, l) * (m.upp(k, lN) - m.upp(k, l)) - haypp(k, lS) * (m.upp(k, l) - m.upp(k, lS))) / m.dydy +
                (haxpp(k, l) * (m.upp(k, lE) - m.upp(k, l)) - haxpp(k, lW) * (m.upp(k, l) - m.upp(k, lW))) / m.dxdx;
        m.ex(k, l) = m.uhpp(k, l) - twodt1 * (advx * p.iadv - corx - hdx);
      }
    });
  } else {
    for (int k = 1; k <= km1; ++k) { haxpp(k, lm1) = 0.0; haypp(k, lm1) = 0.0; }
    par_cols(m.lm, [&](int l) {
      int kmy = std::min(m.kmz(m.lNC(l)), m.kmz(l)), k1y = m.k1v(l);
      for (int k = 1; k <= k1y - 1 && k <= km1; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
      for (int k = kmy + 1; k <= km1; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
      int i = m.l2i(l), j = m.l2j(l);
      if (!m.mask2d(i, j + 1)) {
        for (int k = k1y; k <= kmy; ++k) { haypp(k, l) = 0; haxpp(k, l) = 0; th(k, l) = 0; th1(k, l) = 0; }
        return;
      }
      if (p.ihd == 1)
        for (int k = k1y; k <= kmy; ++k) {
          haypp(k, l) = p.Ay0 * std::min(m.hvpp(k, m.lNC(l)), m.hvpp(k, l));
          haxpp(k, l) = p.Ax0 * std::min(m.hvpp(k, m.lEC(l)), m.hvpp(k, l));
        }
      for (int k = k1y; k <= kmy; ++k) {
        th(k, l) = m.hvp(k - 1, l) / (m.hvp(k - 1, l) + m.hvp(k, l));
        th1(k, l) = 1. - th(k, l);
      }
      th(k1y, l) = 0.0; th1(k1y, l) = 0.0;
      th(kmy + 1, l) = 0.5; th1(kmy + 1, l) = 0.5;
    });
    par_cols(m.lm, [&](int l) {
      for (int k = 1; k <= km1; ++k) m.ex(k, l) = 0.0;
      int i = m.l2i(l), j = m.l2j(l);
      if (!m.mask2d(i, j + 1)) return;
      int kmy = std::min(m.kmz(m.lNC(l)), m.kmz(l)), k1y = m.k1v(l);
      const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l), lNW = m.lWC(lN);
      for (int k = k1y; k <= kmy; ++k) {
        if (m.hp(k, l) <= ZERO || m.hp(k, lN) <= ZERO) { m.ex(k, l) = m.vhpp(k, l); return; }
        real cory = 0.25 * p.f * (m.uhp(k, lN) + m.uhp(k, l) + m.uhp(k, lNW) + m.uhp(k, lW));
        real uE = m.uhp(k, lN) + m.uhp(k, l);
        real uW = m.uhp(k, lNW) + m.uhp(k, lW);
        real vN = m.vhp(k, lN) + m.vhp(k, l);
        real vS = m.vhp(k, l) + m.vhp(k, lS);
        real wU = m.wp(k, lN) + m.wp(k, l); if (k == k1y) wU = 0.0;
        real wD = m.wp(k + 1, lN) + m.wp(k + 1, l); if (k == kmy) wD = 0.0;
        real advy = 0;
        if (p.itrmom == 1) {
          real scE = m.vp(k, lE) + m.vp(k, l), scW = m.vp(k, lW) + m.vp(k, l);
          real scN = m.vp(k, lN) + m.vp(k, l), scS = m.vp(k, lS) + m.vp(k, l);
          advy = (uE * scE - uW * scW) / m.fourdx + (vN * scN - vS * scS) / m.fourdy;
          advy = advy + (wU * (th(k, l) * m.vp(k, l) + th1(k, l) * m.vp(k - 1, l)) -
                         wD * (th(k + 1, l) * m.vp(k + 1, l) + th1(k + 1, l) * m.vp(k, l))) / 2.;
        }
        real hdy = 0.0;
        if (p.ihd == 1)
          hdy = (haypp(k, l) * (m.vpp(k, lN) - m.vpp(k, l)) - haypp(k, lS) * (m.vpp(k, l) - m.vpp(k, lS))) / m.dydy +
                (haxpp(k, l) * (m.vpp(k, lE) - m.vpp(k, l)) - haxpp(k, lW) * (m.vpp(k, l) - m.vpp(k, lW))) / m.dxdx;
        m.ex(k, l) = m.vhpp(k, l) - twodt1 * (advy * p.iadv + cory - hdy);
      }
    });
  }
  if (!m.obc.empty()) mod_exmom_openbc(m, ieq);   // MODexmom4openBCX/Y (:957, :1165)
}

// bclnc_km (si3d_procedures.f90:1633-1746); eps = EPSILON(0.0) of the working precision.
void bclnc_km(Model& m, int l, int kb, int ieq, real& huvpdrho) {
  const real eps = 2.220446049250313e-16;
  if (ieq == 1) {
    const int lE = m.lEC(l);
    real hup_plus = m.hup(kb, l) + eps, hup_minus = m.hup(kb, l) - eps;
    bool ce, cw;
    real rhop_e, rhop_w;
    if (m.hp(kb, lE) > hup_plus || m.hp(kb, lE) < hup_minus) {
      ce = true;
      real dz1 = 0.5 * (m.hp(kb - 1, lE) + m.hp(kb, lE));
      real dz2 = 0.5 * (m.hp(kb - 1, lE) + m.hup(kb, l));
      rhop_e = m.rhop(kb - 1, lE) + (dz2 / dz1) * (m.rhop(kb, lE) - m.rhop(kb - 1, lE));
    } else { ce = false; rhop_e = m.rhop(kb, lE); }
    if (m.hp(kb, l) > hup_plus || m.hp(kb, l) < hup_minus) {
      cw = true;
      real dz1 = 0.5 * (m.hp(kb - 1, l) + m.hp(kb, l));
      real dz2 = 0.5 * (m.hp(kb - 1, l) + m.hup(kb, l));
      rhop_w = m.rhop(kb - 1, l) + (dz2 / dz1) * (m.rhop(kb, l) - m.rhop(kb - 1, l));
    } else { cw = false; rhop_w = m.rhop(kb, l); }
    if (ce || cw) huvpdrho = m.gdtdx * m.hup(kb, l) * (rhop_e - rhop_w);
  } else {
    const int lN = m.lNC(l);
    real hvp_plus = m.hvp(kb, l) + eps, hvp_minus = m.hvp(kb, l) - eps;
    bool cn, cs;
    real rhop_n, rhop_s;
    if (m.hp(kb, lN) > hvp_plus || m.hp(kb, lN) < hvp_minus) {
      cn = true;
      real dz1 = 0.5 * (m.hp(kb - 1, lN) + m.hp(kb, lN));
      real dz2 = 0.5 * (m.hp(kb - 1, lN) + m.hvp(kb, l));
      rhop_n = m.rhop(kb - 1, lN) + (dz2 / dz1) * (m.rhop(kb, lN) - m.rhop(kb - 1, lN));
    } else { cn = false; rhop_n = m.rhop(kb, lN); }
    if (m.hp(kb, l) > hvp_plus || m.hp(kb, l) < hvp_minus) {
      cs = true;
      real dz1 = 0.5 * (m.hp(kb - 1, l) + m.hp(kb, l));
      real dz2 = 0.5 * (m.hp(kb - 1, l) + m.hvp(kb, l));
      rhop_s = m.rhop(kb - 1, l) + (dz2 / dz1) * (m.rhop(kb, l) - m.rhop(kb - 1, l));
    } else { cs = false; rhop_s = m.rhop(kb, l); }
    if (cn || cs) huvpdrho = m.gdtdy * m.hvp(kb, l) * (rhop_n - rhop_s);
  }
}

// matmom (si3d_procedures.f90:1176-1630) + trid.
void matmom(Model& m, int ieq) {
  const int km1 = m.km1;
  const real twodt1 = m.twodt * m.tz, tz = m.tz, theta = m.in.theta;
  const bool X = ieq == 1;
  F3 &huv = X ? m.hup : m.hvp;
  F3 &uvpp = X ? m.upp : m.vpp;
  F3 &agA = X ? m.agx : m.agy, &arA = X ? m.arx : m.ary;
  F1 &eag = X ? m.eagx : m.eagy, &ear = X ? m.earx : m.eary;
  par_cols(m.lm, [&](int l) {
    // per-thread column scratch (every entry a column reads is written for that column first)
    thread_local std::vector<real> Avx, rhopx, hupdrho, bclncx, vdiffx, Avxdudz, deltaz, hh, gg, ag, ar, aa;
    for (auto* v : {&Avx, &rhopx, &hupdrho, &bclncx, &vdiffx, &Avxdudz, &deltaz}) v->resize(km1 + 2);
    for (auto* v : {&hh, &gg, &ag, &ar}) v->resize(km1 + 1);
    aa.resize(3 * (km1 + 1));
    auto AA = [&](int r, int k) -> real& { return aa[3 * (k - 1) + (r - 1)]; };
    int i = m.l2i(l), j = m.l2j(l);
    if (X ? !m.mask2d(i + 1, j) : !m.mask2d(i, j + 1)) return;   // id_columnCE / id_columnCN
    const int lO = X ? m.lEC(l) : m.lNC(l);                         // the other side of the face
    int kmx = std::min(m.kmz(lO), m.kmz(l));
    int k1x = X ? m.k1u(l) : m.k1v(l);
    int nwlayers = (kmx - k1x) + 1;
    if (nwlayers < 1) return;
    std::fill(Avx.begin(), Avx.end(), 0.0);
    // x: k1x+1..kmx (:1269-1271); y: k1y..kmy (:1461-1463) — Avy(k1y) is never used.
    for (int k = (X ? k1x + 1 : k1x); k <= kmx; ++k) Avx[k] = 0.5 * (m.Av(k, lO) + m.Av(k, l));
    real sum = 0;
    for (int k = k1x; k <= kmx; ++k) sum += 1000 + m.rhop(k, l);
    for (int k = k1x; k <= kmx; ++k) rhopx[k] = sum / nwlayers;
    real ws0 = rhopx[k1x] * (X ? m.gdtdx : m.gdtdy) * (m.spp(lO) - m.spp(l));
    if (m.in.ibc == 0) {
      for (int k = k1x; k <= kmx; ++k) bclncx[k] = 0.0;
    } else {
      for (int k = k1x; k <= kmx; ++k)
        hupdrho[k] = (X ? m.gdtdx : m.gdtdy) * huv(k, l) * (m.rhop(k, lO) - m.rhop(k, l));
      bclncx[k1x] = hupdrho[k1x];
      if (kmx > k1x) {
        bclnc_km(m, l, kmx, ieq, hupdrho[kmx]);
        for (int k = k1x + 1; k <= kmx; ++k) {
          if (X) { real aaux = hupdrho[k - 1] + hupdrho[k]; bclncx[k] = bclncx[k - 1] + aaux; }
          else bclncx[k] = bclncx[k - 1] + hupdrho[k - 1] + hupdrho[k];
        }
      }
    }
    if (nwlayers == 1) {
      vdiffx[k1x] = 0.0;
    } else {
      for (int k = k1x + 1; k <= kmx; ++k) {
        deltaz[k] = huv(k - 1, l) + huv(k, l);
        Avxdudz[k] = Avx[k] * (uvpp(k - 1, l) - uvpp(k, l)) / deltaz[k];
      }
      Avxdudz[k1x] = 0.0;
      Avxdudz[kmx + 1] = 0.0;
      for (int k = k1x; k <= kmx; ++k) vdiffx[k] = m.twodt * (Avxdudz[k] - Avxdudz[k + 1]) * 2. * (1. - theta);
    }
    for (int k = k1x; k <= kmx; ++k) hh[k] = huv(k, l) / rhopx[k];
    for (int k = k1x; k <= kmx; ++k) gg[k] = m.ex(k, l) - hh[k] * (bclncx[k] + ws0) * tz + vdiffx[k] * tz;
    if (nwlayers == 1) {
      AA(2, k1x) = 1.0;
    } else {
      for (int k = k1x; k <= kmx - 1; ++k)
        AA(3, k) = -twodt1 * Avx[k + 1] / (huv(k + 1, l) * (huv(k, l) + huv(k + 1, l))) * 2. * theta;
      AA(3, kmx) = 0.0;
      for (int k = k1x + 1; k <= kmx; ++k)
        AA(1, k) = -twodt1 * Avx[k] / (huv(k - 1, l) * (huv(k - 1, l) + huv(k, l))) * 2. * theta;
      AA(1, k1x) = 0.0;
      for (int k = k1x; k <= kmx; ++k)
        AA(2, k) = 1.0 - (huv(k - 1, l) / huv(k, l)) * AA(1, k) - (huv(k + 1, l) / huv(k, l)) * AA(3, k);
    }
    // wind stress (:1348-1360 / :1540-1552)
    real usurf, vsurf;
    if (X) {
      const int lS = m.lSC(l), lE = m.lEC(l), lSE = m.lSC(lE);
      usurf = m.up(k1x, l);
      vsurf = (m.vp(m.k1v(l), l) + m.vp(m.k1v(lS), lS) + m.vp(m.k1v(lE), lE) + m.vp(m.k1v(lSE), lSE)) / 4.;
      real cwx = m.cdw(l) * rhoair * std::sqrt((m.vair(l) - vsurf) * (m.vair(l) - vsurf) + (m.uair(l) - usurf) * (m.uair(l) - usurf));
      real tausx = cwx / rhopx[k1x] * m.uair(l);
      gg[k1x] = gg[k1x] + tausx * twodt1;
      tausx = cwx / rhopx[k1x] / huv(k1x, l);
      AA(2, k1x) = AA(2, k1x) + tausx * twodt1;
      const real q = 0.25 * (m.vhpp(kmx, lE) + m.vhpp(kmx, l) + m.vhpp(kmx, lS) + m.vhpp(kmx, lSE));
      real taubx = m.in.cd * std::sqrt((m.uhpp(kmx, l) * m.uhpp(kmx, l)) + q * q) / (huv(kmx, l) * huv(kmx, l));
      AA(2, kmx) = AA(2, kmx) + taubx * twodt1;
    } else {
      const int lW = m.lWC(l), lN = m.lNC(l), lNW = m.lWC(lN);
      vsurf = m.vp(k1x, l);
      usurf = (m.up(m.k1u(l), l) + m.up(m.k1u(lW), lW) + m.up(m.k1u(lN), lN) + m.up(m.k1u(lNW), lNW)) / 4.;
      real cwy = m.cdw(l) * rhoair * std::sqrt((m.uair(l) - usurf) * (m.uair(l) - usurf) + (m.vair(l) - vsurf) * (m.vair(l) - vsurf));
      real tausy = cwy / rhopx[k1x] * m.vair(l);
      gg[k1x] = gg[k1x] + tausy * twodt1;
      tausy = cwy / rhopx[k1x] / huv(k1x, l);
      AA(2, k1x) = AA(2, k1x) + tausy * twodt1;
      const real q = 0.25 * (m.uhpp(kmx, lN) + m.uhpp(kmx, lNW) + m.uhpp(kmx, lW) + m.uhpp(kmx, l));
      real tauby = m.in.cd * std::sqrt((m.vhpp(kmx, l) * m.vhpp(kmx, l)) + q * q) / (huv(kmx, l) * huv(kmx, l));
      AA(2, kmx) = AA(2, kmx) + tauby * twodt1;
    }
    if (nwlayers == 1) {
      ag[k1x] = gg[k1x] / AA(2, k1x);
      ar[k1x] = hh[k1x] / AA(2, k1x);
    } else {
      trid(aa.data(), gg.data() + 1, hh.data() + 1, ag.data() + 1, ar.data() + 1, k1x, kmx, nwlayers);
    }
    real se = 0, sr = 0;
    for (int k = k1x; k <= kmx; ++k) { agA(k, l) = ag[k]; arA(k, l) = ar[k]; }
    for (int k = k1x; k <= kmx; ++k) se += ag[k];
    for (int k = k1x; k <= kmx; ++k) sr += ar[k];
    eag(l) = se; ear(l) = sr;
  });
}

// matcon (si3d_procedures.f90:1749-1867)
void matcon(Model& m) {
  const real tz = m.tz;
  const real cx = m.gdt2dx2 * tz * tz, cy = m.gdt2dy2 * tz * tz, dtdx1 = m.dtdx * tz, dtdy1 = m.dtdy * tz,
             dt1 = m.dt * tz, rho4sx = 1000., rho4sy = 1000.;
  const int lm1 = m.lm1;
  m.sx(lm1) = 0.0; m.sy(lm1) = 0.0;
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    m.sx(l) = m.mask2d(i + 1, j) ? cx * rho4sx * m.earx(l) : 0.0;
  });
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    m.sy(l) = m.mask2d(i, j + 1) ? cy * rho4sy * m.eary(l) : 0.0;
  });
  par_cols(m.lm, [&](int l) {
    int k1s = m.k1, kms = m.kmz(l);
    const int lW = m.lWC(l), lS = m.lSC(l);
    real sum = 0;
    for (int k = k1s; k <= kms; ++k)
      sum += (m.uhpp(k, l) - m.uhpp(k, lW)) / m.dx + (m.vhpp(k, l) - m.vhpp(k, lS)) / m.dy;
    m.dd(l) = dt1 * sum;
    // Beagx(lWCH(l)) with lWCH = Bend+1 -> lm1 (Beagx(Bend+1) = 0 from InitThreads and never written)
    m.qq(l) = m.spp(l) - dtdx1 * (m.eagx(l) - m.eagx(lW)) - dtdy1 * (m.eagy(l) - m.eagy(lS)) - m.dd(l);
    m.rr(l) = 1 + m.sx(l) + m.sx(lW) + m.sy(l) + m.sy(lS);
  });
  if (!m.obc.empty()) mod_qq_openbc(m);   // MODqqddrr4openBC (:1859), after rr
}

// slayer_h (si3d_procedures.f90:2070-2175)
void slayer_h(Model& m) {
  const int km1 = m.km1, lm1 = m.lm1;
  for (int k = 1; k <= km1; ++k) { m.h(k, lm1) = m.hp(k, lm1); m.hu(k, lm1) = m.hup(k, lm1); m.hv(k, lm1) = m.hvp(k, lm1); }
  par_cols(m.lm, [&](int l) {
    const int kz = m.k1z(l), ku = m.k1u(l), kv = m.k1v(l);
    for (int k = 1; k <= kz - 1; ++k) m.h(k, l) = m.hp(k, l);
    for (int k = 1; k <= ku - 1; ++k) m.hu(k, l) = m.hup(k, l);
    for (int k = 1; k <= kv - 1; ++k) m.hv(k, l) = m.hvp(k, l);
    for (int k = kz + 2; k <= km1; ++k) m.h(k, l) = m.hp(k, l);
    for (int k = ku + 1; k <= km1; ++k) m.hu(k, l) = m.hup(k, l);
    for (int k = kv + 2; k <= km1; ++k) m.hv(k, l) = m.hvp(k, l);
    int k = kz;
    real haux = std::min(m.zl(k + 1), m.hhs(l)) + m.s(l);
    if (haux <= HMIN) {
      m.h(k, l) = ZERO;
      k = k + 1;
      haux = std::min(m.zl(k + 1), m.hhs(l)) + m.s(l);
      m.h(k, l) = (haux <= HMIN) ? ZERO : haux;
    } else m.h(k, l) = haux;
    int i = m.l2i(l), j = m.l2j(l);
    const int lE = m.lEC(l), lN = m.lNC(l);
    if (m.mask2d(i + 1, j)) {
      k = ku;
      haux = std::min(m.zl(k + 1), m.hhu(l)) + std::max(m.s(l), m.s(lE));
      if (haux <= HMIN) {
        m.hu(k, l) = ZERO;
        k = k + 1; k = ku;   // the reference resets k to k1u(l) here (:2136)
        haux = std::min(m.zl(k + 1), m.hhu(l)) + std::max(m.s(l), m.s(lE));
        m.hu(k, l) = (haux <= HMIN) ? ZERO : haux;
      } else m.hu(k, l) = haux;
    } else {
      for (int kk = ku; kk <= ku + 1 && kk <= km1; ++kk) m.hu(kk, l) = m.hup(kk, l);
    }
    if (m.mask2d(i, j + 1)) {
      k = kv;
      haux = std::min(m.zl(k + 1), m.hhv(l)) + std::max(m.s(l), m.s(lN));
      if (haux <= HMIN) {
        m.hv(k, l) = ZERO;
        k = k + 1;
        haux = std::min(m.zl(k + 1), m.hhv(l)) + std::max(m.s(l), m.s(lN));
        m.hv(k, l) = (haux <= HMIN) ? ZERO : haux;
      } else m.hv(k, l) = haux;
    } else {
      for (int kk = kv; kk <= kv + 1 && kk <= km1; ++kk) m.hv(kk, l) = m.hvp(kk, l);
    }
  });
}

// SolverSparse (si3d_procedures.f90:1870-2065): ELLPACK assembly, NSPCG mic1+cg, s = zeta, slayer_h.
bool solver_sparse(Model& m) {
  const int lm = m.lm, lm1 = m.lm1;
  std::vector<real> coef((size_t)lm * 5), rhs(lm), zeta(lm);
  std::vector<int> jcoef((size_t)lm * 5);
  for (int mm = 1; mm <= lm; ++mm) {
    const int lW = m.lWC(mm), lS = m.lSC(mm);
    coef[(size_t)0 * lm + mm - 1] = m.rr(mm);
    coef[(size_t)1 * lm + mm - 1] = -m.sx(lW);
    coef[(size_t)2 * lm + mm - 1] = -m.sy(lS);
    coef[(size_t)3 * lm + mm - 1] = -m.sy(mm);
    coef[(size_t)4 * lm + mm - 1] = -m.sx(mm);
    int jc[5] = {mm, m.lWC(mm), m.lSC(mm), m.lNC(mm), m.lEC(mm)};
    for (int c = 1; c < 5; ++c) if (jc[c] == lm1) jc[c] = 0;
    for (int c = 0; c < 5; ++c) jcoef[(size_t)c * lm + mm - 1] = jc[c];
    rhs[mm - 1] = m.qq(mm);
    zeta[mm - 1] = (m.opt.x0_mode == 1) ? 0.0 : m.sp(mm);
  }
  std::vector<int> colors;
  if (m.opt.ordering == 1) {
    colors = redblack_colors(lm, coef, jcoef);
    if (colors.empty()) { m.err = "matrix lacks property A (red-black ordering impossible)"; return false; }
  }
  PcgResult r = nspcg_mic_cg(lm, coef, jcoef, rhs, zeta, m.opt, m.opt.ordering == 1 ? &colors : nullptr);
  m.solves.push_back({m.n, m.istep, m.iter, r.iters, r.ier, r.stptst, r.emin, r.emax});
  if (r.ier < 0) { m.err = "fatal error in matrix solution (ier < 0)"; return false; }
  for (int mm = 1; mm <= lm; ++mm) m.s(mm) = zeta[mm - 1];
  slayer_h(m);
  return true;
}

// continuity (si3d_procedures.f90:2635-2824), cases 1 and 2 (no point sources).
void continuity(Model& m, int ist) {
  const int km1 = m.km1;
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l), k1s = m.k1z(l);
    if (k1s > kms) return;
    const int lW = m.lWC(l), lS = m.lSC(l);
    for (int k = 1; k <= km1; ++k) m.wp(k, l) = 0.0;
    if (ist == 1) {
      for (int k = kms; k >= k1s; --k)
        m.wp(k, l) = m.wp(k + 1, l) - (m.uh(k, l) - m.uh(k, lW) + m.uhpp(k, l) - m.uhpp(k, lW)) / m.twodx -
                     (m.vh(k, l) - m.vh(k, lS) + m.vhpp(k, l) - m.vhpp(k, lS)) / m.twody;
      for (int k = m.k1; k <= k1s - 1; ++k)
        m.wp(k1s, l) = m.wp(k1s, l) - (m.uh(k, l) - m.uh(k, lW) + m.uhpp(k, l) - m.uhpp(k, lW)) / m.twodx -
                       (m.vh(k, l) - m.vh(k, lS) + m.vhpp(k, l) - m.vhpp(k, lS)) / m.twody;
    } else {
      for (int k = kms; k >= k1s; --k)
        m.wp(k, l) = m.wp(k + 1, l) - (m.uhp(k, l) - m.uhp(k, lW)) / m.dx - (m.vhp(k, l) - m.vhp(k, lS)) / m.dy;
      for (int k = m.k1; k <= k1s - 1; ++k)
        m.wp(k1s, l) = m.wp(k1s, l) - (m.uhp(k, l) - m.uhp(k, lW)) / m.dx - (m.vhp(k, l) - m.vhp(k, lS)) / m.dy;
    }
  });
  if (!m.obc.empty()) mod_vel_openbc(m);   // MODvel4openBC (:2821)
}

// vel (si3d_procedures.f90:2430-2567)
void vel(Model& m) {
  const real gthx1 = m.gdtdx * m.tz, gthy1 = m.gdtdy * m.tz, rho4cxx = 1000., rho4cyy = 1000.;
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    if (!m.mask2d(i + 1, j)) return;
    int kmx = std::min(m.kmz(m.lEC(l)), m.kmz(l)), k0x = m.k1u(l);
    real cxx = gthx1 * rho4cxx * (m.s(m.lEC(l)) - m.s(l));
    for (int k = k0x; k <= kmx; ++k) m.uh(k, l) = m.agx(k, l) - cxx * m.arx(k, l);
    int k = k0x;
    if (m.hu(k, l) <= ZERO) { m.uh(k + 1, l) = m.uh(k, l) + m.uh(k + 1, l); m.uh(k, l) = 0.0; m.k1u(l) = k0x + 1; }
  });
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    if (!m.mask2d(i, j + 1)) return;
    int kmy = std::min(m.kmz(m.lNC(l)), m.kmz(l)), k0y = m.k1v(l);
    real cyy = gthy1 * rho4cyy * (m.s(m.lNC(l)) - m.s(l));
    for (int k = k0y; k <= kmy; ++k) m.vh(k, l) = m.agy(k, l) - cyy * m.ary(k, l);
    int k = k0y;
    if (m.hv(k, l) <= ZERO) { m.vh(k + 1, l) = m.vh(k, l) + m.vh(k + 1, l); m.vh(k, l) = 0.0; m.k1v(l) = k0y + 1; }
  });
  continuity(m, 1);
  par_cols(m.lm, [&](int l) {
    int k0s = m.k1z(l);
    if (m.h(k0s, l) <= ZERO) m.k1z(l) = std::min(k0s + 1, m.km1);
  });
}

// exsal (si3d_procedures.f90:2827-3076): Superbee flux-limited advection (itrsca ignored).
void exsal(Model& m) {
  const int km1 = m.km1, lm1 = m.lm1;
  const real twodt1 = m.twodt * m.tz;
  const Inp& p = m.in;
  for (int k = 1; k <= km1; ++k) { m.Bhaxpp(k, lm1) = 0.0; m.Bhaypp(k, lm1) = 0.0; }
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l);
    for (int k = 1; k <= m.k1 - 1; ++k) { m.Bhaxpp(k, l) = 0.0; m.Bhaypp(k, l) = 0.0; }
    for (int k = kms + 1; k <= km1; ++k) { m.Bhaxpp(k, l) = 0.0; m.Bhaypp(k, l) = 0.0; }
    for (int k = m.k1; k <= kms; ++k) { m.Bhaxpp(k, l) = p.Ax0 * m.hupp(k, l); m.Bhaypp(k, l) = p.Ay0 * m.hvpp(k, l); }
  });
  for (int k = 1; k <= km1; ++k) { m.Bth3(k, lm1) = 0; m.Bex(k, lm1) = 0.0; m.Bth4(k, lm1) = 0.0; m.Bth2(k, lm1) = 0.0; }
  auto limiter = [](real ss1, real ss2, real ss3, real ss4, real vel, real cf0) {
    real C_f = cf0;
    const real ss[5] = {0, ss1, ss2, ss3, ss4};
    int gamma1 = -(int)std::copysign(1.0, vel);
    if (ss3 - ss2 != 0) {
      real ratio = (ss[3 + gamma1] - ss[2 + gamma1]) / (ss3 - ss2);
      C_f = std::max(std::max(0., std::min(1., 2. * ratio)), std::min(2., ratio));
    }
    return C_f;
  };
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l), k1s = m.k1z(l);
    const int lE = m.lEC(l), lW = m.lWC(l);
    for (int k = k1s; k <= kms; ++k) {
      if (m.hup(k, l) > ZERO) {
        real vel = (m.uhpp(k, l) + m.uh(k, l)) / 2.;
        real ss2 = m.salpp(k, l), ss3 = m.salpp(k, lE);
        real ss1 = (m.hpp(k, lW) <= ZERO) ? ss2 : m.salpp(k, lW);
        const int lEE = m.lEC(lE);
        real ss4 = (m.hpp(k, lEE) <= ZERO) ? ss3 : m.salpp(k, lEE);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 0.0);
        m.Bth2(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / m.dx * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth2(k, l) = 0.0;
    }
  });
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l), k1s = m.k1z(l);
    const int lN = m.lNC(l), lS = m.lSC(l);
    for (int k = k1s; k <= kms; ++k) {
      if (m.hvp(k, l) > ZERO) {
        real vel = (m.vhpp(k, l) + m.vh(k, l)) / 2.;
        real ss2 = m.salpp(k, l), ss3 = m.salpp(k, lN);
        real ss1 = (m.hpp(k, lS) <= ZERO) ? ss2 : m.salpp(k, lS);
        const int lNN = m.lNC(lN);
        real ss4 = (m.hpp(k, lNN) <= ZERO) ? ss3 : m.salpp(k, lNN);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 0.0);
        m.Bth4(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / m.dy * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth4(k, l) = 0.0;
      if (m.hp(k - 1, l) > ZERO) {
        real vel = m.wp(k, l); if (k == k1s) vel = 0.0;
        real ss2 = m.salpp(k, l), ss3 = m.salpp(k - 1, l);
        real ss4 = (m.hpp(k - 2, l) <= ZERO) ? ss3 : m.salpp(k - 2, l);
        real ss1 = (m.hpp(k + 1, l) <= ZERO) ? ss2 : m.salpp(k + 1, l);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 1.0);
        real delz = (m.hp(k, l) + m.hp(k - 1, l)) / 2.;
        m.Bth3(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / delz * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth3(k, l) = 0.0;
    }
  });
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l), k1s = m.k1z(l);
    const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l);
    for (int k = 1; k <= k1s - 1; ++k) m.Bex(k, l) = 0.0;
    for (int k = kms + 1; k <= km1; ++k) m.Bex(k, l) = 0.0;
    for (int k = k1s; k <= kms; ++k) {
      real hd = (m.Bhaxpp(k, l) * (m.salpp(k, lE) - m.salpp(k, l)) - m.Bhaxpp(k, lW) * (m.salpp(k, l) - m.salpp(k, lW))) / m.dxdx +
                (m.Bhaypp(k, l) * (m.salpp(k, lN) - m.salpp(k, l)) - m.Bhaypp(k, lS) * (m.salpp(k, l) - m.salpp(k, lS))) / m.dydy;
      m.Bex(k, l) = m.hpp(k, l) * m.salpp(k, l) / twodt1 - (m.Bth2(k, l) - m.Bth2(k, lW)) / m.dx -
                    (m.Bth4(k, l) - m.Bth4(k, lS)) / m.dy - (m.Bth3(k, l) - m.Bth3(k + 1, l));
      if (p.ihd > 0) m.Bex(k, l) = m.Bex(k, l) + hd;
    }
  });
}

// imsal (si3d_procedures.f90:3079-3207) + trid1
void imsal(Model& m) {
  const int km1 = m.km1;
  const real twodt1 = m.twodt * m.tz;
  par_cols(m.lm, [&](int l) {
    // per-thread column scratch (every entry a column reads is written for that column first)
    thread_local std::vector<real> hn, aa, dsal, sal1;
    hn.resize(km1 + 2); aa.resize(3 * (km1 + 1)); dsal.resize(km1 + 1); sal1.resize(km1 + 1);
    auto AA = [&](int r, int k) -> real& { return aa[3 * (k - 1) + (r - 1)]; };
    int kms = m.kmz(l), k1s = m.k1z(l), nwlayers = kms - k1s + 1;
    for (int k = k1s + 1; k <= kms; ++k) hn[k] = m.h(k, l);
    hn[k1s] = twodt1 * m.wp(k1s, l) + m.hpp(k1s, l);
    if (m.hpp(k1s, l) <= ZERO) hn[k1s + 1] = m.hpp(k1s + 1, l);
    if (nwlayers == 1) {
      AA(2, k1s) = hn[k1s] / twodt1;
      dsal[k1s] = m.Bex(k1s, l) + m.HeatSource(k1s, l);
      m.sal(k1s, l) = dsal[k1s] / AA(2, k1s);
      if (m.h(k1s, l) < 1.E-2) m.sal(k1s, l) = m.salpp(k1s, l);
    } else if (nwlayers >= 2) {
      for (int k = k1s; k <= kms - 1; ++k) AA(3, k) = -m.Dv(k + 1, l) / (hn[k] + hn[k + 1]) * 2.;
      AA(3, kms) = 0.0;
      for (int k = k1s + 1; k <= kms; ++k) AA(1, k) = -m.Dv(k, l) / (hn[k - 1] + hn[k]) * 2.;
      AA(1, k1s) = 0.0;
      for (int k = k1s; k <= kms; ++k) AA(2, k) = hn[k] / twodt1 - AA(1, k) - AA(3, k);
      for (int k = k1s; k <= kms; ++k) dsal[k] = m.Bex(k, l) + m.HeatSource(k, l);
      trid1(aa.data(), dsal.data() + 1, sal1.data() + 1, k1s, kms, nwlayers);
      for (int k = k1s; k <= kms; ++k) m.sal(k, l) = sal1[1 + k - k1s];
      for (int k = m.k1; k <= k1s - 1; ++k) m.sal(k, l) = sal1[1];
      m.sal(kms + 1, l) = m.sal(kms, l);
    }
  });
}

// exTracer (si3d_procedures.f90:4090-4356) for tracer nt, ecomod = 0: the three flux loops of
// exsal on tracerpp (no settling velocities: the suspended-sediment and water-quality species
// indices are not set for conservative tracers, so vel = wp), Bex on the wet layers and on the
// sediment layer kms + 1.  Bex and the flux arrays keep whatever an earlier routine left elsewhere.
void extracer(Model& m, int nt) {
  const int km1 = m.km1, lm1 = m.lm1;
  const real twodt1 = m.twodt * m.tz;
  const Inp& p = m.in;
  const F3& c = m.tracerpp[nt - 1];
  for (int k = 1; k <= km1; ++k) { m.Bhaxpp(k, lm1) = 0.0; m.Bhaypp(k, lm1) = 0.0; }
  par_cols(m.lm, [&](int l) {
    for (int k = m.k1; k <= m.kmz(l); ++k) { m.Bhaxpp(k, l) = p.Ax0 * m.hupp(k, l); m.Bhaypp(k, l) = p.Ay0 * m.hvpp(k, l); }
  });
  for (int k = 1; k <= km1; ++k) { m.Bth3(k, lm1) = 0.0; m.Bex(k, lm1) = 0.0; m.Bth2(k, lm1) = 0.0; m.Bth4(k, lm1) = 0.0; }
  auto limiter = [](real ss1, real ss2, real ss3, real ss4, real vel, real cf0) {
    real C_f = cf0;
    const real ss[5] = {0, ss1, ss2, ss3, ss4};
    int gamma1 = -(int)std::copysign(1.0, vel);
    if (ss3 - ss2 != 0) {
      real ratio = (ss[3 + gamma1] - ss[2 + gamma1]) / (ss3 - ss2);
      C_f = std::max(std::max(0., std::min(1., 2. * ratio)), std::min(2., ratio));
    }
    return C_f;
  };
  par_cols(m.lm, [&](int l) {
    const int kms = m.kmz(l), k1s = m.k1z(l), lE = m.lEC(l), lW = m.lWC(l), lEE = m.lEC(lE);
    for (int k = k1s; k <= kms; ++k) {
      if (m.hup(k, l) > ZERO) {
        real vel = (m.uhpp(k, l) + m.uh(k, l)) / 2.;
        real ss2 = c(k, l), ss3 = c(k, lE);
        real ss1 = (m.hpp(k, lW) <= ZERO) ? ss2 : c(k, lW);
        real ss4 = (m.hpp(k, lEE) <= ZERO) ? ss3 : c(k, lEE);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 0.0);
        m.Bth2(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / m.dx * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth2(k, l) = 0.0;
    }
  });
  par_cols(m.lm, [&](int l) {
    const int kms = m.kmz(l), k1s = m.k1z(l), lN = m.lNC(l), lS = m.lSC(l), lNN = m.lNC(lN);
    for (int k = k1s; k <= kms; ++k) {
      if (m.hvp(k, l) > ZERO) {
        real vel = (m.vhpp(k, l) + m.vh(k, l)) / 2.;
        real ss2 = c(k, l), ss3 = c(k, lN);
        real ss1 = (m.hpp(k, lS) <= ZERO) ? ss2 : c(k, lS);
        real ss4 = (m.hpp(k, lNN) <= ZERO) ? ss3 : c(k, lNN);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 0.0);
        m.Bth4(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / m.dy * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth4(k, l) = 0.0;
      if (m.hp(k - 1, l) > ZERO) {
        real vel = (k == k1s) ? 0.0 : m.wp(k, l);
        real ss2 = c(k, l), ss3 = c(k - 1, l);
        real ss4 = (m.hpp(k - 2, l) <= ZERO) ? ss3 : c(k - 2, l);
        real ss1 = (m.hpp(k + 1, l) <= ZERO) ? ss2 : c(k + 1, l);
        real C_f = limiter(ss1, ss2, ss3, ss4, vel, 1.0);
        real delz = (m.hp(k, l) + m.hp(k - 1, l)) / 2.;
        m.Bth3(k, l) = vel / 2. * (ss3 + ss2) - ((1. - C_f) * std::fabs(vel) + vel * vel * twodt1 / delz * C_f) * (ss3 - ss2) / 2.;
      } else m.Bth3(k, l) = 0.0;
    }
  });
  par_cols(m.lm, [&](int l) {
    const int kms = m.kmz(l), k1s = m.k1z(l);
    const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l);
    for (int k = k1s; k <= kms; ++k) {
      m.Bex(k, l) = m.hpp(k, l) * c(k, l) / twodt1 - (m.Bth2(k, l) - m.Bth2(k, lW)) / m.dx -
                    (m.Bth4(k, l) - m.Bth4(k, lS)) / m.dy - (m.Bth3(k, l) - m.Bth3(k + 1, l));
      if (p.ihd > 0) {
        real hd = (m.Bhaxpp(k, l) * (c(k, lE) - c(k, l)) - m.Bhaxpp(k, lW) * (c(k, l) - c(k, lW))) / m.dxdx +
                  (m.Bhaypp(k, l) * (c(k, lN) - c(k, l)) - m.Bhaypp(k, lS) * (c(k, l) - c(k, lS))) / m.dydy;
        m.Bex(k, l) = m.Bex(k, l) + hd;
      }
    }
    m.Bex(kms + 1, l) = m.hpp(kms + 1, l) * c(kms + 1, l) / twodt1;
  });
}

// ImTracer (si3d_procedures.f90:4359-4487) for tracer nt with sourcesink = 0 (srcsnk00) and no
// point sources: the implicit vertical diffusion per column (trid1), the sediment layer kms + 1,
// and negative concentrations clipped to zero from layer k1 - 1 to kms + 1.
void imtracer(Model& m, int nt) {
  const int km1 = m.km1;
  const real twodt1 = m.twodt * m.tz;
  F3& t = m.tracer[nt - 1];
  par_cols(m.lm, [&](int l) {
    thread_local std::vector<real> hn, aa, ds, sal1;
    hn.resize(km1 + 2); aa.resize(3 * (km1 + 1)); ds.resize(km1 + 1); sal1.resize(km1 + 1);
    auto AA = [&](int r, int k) -> real& { return aa[3 * (k - 1) + (r - 1)]; };
    const int kms = m.kmz(l), k1s = m.k1z(l), nwlayers = kms - k1s + 1;
    for (int k = k1s + 1; k <= kms; ++k) hn[k] = m.h(k, l);
    hn[k1s] = twodt1 * m.wp(k1s, l) + m.hpp(k1s, l);
    if (m.hpp(k1s, l) <= ZERO) hn[k1s + 1] = m.hpp(k1s + 1, l);
    if (nwlayers == 1) {
      AA(2, k1s) = hn[k1s] / twodt1;
      ds[k1s] = m.Bex(k1s, l) + 0.0;
      t(k1s, l) = ds[k1s] / AA(2, k1s);
    } else if (nwlayers >= 2) {
      for (int k = k1s; k <= kms - 1; ++k) AA(3, k) = -m.Dv(k + 1, l) / (hn[k] + hn[k + 1]) * 2.;
      AA(3, kms) = 0.0;
      for (int k = k1s + 1; k <= kms; ++k) AA(1, k) = -m.Dv(k, l) / (hn[k - 1] + hn[k]) * 2.;
      AA(1, k1s) = 0.0;
      for (int k = k1s; k <= kms; ++k) AA(2, k) = hn[k] / twodt1 - AA(1, k) - AA(3, k);
      for (int k = k1s; k <= kms; ++k) ds[k] = m.Bex(k, l) + 0.0;
      trid1(aa.data(), ds.data() + 1, sal1.data() + 1, k1s, kms, nwlayers);
      for (int k = k1s; k <= kms; ++k) t(k, l) = sal1[1 + k - k1s];
      for (int k = m.k1; k <= k1s - 1; ++k) t(k, l) = sal1[1];
      t(m.k1 - 1, l) = sal1[1];
    }
    hn[kms + 1] = m.hpp(kms + 1, l);
    const real a2 = hn[kms + 1] / twodt1;
    t(kms + 1, l) = (m.Bex(kms + 1, l) + 0.0) / a2;
    for (int k = m.k1 - 1; k <= kms + 1; ++k)
      if (t(k, l) < 0.0) t(k, l) = 0.0;
  });
}

// fd's non-active scalar block (si3d_procedures.f90:520-544) for ecomod = 0 and nopen = 0.
void tracers(Model& m) {
  for (int nt = 1; nt <= m.in.ntr; ++nt) { extracer(m, nt); imtracer(m, nt); }
}

// layer_h (si3d_procedures.f90:2181-2231)
void layer_h(Model& m) {
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l);
    for (int k = m.k1; k <= kms; ++k) {
      m.h(k, l) = std::min(m.zl(k + 1), m.hhs(l)) - std::max(m.zl(k), -m.s(l));
      if (m.h(k, l) <= HMIN) m.h(k, l) = ZERO;
    }
    int i = m.l2i(l), j = m.l2j(l);
    if (m.mask2d(i + 1, j)) {
      int kmx = std::min(m.kmz(l), m.kmz(m.lEC(l)));
      for (int k = m.k1; k <= kmx; ++k) {
        m.hu(k, l) = std::min(m.zl(k + 1), m.hhu(l)) - std::max(m.zl(k), -std::max(m.s(l), m.s(m.lEC(l))));
        if (m.hu(k, l) <= HMIN) m.hu(k, l) = ZERO;
      }
    }
    if (m.mask2d(i, j + 1)) {
      int kmy = std::min(m.kmz(l), m.kmz(m.lNC(l)));
      for (int k = m.k1; k <= kmy; ++k) {
        m.hv(k, l) = std::min(m.zl(k + 1), m.hhv(l)) - std::max(m.zl(k), -std::max(m.s(l), m.s(m.lNC(l))));
        if (m.hv(k, l) <= HMIN) m.hv(k, l) = ZERO;
      }
    }
  });
}

// layer_hp2 (si3d_procedures.f90:2238-2292)
void layer_hp2(Model& m) {
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l), kms = m.kmz(l);
    for (int k = m.k1; k <= kms; ++k) {
      m.hp(k, l) = std::min(m.zl(k + 1), m.hhs(l)) - std::max(m.zl(k), -m.sp(l));
      if (m.hp(k, l) <= HMIN) m.hp(k, l) = ZERO;
    }
    if (m.mask2d(i + 1, j)) {
      int kmx = std::min(m.kmz(l), m.kmz(m.lEC(l)));
      for (int k = m.k1; k <= kmx; ++k) {
        m.hup(k, l) = std::min(m.zl(k + 1), m.hhu(l)) - std::max(m.zl(k), -std::max(m.sp(l), m.sp(m.lEC(l))));
        if (m.hup(k, l) <= HMIN) m.hup(k, l) = ZERO;
      }
    }
    if (m.mask2d(i, j + 1)) {
      int kmy = std::min(m.kmz(l), m.kmz(m.lNC(l)));
      for (int k = m.k1; k <= kmy; ++k) {
        m.hvp(k, l) = std::min(m.zl(k + 1), m.hhv(l)) - std::max(m.zl(k), -std::max(m.sp(l), m.sp(m.lNC(l))));
        if (m.hvp(k, l) <= HMIN) m.hvp(k, l) = ZERO;
      }
    }
  });
}

// TopLayerIndexp2 (si3d_procedures.f90:2368-2427)
void top_layer_index_p2(Model& m) {
  par_cols(m.lm, [&](int l) {
    m.k1z(l) = m.km1; m.k1u(l) = m.km1; m.k1v(l) = m.km1;
    int i = m.l2i(l), j = m.l2j(l), kms = m.kmz(l);
    for (int k = m.k1; k <= kms; ++k) if (m.hp(k, l) > ZERO) { m.k1z(l) = k; break; }
    if (m.mask2d(i + 1, j)) {
      int kmx = std::min(m.kmz(l), m.kmz(m.lEC(l)));
      for (int k = m.k1; k <= kmx; ++k) if (m.hup(k, l) > ZERO) { m.k1u(l) = k; break; }
    }
    if (m.mask2d(i, j + 1)) {
      int kmy = std::min(m.kmz(l), m.kmz(m.lNC(l)));
      for (int k = m.k1; k <= kmy; ++k) if (m.hvp(k, l) > ZERO) { m.k1v(l) = k; break; }
    }
  });
}

// vel2 (si3d_procedures.f90:2570-2631)
void vel2(Model& m) {
  layer_h(m);
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    if (m.mask2d(i + 1, j)) {
      int k = m.k1u(l);
      if (m.hu(k - 1, l) > ZERO) {
        real uutemp = m.uh(k, l) / (m.hu(k, l) + m.hu(k - 1, l));
        m.uh(k, l) = uutemp * m.hu(k, l);
        m.uh(k - 1, l) = uutemp * m.hu(k - 1, l);
      }
    }
    if (m.mask2d(i, j + 1)) {
      int k = m.k1v(l);
      if (m.hv(k - 1, l) > ZERO) {
        real vvtemp = m.vh(k, l) / (m.hv(k, l) + m.hv(k - 1, l));
        m.vh(k, l) = vvtemp * m.hv(k, l);
        m.vh(k - 1, l) = vvtemp * m.hv(k - 1, l);
      }
    }
  });
}

real zmid(const Model& m, int k, int l) {
  return (m.zl(k) == -100.) ? 0.5 * m.hp(k, l) : m.zl(k) + 0.5 * m.hp(k, l);
}

// Velocity averaging to n+1/2 shared by settrap (:3481-3543) and settrap2 (:4011-4079);
// settrap additionally rotates uhpp/upp first.
void half_level_velocities(Model& m, bool rotate) {
  par_cols(m.lm, [&](int l) {
    int i = m.l2i(l), j = m.l2j(l);
    if (m.mask2d(i + 1, j)) {
      int kmx = std::min(m.kmz(l), m.kmz(m.lEC(l)));
      for (int k = m.k1; k <= kmx; ++k) {
        if (rotate) { m.uhpp(k, l) = m.uhp(k, l); m.upp(k, l) = m.up(k, l); }
        if (m.hup(k, l) > ZERO) { m.uhp(k, l) = 0.5 * (m.uh(k, l) + m.uhpp(k, l)); m.up(k, l) = m.uhp(k, l) / m.hup(k, l); }
        else { m.uhp(k, l) = 0.0; m.up(k, l) = 0.0; }
      }
      int k = m.k1u(l);
      if (m.hu(k - 1, l) > ZERO) { m.uhp(k, l) = m.uhp(k, l) + m.uh(k - 1, l) / 2.; m.up(k, l) = m.uhp(k, l) / m.hup(k, l); }
      if (m.hupp(k - 1, l) > ZERO) { m.uhp(k, l) = m.uhp(k, l) + m.uhpp(k - 1, l) / 2.; m.up(k, l) = m.uhp(k, l) / m.hup(k, l); }
    }
    if (m.mask2d(i, j + 1)) {
      int kmy = std::min(m.kmz(l), m.kmz(m.lNC(l)));
      for (int k = m.k1; k <= kmy; ++k) {
        if (rotate) { m.vhpp(k, l) = m.vhp(k, l); m.vpp(k, l) = m.vp(k, l); }
        if (m.hvp(k, l) > ZERO) { m.vhp(k, l) = 0.5 * (m.vh(k, l) + m.vhpp(k, l)); m.vp(k, l) = m.vhp(k, l) / m.hvp(k, l); }
        else { m.vhp(k, l) = 0.0; m.vp(k, l) = 0.0; }
      }
      int k = m.k1v(l);
      if (m.hv(k - 1, l) > ZERO) { m.vhp(k, l) = m.vhp(k, l) + m.vh(k - 1, l) / 2.; m.vp(k, l) = m.vhp(k, l) / m.hvp(k, l); }
      if (m.hvpp(k - 1, l) > ZERO) { m.vhp(k, l) = m.vhp(k, l) + m.vhpp(k - 1, l) / 2.; m.vp(k, l) = m.vhp(k, l) / m.hvp(k, l); }
    }
  });
}

// settrap (si3d_procedures.f90:3418-3618)
void settrap(Model& m) {
  const int km1 = m.km1, lm1 = m.lm1;
  m.spp(lm1) = m.sp(lm1);
  for (int k = 1; k <= km1; ++k) { m.hpp(k, lm1) = m.hp(k, lm1); m.hupp(k, lm1) = m.hup(k, lm1); m.hvpp(k, lm1) = m.hvp(k, lm1); }
  par_cols(m.lm, [&](int l) {
    m.spp(l) = m.sp(l);
    m.sp(l) = 0.5 * (m.s(l) + m.spp(l));
    for (int k = 1; k <= km1; ++k) { m.hpp(k, l) = m.hp(k, l); m.hupp(k, l) = m.hup(k, l); m.hvpp(k, l) = m.hvp(k, l); }
  });
  layer_hp2(m);
  top_layer_index_p2(m);
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l);
    for (int k = m.k1; k <= kms; ++k) {
      real z = zmid(m, k, l);
      m.salpp(k, l) = m.salp(k, l);
      m.salp(k, l) = (m.sal(k, l) + m.salpp(k, l)) / 2.;
      m.rhop(k, l) = densty_s(m.salp(k, l), 0.00004, z) - 1000.;
    }
  });
  half_level_velocities(m, true);
  continuity(m, 2);
  if (m.in.iturb > 0) settrap_2eq(m);   // :3612
}

// settrap2 (si3d_procedures.f90:3944-4087)
void settrap2(Model& m) {
  const int lm1 = m.lm1;
  m.sp(lm1) = 0.5 * (m.s(lm1) + m.spp(lm1));
  for (int l = 1; l <= m.lm; ++l) m.sp(l) = 0.5 * (m.s(l) + m.spp(l));
  layer_hp2(m);
  top_layer_index_p2(m);
  par_cols(m.lm, [&](int l) {
    int kms = m.kmz(l);
    for (int k = m.k1; k <= kms; ++k) {
      real z = zmid(m, k, l);
      m.salp(k, l) = (m.sal(k, l) + m.salpp(k, l)) / 2.;
      m.rhop(k, l) = densty_s(m.salp(k, l), 0.00004, z) - 1000.;
    }
  });
  half_level_velocities(m, false);
  continuity(m, 2);
  if (m.in.iturb > 0) settrap2_2eq(m);   // :4085
}

// save (si3d_procedures.f90:3621-3941)
void save(Model& m, int istep) {
  const int km1 = m.km1, lm1 = m.lm1;
  if (istep == 2) {
    m.sp(lm1) = m.s(lm1);
    for (int k = 1; k <= km1; ++k) { m.hp(k, lm1) = m.h(k, lm1); m.hup(k, lm1) = m.hu(k, lm1); m.hvp(k, lm1) = m.hv(k, lm1); }
    par_cols(m.lm, [&](int l) {
      m.sp(l) = m.s(l);
      for (int k = 1; k <= km1; ++k) { m.hp(k, l) = m.h(k, l); m.hup(k, l) = m.hu(k, l); m.hvp(k, l) = m.hv(k, l); }
    });
    top_layer_index_p2(m);
    par_cols(m.lm, [&](int l) {
      for (int k = m.k1; k <= m.km; ++k) {
        real z = zmid(m, k, l);
        m.salp(k, l) = m.sal(k, l);
        m.rhop(k, l) = densty_s(m.salp(k, l), 0.00004, z) - 1000.;
      }
      for (int k = m.k1; k <= m.km; ++k) {
        if (m.hup(k, l) > ZERO) { m.uhp(k, l) = m.uh(k, l); m.up(k, l) = m.uhp(k, l) / m.hup(k, l); m.u(k, l) = m.up(k, l); }
        else { m.uhp(k, l) = 0.0; m.up(k, l) = 0.0; m.u(k, l) = 0.0; }
      }
      for (int k = m.k1; k <= m.km; ++k) {
        if (m.hvp(k, l) > ZERO) { m.vhp(k, l) = m.vh(k, l); m.vp(k, l) = m.vhp(k, l) / m.hvp(k, l); m.v(k, l) = m.vp(k, l); }
        else { m.vhp(k, l) = 0.0; m.vp(k, l) = 0.0; m.v(k, l) = 0.0; }
      }
    });
    continuity(m, 2);
  } else {
    m.sp(lm1) = m.s(lm1);
    for (int k = 1; k <= km1; ++k) {
      m.hp(k, lm1) = m.h(k, lm1); m.hup(k, lm1) = m.hu(k, lm1); m.hvp(k, lm1) = m.hv(k, lm1);
      m.hpp(k, lm1) = m.hp(k, lm1); m.hupp(k, lm1) = m.hup(k, lm1); m.hvpp(k, lm1) = m.hvp(k, lm1);
    }
    par_cols(m.lm, [&](int l) {
      m.spp(l) = m.sp(l); m.sp(l) = m.s(l);
      for (int k = 1; k <= km1; ++k) {
        m.hpp(k, l) = m.hp(k, l); m.hupp(k, l) = m.hup(k, l); m.hvpp(k, l) = m.hvp(k, l);
        m.hp(k, l) = m.h(k, l); m.hup(k, l) = m.hu(k, l); m.hvp(k, l) = m.hv(k, l);
      }
    });
    top_layer_index_p2(m);
    par_cols(m.lm, [&](int l) {
      for (int k = m.k1; k <= m.km; ++k) {
        real z = zmid(m, k, l);
        m.salpp(k, l) = m.salp(k, l);
        m.salp(k, l) = m.sal(k, l);
        m.rhop(k, l) = densty_s(m.salp(k, l), 0.00004, z) - 1000.;
      }
      for (int k = m.k1; k <= m.km; ++k) {
        m.uhpp(k, l) = m.uhp(k, l); m.vhpp(k, l) = m.vhp(k, l); m.upp(k, l) = m.up(k, l); m.vpp(k, l) = m.vp(k, l);
      }
      for (int k = m.k1; k <= m.km; ++k) {
        if (m.hup(k, l) > ZERO) { m.uhp(k, l) = m.uh(k, l); m.up(k, l) = m.uhp(k, l) / m.hup(k, l); m.u(k, l) = m.up(k, l); }
        else { m.uhp(k, l) = 0.0; m.up(k, l) = 0.0; m.u(k, l) = 0.0; }
      }
      for (int k = m.k1; k <= m.km; ++k) {
        if (m.hvp(k, l) > ZERO) { m.vhp(k, l) = m.vh(k, l); m.vp(k, l) = m.vhp(k, l) / m.hvp(k, l); m.v(k, l) = m.vp(k, l); }
        else { m.vhp(k, l) = 0.0; m.vp(k, l) = 0.0; m.v(k, l) = 0.0; }
      }
    });
    continuity(m, 2);
  }
  if (m.in.iturb > 0) save_2eq(m, istep);   // :3769, :3924
  // both branches end with tracerpp = tracer (:3771-3774, :3926-3929)
  if (m.in.ntr > 0) m.tracerpp = m.tracer;
}

// fd (si3d_procedures.f90:382-575) for the hot-path configuration.
bool fd(Model& m, ExCoef& C) {
  m.tz = 1.0 / m.istep;
  if (!m.obc.empty() && !openbc_uvh(m)) return false;   // :423
  surfbc(m);
  exmom(m, 1, C);
  matmom(m, 1);
  exmom(m, 2, C);
  matmom(m, 2);
  matcon(m);
  if (!solver_sparse(m)) return false;
  if (!m.obc.empty() && !openbc_uvh(m)) return false;   // :482
  vel(m);
  if (m.in.isal != 0) {
    exsal(m);
    imsal(m);
    if (!m.obc.empty()) openbc_sca(m);   // :515
  }
  if (m.in.ntr > 0 && m.in.niter > 0 && m.lastiter == 1) tracers(m);
  vel2(m);
  if (m.in.ismooth >= 1 && m.istep == 1) { m.err = "ismooth>=1 is not on the hot path"; return false; }
  if (m.in.iturb == 1) update_mixing(m, m.istep);   // UpdateMixingCoefficients (:571)
  return true;
}

}  // namespace

// One routine of the time step, for stage-by-stage parity checks.
bool run_stage(Model& m, const std::string& stage, int istep) {
  ExCoef C;
  C.haxpp.init(m.km1, m.lm1); C.haypp.init(m.km1, m.lm1); C.th.init(m.km1, m.lm1); C.th1.init(m.km1, m.lm1);
  m.istep = istep;
  m.tz = 1.0 / istep;
  if (stage == "momentum") { surfbc(m); exmom(m, 1, C); matmom(m, 1); exmom(m, 2, C); matmom(m, 2); }
  else if (stage == "matcon") matcon(m);
  else if (stage == "solve") return solver_sparse(m);
  else if (stage == "vel") vel(m);
  else if (stage == "scalar") { exsal(m); imsal(m); if (!m.obc.empty()) openbc_sca(m); }
  else if (stage == "tracer") tracers(m);
  else if (stage == "turbulence") { if (m.in.iturb == 1) update_mixing(m, istep); }
  else if (stage == "vel2") vel2(m);
  else if (stage == "fd") return fd(m, C);
  else if (stage == "settrap") settrap(m);
  else if (stage == "settrap2") settrap2(m);
  else if (stage == "save") save(m, istep);
  else { m.err = "unknown stage " + stage; return false; }
  return true;
}

// Time loop si3d.f90:324-458 (logs omitted; the binary outputs outh, outz and outp are written).
bool run_steps(Model& m, int nsteps) {
  ExCoef C;
  C.haxpp.init(m.km1, m.lm1); C.haypp.init(m.km1, m.lm1); C.th.init(m.km1, m.lm1); C.th1.init(m.km1, m.lm1);
  for (int s = 0; s < nsteps; ++s) {
    m.n += 1;
    m.thrs = (double)m.n * m.in.idt / 3600.;   // its = its + idt, thrs = its / 3600. (si3d.f90:326-327)
    compute_date(m, m.in.idt);   // si3d.f90:333
    int niter1 = m.in.niter;
    m.lastiter = 0;
    bool first = (m.n == 1);
    if (first) niter1 = std::max(2, m.in.niter);
    if (!first) {
      m.istep = 1;
      m.iter = 0;
      if (m.in.itrap == 0 || (m.n % std::max(m.in.itrap, 1)) != 0) m.lastiter = 1;
      if (!fd(m, C)) { m.failed = true; return false; }
      if (m.in.itrap == 0 || (m.n % std::max(m.in.itrap, 1)) != 0) {
        save(m, m.istep);
        if (!write_outputs(m, m.n)) { m.failed = true; return false; }
        continue;
      }
      settrap(m);
    }
    m.istep = 2;
    for (int it = 1; it <= niter1; ++it) {
      m.iter = it;
      if (it == niter1) m.lastiter = 1;
      if (!fd(m, C)) { m.failed = true; return false; }
      if (it < niter1) settrap2(m);
      if (it > 20) break;
    }
    save(m, m.istep);
    if (!write_outputs(m, m.n)) { m.failed = true; return false; }
  }
  return true;
}

}  // namespace orc
