// Mellor-Yamada 2.5 closure (iturb = 1) restated for the CPU oracle — TEST INFRASTRUCTURE ONLY
// (see oracle.hpp): InitializeTurbulenceModel CASE(1) (si3d_mixing.f90:615-724), the time levels
// of q2 and q2l (settrap_2EqTVars :727-771, settrap2_2EqTVars :775-816, save_2EqTvars :819-889),
// and UpdateMixingCoefficients CASE(1:) (:33-298) with SolveTKEandLengthScale (:301-551) and tridT
// (:554-612).  Every REAL as double; the model constants (si3d_types.f90:209-219) as written.
// The subsurface fix-ups of the time-level routines copy layer k1s + 2 into k1s + 1 where the top
// cell is dry; a column with fewer than two layers below its top has no such layer and is left
// alone (the reference would read past the column).
#include <cmath>

#include "oracle.hpp"

namespace orc {

namespace {
const real ZERO = 0.0, g = 9.806, rhoair = 1.3, kappaS = .41;
const real AvMolecular = 1.3e-6, DvMolecular = 1.4e-7, q2_min = 2.e-6, q2l_min = 6.80236723501E-009;
const real Gh_max_Kc = 2.9E-2, Gh_min_Kc = -2.8E-1;
const real A_1 = 0.92, A_2 = 0.74, B_1 = 16.6, B_2 = 10.1, E_1 = 1.80, E_2 = 1.33, E_3 = 0.25, C_2 = 0.70,
           C_3 = 0.20, Sq = 0.20;
const real t_1 = A_2 * (1. - 6. * A_1 / B_1), t_2 = 3. * A_2 * (6. * A_1 + B_2 * (1. - C_3)),
           t_3 = std::pow(B_1, -1. / 3.), t_4 = 9. * A_1 * (2. * A_1 + A_2 * (1. - C_2)), t_5 = 9. * A_1 * A_2;

void subsurface_fix(Model& m, int l) {
  const int k1s = m.k1z(l);
  if (k1s + 2 > m.km1) return;
  if (m.hpp(k1s, l) <= ZERO) {
    m.q2lp(k1s + 1, l) = m.q2lp(k1s + 2, l);
    m.q2p(k1s + 1, l) = m.q2p(k1s + 2, l);
  }
}
}  // namespace

void init_turbulence(Model& m) {
  for (F3* a : {&m.q2, &m.q2p, &m.q2pp}) a->init(m.km1, m.lm1, q2_min);
  m.q2l.init(m.km1, m.lm1, 0.0);
  for (int l = 1; l <= m.lm; ++l) {
    const int kms = m.kmz(l), k1s = m.k1z(l);
    real htot = 0.0;
    for (int k = 1; k <= m.km1; ++k) htot += m.hp(k, l);
    if (kms > k1s) {
      std::vector<real> zfromt(m.km1 + 2, 0.0);
      real zfromt0 = 0.0;
      for (int k = k1s + 1; k <= kms; ++k) { zfromt0 = zfromt0 + m.hp(k - 1, l); zfromt[k] = zfromt0; }
      for (int k = k1s + 1; k <= kms; ++k) {
        const real mixl = kappaS * zfromt[k] * std::sqrt(std::max(1. - (zfromt[k] / htot), 0.0));
        m.q2l(k, l) = m.q2(k, l) * mixl;
      }
      m.q2l(k1s, l) = 0.0;
      m.q2l(kms + 1, l) = 0.0;
    }
  }
  m.q2lp = m.q2l;
  m.q2lpp = m.q2l;
}

void settrap_2eq(Model& m) {
  for (int l = 1; l <= m.lm; ++l) {
    for (int k = m.k1; k <= m.kmz(l); ++k) {
      m.q2pp(k, l) = m.q2p(k, l);
      m.q2lpp(k, l) = m.q2lp(k, l);
      m.q2p(k, l) = 0.5 * (m.q2(k, l) + m.q2pp(k, l));
      m.q2lp(k, l) = 0.5 * (m.q2l(k, l) + m.q2lpp(k, l));
    }
    subsurface_fix(m, l);
  }
}

void settrap2_2eq(Model& m) {
  for (int l = 1; l <= m.lm; ++l) {
    for (int k = m.k1; k <= m.kmz(l); ++k) {
      m.q2p(k, l) = 0.5 * (m.q2(k, l) + m.q2pp(k, l));
      m.q2lp(k, l) = 0.5 * (m.q2l(k, l) + m.q2lpp(k, l));
    }
    subsurface_fix(m, l);
  }
}

void save_2eq(Model& m, int istep) {
  for (int l = 1; l <= m.lm1; ++l) {
    for (int k = 1; k <= m.km1; ++k) {
      if (istep == 1) { m.q2pp(k, l) = m.q2p(k, l); m.q2lpp(k, l) = m.q2lp(k, l); }
      m.q2p(k, l) = m.q2(k, l);
      m.q2lp(k, l) = m.q2l(k, l);
    }
    if (l <= m.lm && (istep == 1 || m.km1 - m.k1z(l) > 1)) subsurface_fix(m, l);
  }
}

// UpdateMixingCoefficients CASE(1:) for iturb = 1: SolveTKEandLengthScale, then Av and Dv from q2
// and q2l at time n.
void update_mixing(Model& m, int istep) {
  const real twodt1 = m.twodt / istep;
  const int km1 = m.km1;
  const real B1_23 = std::pow(B_1, 2. / 3.);
  std::vector<real> zfromb(km1 + 2), zfromt(km1 + 2), xl(km1 + 2), N2(km1 + 2), ShearP(km1 + 2), BuoyP(km1 + 2),
      dcoeff(km1 + 2), ds(km1 + 2), aa(3 * (km1 + 2)), sal1(km1 + 2);
  auto AA = [&](int r, int k) -> real& { return aa[3 * (k - 1) + (r - 1)]; };
  for (int l = 1; l <= m.lm; ++l) {
    const int kms = m.kmz(l), k1s = m.k1z(l), nw = kms - k1s + 1;
    if (nw <= 1) continue;
    const int lW = m.lWC(l), lS = m.lSC(l);
    // ---- SolveTKEandLengthScale (:301-551)
    real htot = 0.0;
    for (int k = k1s; k <= kms; ++k) htot += m.hp(k, l);
    real z0 = 0.0;
    for (int k = kms; k >= k1s + 1; --k) { z0 = z0 + m.hp(k, l); zfromb[k] = z0; }
    zfromb[k1s] = htot; zfromb[kms + 1] = 0.0;
    z0 = 0.0;
    for (int k = k1s + 1; k <= kms; ++k) { z0 = z0 + m.hp(k - 1, l); zfromt[k] = z0; }
    zfromt[k1s] = 0.0; zfromt[kms + 1] = htot;
    for (int k = k1s + 1; k <= kms; ++k) xl[k] = m.q2lp(k, l) / m.q2p(k, l);
    xl[k1s] = 0.0; xl[kms + 1] = 0.0;
    for (int k = k1s + 1; k <= kms; ++k) {
      const real deltaz = 0.5 * (m.hp(k - 1, l) + m.hp(k, l));
      const real rhoavg = 0.5 * (m.rhop(k - 1, l) + m.rhop(k, l)) + 1000.;
      const real drhodz = (m.rhop(k - 1, l) - m.rhop(k, l)) / deltaz;
      N2[k] = -g / rhoavg * drhodz;
      const real dudz = 0.5 * (m.up(k - 1, l) + m.up(k - 1, lW) - m.up(k, l) - m.up(k, lW)) / deltaz;
      const real dvdz = 0.5 * (m.vp(k - 1, l) + m.vp(k - 1, lS) - m.vp(k, l) - m.vp(k, lS)) / deltaz;
      if (N2[k] > 0.0) xl[k] = std::min(xl[k], 0.53 * std::sqrt(m.q2p(k, l) / N2[k]));
      ShearP[k] = m.Av(k, l) * (dudz * dudz + dvdz * dvdz);
      BuoyP[k] = -m.Dv(k, l) * (N2[k]);
    }
    for (int k = k1s; k <= kms; ++k)
      dcoeff[k] = Sq * 0.50 * (xl[k] + xl[k + 1]) * std::sqrt(0.50 * (m.q2p(k, l) + m.q2p(k + 1, l)));
    AA(3, k1s) = 0.0;
    for (int k = k1s + 1; k <= kms; ++k) AA(3, k) = -dcoeff[k] / (m.hp(k, l) * 0.50 * (m.hp(k, l) + m.hp(k - 1, l)));
    AA(3, kms + 1) = 0.0;
    AA(1, kms + 1) = 0.0;
    for (int k = k1s + 1; k <= kms; ++k)
      AA(1, k) = -dcoeff[k - 1] / (m.hp(k - 1, l) * 0.50 * (m.hp(k, l) + m.hp(k - 1, l)));
    AA(1, k1s) = 0.0;
    AA(2, k1s) = 3. / twodt1;
    for (int k = k1s + 1; k <= kms; ++k)
      AA(2, k) = 3. / twodt1 - AA(1, k) - AA(3, k) + 2. * (std::sqrt(m.q2p(k, l)) / (B_1 * xl[k]));
    AA(2, kms + 1) = 3. / twodt1;
    for (int k = k1s + 1; k <= kms; ++k) ds[k] = 4. * m.q2p(k, l) / twodt1 - m.q2pp(k, l) / twodt1;
    for (int k = k1s + 1; k <= kms; ++k) {
      if (BuoyP[k] >= 0.0) ds[k] = ds[k] + 2. * (ShearP[k] + BuoyP[k]);
      else { ds[k] = ds[k] + 2. * (ShearP[k]); AA(2, k) = AA(2, k) - BuoyP[k] * 2. / m.q2p(k, l); }
    }
    const real ubot = 0.5 * (m.u(kms, l) + m.u(kms, lW)), vbot = 0.5 * (m.v(kms, l) + m.v(kms, lS));
    real ustar = m.in.cd * (ubot * ubot + vbot * vbot);
    ds[kms + 1] = 3. * B1_23 * ustar / twodt1;
    const real usurf = 0.5 * (m.up(m.k1u(l), l) + m.up(m.k1u(lW), lW));
    const real vsurf = 0.5 * (m.vp(m.k1v(l), l) + m.vp(m.k1v(lS), lS));
    const real du = m.uair(l) - usurf, dv = m.vair(l) - vsurf;
    ustar = m.cdw(l) * rhoair * (du * du + dv * dv) / 1000.;
    ds[k1s] = 3. * B1_23 * ustar / twodt1;
    trid1(aa.data(), ds.data() + 1, sal1.data() + 1, k1s, kms + 1, nw + 1);
    for (int k = k1s; k <= kms + 1; ++k) m.q2(k, l) = std::max(q2_min, sal1[1 + k - k1s]);
    for (int k = m.k1; k <= k1s - 1; ++k) m.q2(k, l) = m.q2(k1s, l);
    // length scale: the same off-diagonals, a wall-function diagonal
    for (int k = k1s + 1; k <= kms; ++k) {
      const real a = xl[k] / (kappaS * zfromb[k]), b = xl[k] / (kappaS * zfromt[k]);
      AA(2, k) = 3. / twodt1 - AA(1, k) - AA(3, k) +
                 std::sqrt(m.q2p(k, l)) / (B_1 * xl[k]) * (1. + E_2 * (a * a) + E_3 * (b * b));
    }
    AA(2, k1s) = 3. / twodt1;
    AA(2, kms + 1) = 3. / twodt1;
    for (int k = k1s + 1; k <= kms; ++k) {
      if (BuoyP[k] >= 0) ds[k] = xl[k] * (E_1 * ShearP[k] + E_1 * BuoyP[k]);
      else { ds[k] = xl[k] * (E_1 * ShearP[k]); AA(2, k) = AA(2, k) - E_1 * BuoyP[k] / m.q2p(k, l); }
    }
    for (int k = k1s + 1; k <= kms; ++k) ds[k] = ds[k] + 4 * m.q2lp(k, l) / twodt1 - m.q2lpp(k, l) / twodt1;
    ds[kms + 1] = 0.0;
    ds[k1s] = 0.0;
    trid1(aa.data(), ds.data() + 1, sal1.data() + 1, k1s, kms + 1, nw + 1);
    for (int k = k1s; k <= kms + 1; ++k) m.q2l(k, l) = std::max(q2l_min, sal1[1 + k - k1s]);
    for (int k = m.k1; k <= k1s - 1; ++k) m.q2l(k, l) = m.q2l(k1s, l);
    // ---- eddy coefficients at time n (:253-296)
    for (int k = k1s + 1; k <= kms; ++k) {
      const real deltaz = 0.5 * (m.hp(k - 1, l) + m.hp(k, l));
      const real rhoavg = 0.5 * (m.rhop(k - 1, l) + m.rhop(k, l)) + 1000.;
      const real drhodz = (m.rhop(k - 1, l) - m.rhop(k, l)) / deltaz;
      const real n2 = -g * drhodz / rhoavg;
      real x = m.q2lp(k, l) / m.q2p(k, l);
      if (n2 > 0.0) x = std::min(x, 0.53 * std::sqrt(m.q2p(k, l) / n2));
      real Gh = -n2 * (x * x) / m.q2p(k, l);
      Gh = std::max(Gh_min_Kc, std::min(Gh_max_Kc, Gh));
      const real Sh = t_1 / (1. - Gh * t_2);
      const real Sm = (t_3 + Sh * Gh * t_4) / (1. - t_5 * Gh);
      const real Rt = std::sqrt(m.q2p(k, l)) * x;
      m.Av(k, l) = Rt * Sm + AvMolecular;
      m.Dv(k, l) = Rt * Sh + DvMolecular;
    }
    if (m.hp(k1s, l) < 1.E-2) {
      m.Av(k1s + 1, l) = std::max(m.Av(k1s + 1, l), 1.E-4);
      m.Dv(k1s + 1, l) = std::max(m.Dv(k1s + 1, l), 1.E-4);
    }
    for (int k = 1; k <= k1s; ++k) { m.Av(k, l) = 0.0; m.Dv(k, l) = 0.0; }
    for (int k = kms + 1; k <= km1; ++k) { m.Av(k, l) = 0.0; m.Dv(k, l) = 0.0; }
  }
}

}  // namespace orc
