// Open boundaries with a specified water-surface elevation (itype = 1) — TEST INFRASTRUCTURE ONLY
// (see oracle.hpp).
//
// Restates, in FP64 and as one thread runs them (the per-thread ranges isbcH/isbcHH/jsbcH of
// si3d.f90:195-270 then equal the input ranges):
//   openbc0 CASE(1)            si3d_boundaryconditions.f90:23-897 (series files :55-91, t = 0 :282-460)
//   openbcUVH CASE(1)          :900-970    s on the boundary cells, parabolic in time (parab)
//   MODexmom4openBCX CASE(1)   :1801-1880  west: upwind advection only; east: ex = 0 (the reference's
//                                          assignment is commented out, :1879)
//   MODexmom4openBCY CASE(1)   :2370-2510  north and south: upwind advection only
//   MODqqddrr4openBC CASE(1)   :1508-1580  the boundary value moves to the right-hand side of the
//                                          neighbouring interior cell and the face is cut (after rr)
//   MODvel4openBC CASE(1)      :2941-3010  the velocity along the boundary is zeroed and wp copied
//                                          from the interior neighbour (end of continuity, :2821)
//   openbcSCA CASE(1)          :3157-3250  temperature of the boundary cells: the boundary value on
//                                          inflow, the interior neighbour's otherwise (after imsal)
//   parab                      si3d_utils.f90:895-920
// MODexsal4openbc does nothing for CASE(1) (:3334).  Other boundary types are refused at input.
#include <cmath>
#include <cstdio>
#include <fstream>

#include "oracle.hpp"

namespace orc {

// parab (si3d_utils.f90:895-920): parabolic interpolation in a series of spacing dx from frstpt.
double parab(double frstpt, double x, const std::vector<double>& fx, double dx) {
  int m = (int)((x - frstpt) / dx);   // Fortran INTEGER assignment truncates
  const double om = m;
  double theta = (x - frstpt - om * dx) / dx;
  if (m == 0) {
    m = 2;
    theta = theta - 1.0;
  } else {
    m = m + 1;
  }
  if (m + 1 > (int)fx.size()) return std::nan("");   // past the end of the series
  auto f = [&](int i) { return fx[(size_t)(i - 1)]; };
  return f(m) + 0.5 * theta * (f(m + 1) - f(m - 1) + theta * (f(m + 1) + f(m - 1) - 2.0 * f(m)));
}

// The series of each boundary: openbcNN.txt, five header records, npts in '(10X,I7)', then npts
// records '(10X,(ntr+2)G11.2)' of which the first two values (wse, scalar) are used.
bool read_openbc_files(Model& m, const std::string& dir) {
  for (size_t nn = 1; nn <= m.obc.size(); ++nn) {
    char name[32];
    std::snprintf(name, sizeof name, nn < 10 ? "openbc0%zu.txt" : "openbc%zu.txt", nn);
    std::ifstream f(dir + "/" + name);
    if (!f) { m.err = std::string("Error opening ") + name; return false; }
    std::string line;
    for (int r = 0; r < 5; ++r) std::getline(f, line);
    std::getline(f, line);
    const int npts = line.size() > 10 ? std::atoi(line.substr(10, 7).c_str()) : 0;
    OpenBC& b = m.obc[nn - 1];
    b.wse.clear();
    b.sal.clear();
    for (int j = 0; j < npts; ++j) {
      if (!std::getline(f, line)) { m.err = std::string(name) + ": fewer records than npts"; return false; }
      auto val = [&](int c) { return line.size() > (size_t)(10 + 11 * c) ? std::atof(line.substr(10 + 11 * c, 11).c_str()) : 0.0; };
      b.wse.push_back(val(0));
      b.sal.push_back(val(1));
    }
    if (npts < 3) { m.err = std::string(name) + ": parab needs at least three records"; return false; }
  }
  return true;
}

namespace {

// Boundary cells of boundary b in the order the reference visits them.
template <class F>
void for_cells(const Model& m, const OpenBC& b, F&& f) {
  if (b.iside == 1 || b.iside == 3) {
    for (int j = b.jsbc; j <= b.jebc; ++j) f(b.isbc, j);
  } else {
    for (int i = b.isbc; i <= b.iebc; ++i) f(i, b.jsbc);
  }
}

}  // namespace

// openbc0 CASE(1): every boundary cell is wet, with a dry cell on its outer side and at least one
// wet layer; sp takes the series' first value (after init, so hp keeps the init value).
bool openbc0(Model& m) {
  for (const OpenBC& b : m.obc) {
    const double sbc = b.wse[0];
    bool ok = true;
    for_cells(m, b, [&](int i, int j) {
      if (i < 2 || j < 2 || i > m.im1 - 1 || j > m.jm1 - 1) { ok = false; return; }
      const int l = m.ij2l(i, j);
      bool outer_wet = false;
      switch (b.iside) {
        case 1: outer_wet = m.mask2d(i - 1, j); break;
        case 2: outer_wet = m.mask2d(i, j + 1); break;
        case 3: outer_wet = m.mask2d(i + 1, j); break;
        default: outer_wet = m.mask2d(i, j - 1); break;
      }
      if (!m.mask2d(i, j) || outer_wet) { ok = false; return; }
      m.sp(l) = sbc;
      if (m.kmz(l) - m.k1z(l) + 1 < 1) ok = false;
    });
    if (!ok) { m.err = "open boundary: a cell is not a wet boundary cell"; return false; }
  }
  return true;
}

bool openbc_uvh(Model& m) {
  for (const OpenBC& b : m.obc) {
    const double sbc = parab(0., m.thrs, b.wse, m.dtsec_obc / 3600.);
    if (std::isnan(sbc)) { m.err = "open-boundary series ends before the run"; return false; }
    for_cells(m, b, [&](int i, int j) { m.s(m.ij2l(i, j)) = sbc; });
  }
  return true;
}

void mod_exmom_openbc(Model& m, int ieq) {
  const double twodt1 = m.twodt * m.tz;
  const int km1 = m.km1;
  const double iadv = m.in.iadv;
  auto P = [](double a) { return a + std::fabs(a); };
  auto N = [](double a) { return a - std::fabs(a); };
  for (const OpenBC& b : m.obc) {
    if (ieq == 1 && (b.iside == 1 || b.iside == 3)) {
      const int i = b.iside == 1 ? b.isbc : b.isbc - 1;
      for (int j = b.jsbc; j <= b.jebc; ++j) {
        const int l = m.ij2l(i, j);
        const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l);
        const int kmx = std::min(m.kmz(lE), m.kmz(l)), k1x = m.k1u(l);
        if (kmx - k1x + 1 < 1) continue;
        for (int k = 1; k <= km1; ++k) m.ex(k, l) = 0.0;
        if (b.iside == 3) continue;   // east: the reference leaves ex at zero (:1879)
        for (int k = k1x; k <= kmx; ++k) {
          const double uE = m.uhp(k, lE) + m.uhp(k, l), uW = m.uhp(k, l) + m.uhp(k, l);
          const double vN = m.vhp(k, lE) + m.vhp(k, l), vS = m.vhp(k, m.lSC(lE)) + m.vhp(k, lS);
          const double wU = m.wp(k, lE) + m.wp(k, l), wD = m.wp(k + 1, lE) + m.wp(k + 1, l);
          double advx = (P(uE) * m.upp(k, l) + N(uE) * m.upp(k, lE) - P(uW) * m.upp(k, l) - N(uW) * m.upp(k, l)) / m.fourdx +
                        (P(vN) * m.upp(k, l) + N(vN) * m.upp(k, lN) - P(vS) * m.upp(k, lS) - N(vS) * m.upp(k, l)) / m.fourdy;
          advx = advx + (P(wU) * m.upp(k, l) + N(wU) * m.upp(k - 1, l)) / 4. -
                 (P(wD) * m.upp(k + 1, l) + N(wD) * m.upp(k, l)) / 4.;
          m.ex(k, l) = m.uhpp(k, l) - twodt1 * (advx * iadv);
        }
        (void)lW;
      }
    } else if (ieq == 2 && (b.iside == 2 || b.iside == 4)) {
      const int j = b.iside == 2 ? b.jsbc - 1 : b.jsbc;
      for (int i = b.isbc; i <= b.iebc; ++i) {
        const int l = m.ij2l(i, j);
        const int lE = m.lEC(l), lW = m.lWC(l), lN = m.lNC(l), lS = m.lSC(l);
        const int kmy = std::min(m.kmz(lN), m.kmz(l)), k1y = m.k1v(l);
        if (kmy - k1y + 1 < 1) continue;
        for (int k = 1; k <= km1; ++k) m.ex(k, l) = 0.0;
        for (int k = k1y; k <= kmy; ++k) {
          const double uE = m.uhp(k, lN) + m.uhp(k, l), uW = m.uhp(k, m.lWC(lN)) + m.uhp(k, lW);
          const double vN = b.iside == 2 ? m.vhp(k, l) + m.vhp(k, l) : m.vhp(k, lN) + m.vhp(k, l);
          const double vS = b.iside == 2 ? m.vhp(k, l) + m.vhp(k, lS) : m.vhp(k, l) + m.vhp(k, l);
          const double wU = m.wp(k, lN) + m.wp(k, l), wD = m.wp(k + 1, lN) + m.wp(k + 1, l);
          const double vNn = b.iside == 2 ? m.vpp(k, l) : m.vpp(k, lN);   // north: the row's own value
          const double vSs = b.iside == 2 ? m.vpp(k, lS) : m.vpp(k, l);   // south: the row's own value
          double advy = (P(uE) * m.vpp(k, l) + N(uE) * m.vpp(k, lE) - P(uW) * m.vpp(k, lW) - N(uW) * m.vpp(k, l)) / m.fourdx +
                        (P(vN) * m.vpp(k, l) + N(vN) * vNn - P(vS) * vSs - N(vS) * m.vpp(k, l)) / m.fourdy;
          advy = advy + (P(wU) * m.vpp(k, l) + N(wU) * m.vpp(k - 1, l)) / 4. -
                 (P(wD) * m.vpp(k + 1, l) + N(wD) * m.vpp(k, l)) / 4.;
          m.ex(k, l) = m.vhpp(k, l) - twodt1 * (advy * iadv);
        }
      }
    }
  }
}

void mod_qq_openbc(Model& m) {
  for (const OpenBC& b : m.obc) {
    for_cells(m, b, [&](int i, int j) {
      const int lb = m.ij2l(i, j);
      switch (b.iside) {
        case 1: { const int li = m.ij2l(i + 1, j); m.qq(li) = m.qq(li) + m.sx(lb) * m.s(lb); break; }
        case 2: { const int li = m.ij2l(i, j - 1); m.qq(li) = m.qq(li) + m.sy(li) * m.s(lb); break; }
        case 3: { const int li = m.ij2l(i - 1, j); m.qq(li) = m.qq(li) + m.sx(li) * m.s(lb); break; }
        default: { const int li = m.ij2l(i, j + 1); m.qq(li) = m.qq(li) + m.sy(lb) * m.s(lb); break; }
      }
    });
    for_cells(m, b, [&](int i, int j) {
      switch (b.iside) {
        case 1: m.sx(m.ij2l(i, j)) = 0.0; break;
        case 2: m.sy(m.ij2l(i, j - 1)) = 0.0; break;
        case 3: m.sx(m.ij2l(i - 1, j)) = 0.0; break;
        default: m.sy(m.ij2l(i, j)) = 0.0; break;
      }
    });
  }
}

void mod_vel_openbc(Model& m) {
  const int km1 = m.km1;
  for (const OpenBC& b : m.obc) {
    for_cells(m, b, [&](int i, int j) {
      const int l = m.ij2l(i, j);
      int src;
      switch (b.iside) {
        case 1: src = m.lEC(l); for (int k = 1; k <= km1; ++k) m.vh(k, l) = 0.0; break;
        case 2: src = m.lSC(l); for (int k = 1; k <= km1; ++k) m.uh(k, l) = 0.0; break;
        case 3: src = m.lWC(l); for (int k = 1; k <= km1; ++k) m.vh(k, l) = 0.0; break;
        default: src = m.lNC(l); for (int k = 1; k <= km1; ++k) m.uh(k, l) = 0.0; break;
      }
      for (int k = 1; k <= km1; ++k) m.wp(k, l) = m.wp(k, src);
    });
  }
}

void openbc_sca(Model& m) {
  for (const OpenBC& b : m.obc) {
    const double salbc = parab(0., m.thrs, b.sal, m.dtsec_obc / 3600.);
    for_cells(m, b, [&](int i, int j) {
      const int l = m.ij2l(i, j);
      for (int k = m.k1z(l); k <= m.kmz(l); ++k) {
        bool in;
        int src;
        switch (b.iside) {
          case 1: in = m.uh(k, l) > 0.0; src = m.lEC(l); break;
          case 2: in = m.vh(k, m.lSC(l)) < 0.0; src = m.lSC(l); break;
          case 3: in = m.uh(k, m.lWC(l)) < 0.0; src = m.lWC(l); break;
          default: in = m.vh(k, l) > 0.0; src = m.lNC(l); break;
        }
        m.sal(k, l) = (in && salbc > 0.0) ? salbc : m.sal(k, src);
      }
    });
  }
}

}  // namespace orc
