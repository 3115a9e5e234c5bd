// Oracle input readers and model set-up — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
//
// Restates, in FP64: `input` (si3d_utils.f90:21-315), `ZGridDimensions` (:318-382),
// `bathy` (:595-892), `init` (si3d_procedures.f90:23-181), `InitializeScalarFields`
// (:184-379, InitProc = 4 file branch), `InitializeTurbulenceModel` CASE(0)
// (si3d_mixing.f90:650-671).  The readers follow the reference's fixed-column record
// formats; only the records the hot-path configuration uses are interpreted.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "oracle.hpp"

namespace orc {

real densty_s(real temperature, real salinity, real elevation);

namespace {

struct Lines {
  std::vector<std::string> l;
  size_t pos = 0;
  bool eof() const { return pos >= l.size(); }
  const std::string& next() {
    static const std::string empty;
    if (pos >= l.size()) { pos++; return empty; }
    return l[pos++];
  }
  void skip(int n) { pos += n; }
};

bool load_lines(const std::string& path, Lines& L) {
  std::ifstream f(path);
  if (!f) return false;
  std::string s;
  while (std::getline(f, s)) {
    if (!s.empty() && s.back() == '\r') s.pop_back();
    L.l.push_back(s);
  }
  return true;
}

std::string field(const std::string& s, size_t start, size_t width) {
  if (start >= s.size()) return std::string();
  return s.substr(start, width);
}

// Fortran list of a G/I field: blanks are ignored (BN), empty field reads as zero.
bool parse_num(const std::string& fld, real& out) {
  std::string t;
  for (char c : fld) if (c != ' ' && c != '\t') t.push_back(c);
  if (t.empty()) { out = 0; return true; }
  // Fortran allows D exponents
  for (char& c : t) if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  out = std::strtod(t.c_str(), &end);
  return end && *end == '\0';
}

// '(14X,G20.2)' record: value in columns 15-34.
bool rec_g(Lines& L, real& v) { return parse_num(field(L.next(), 14, 20), v); }
bool rec_i(Lines& L, int& v) {
  real x;
  if (!parse_num(field(L.next(), 14, 20), x)) return false;
  v = (int)std::lround(x);
  return true;
}

// '(14X,20I)' record: n integers after column 14, separated by blanks or commas.
bool rec_ints(Lines& L, int n, std::vector<int>& out) {
  const std::string rec = field(L.next(), 14, 1000);
  out.clear();
  size_t i = 0;
  while ((int)out.size() < n) {
    while (i < rec.size() && (rec[i] == ' ' || rec[i] == ',' || rec[i] == '\t')) ++i;
    size_t j = i;
    while (j < rec.size() && (std::isdigit((unsigned char)rec[j]) || rec[j] == '-')) ++j;
    if (j == i) return false;
    out.push_back(std::atoi(rec.substr(i, j - i).c_str()));
    i = j;
  }
  return true;
}

}  // namespace

// si3d_utils.f90:21-315 (records read in the order the reference reads them)
static bool read_inp(Model& m, const std::string& dir) {
  Lines L;
  if (!load_lines(dir + "/si3d_inp.txt", L)) { m.err = "Error opening si3d_inp.txt"; return false; }
  Inp& p = m.in;
  bool ok = true;
  L.skip(1); p.title = L.next();                                      // '(/(A))'
  L.skip(3);                                                          // '(///(14X,G20.2))'
  ok &= rec_i(L, p.iyr0); ok &= rec_i(L, p.imon0); ok &= rec_i(L, p.iday0); ok &= rec_i(L, p.ihr0);
  L.skip(3);
  ok &= rec_g(L, p.xl); ok &= rec_g(L, p.yl); ok &= rec_g(L, p.zl); ok &= rec_g(L, p.tl);
  ok &= rec_g(L, p.idx); ok &= rec_g(L, p.idy); ok &= rec_g(L, p.idz); ok &= rec_g(L, p.dzmin);
  ok &= rec_g(L, p.datadj); ok &= rec_g(L, p.zetainit); ok &= rec_g(L, p.idt); ok &= rec_i(L, p.ibathyf);
  L.skip(3);                                                          // si3d_utils.f90:51-53
  ok &= rec_i(L, p.itrap); ok &= rec_i(L, p.niter); ok &= rec_i(L, p.ismooth); ok &= rec_g(L, p.beta);
  ok &= rec_i(L, p.iturb); ok &= rec_g(L, p.Av0); ok &= rec_g(L, p.Dv0); ok &= rec_i(L, p.iadv);
  ok &= rec_i(L, p.itrmom); ok &= rec_i(L, p.ihd); ok &= rec_g(L, p.Ax0); ok &= rec_g(L, p.Ay0);
  ok &= rec_g(L, p.f); ok &= rec_g(L, p.theta); ok &= rec_i(L, p.ibc); ok &= rec_i(L, p.isal);
  ok &= rec_i(L, p.itrsca); ok &= rec_g(L, p.cd); ok &= rec_i(L, p.ifsurfbc); ok &= rec_g(L, p.dtsurfbc);
  ok &= rec_i(L, p.icw); ok &= rec_g(L, p.cw); ok &= rec_g(L, p.wa); ok &= rec_g(L, p.phi);
  ok &= rec_i(L, p.idbg); ok &= rec_i(L, p.num_threads);
  if (!ok) { m.err = "si3d_inp.txt: bad record in parameter blocks 2-4"; return false; }
  L.skip(3); ok &= rec_i(L, p.ipt); ok &= rec_i(L, p.nnodes);        // :56-69
  L.skip(2);                                                          // node lists or '(/)'
  L.skip(3); ok &= rec_i(L, p.iop); ok &= rec_i(L, p.itspfh); ok &= rec_i(L, p.n_planes);
  {                                                                   // planes '(14X,20I)'
    const std::string rec = field(L.next(), 14, 1000);
    p.p_out.clear();
    size_t i = 0;
    while ((int)p.p_out.size() < p.n_planes) {
      while (i < rec.size() && (rec[i] == ' ' || rec[i] == ',' || rec[i] == '\t')) ++i;
      size_t j = i;
      while (j < rec.size() && (std::isdigit((unsigned char)rec[j]) || rec[j] == '-')) ++j;
      if (j == i) { m.err = "si3d_inp.txt: bad output plane list"; return false; }
      p.p_out.push_back(std::atoi(rec.substr(i, j - i).c_str()));
      i = j;
    }
  }
  L.skip(3); ok &= rec_i(L, p.iox);                                   // :91-93
  if (p.iox != 0) { m.err = "si3d_inp.txt: cross-section output (iox/=0) is not supported"; return false; }
  L.skip(3); ok &= rec_i(L, p.ipxml); ok &= rec_i(L, p.itspf); ok &= rec_i(L, p.iTurbVars);
  if (p.ipxml > 0 && p.iTurbVars != 0) { m.err = "turbulence variables in the 3-D output need iturb > 0"; return false; }
  if (p.nnodes > 0) { m.err = "the time-series writer (outt) is not restated"; return false; }
  L.skip(3); ok &= rec_i(L, p.nopen);                                 // :124-145
  if (p.nopen > 0) {
    // dtsecopenbc, then iside, itype, isbc, jsbc, iebc, jebc, nopen values each
    ok &= rec_g(L, m.dtsec_obc);
    std::vector<int> v[6];
    for (int r = 0; r < 6; ++r) ok &= rec_ints(L, p.nopen, v[r]);
    if (!ok) { m.err = "si3d_inp.txt: bad open-boundary records"; return false; }
    m.obc.assign(p.nopen, OpenBC{});
    for (int nn = 0; nn < p.nopen; ++nn) {
      OpenBC& b = m.obc[nn];
      b.iside = v[0][nn]; b.itype = v[1][nn]; b.isbc = v[2][nn]; b.jsbc = v[3][nn]; b.iebc = v[4][nn]; b.jebc = v[5][nn];
      if (b.itype != 1) { m.err = "only water-surface-elevation open boundaries (itype = 1) are restated"; return false; }
      if (b.iside < 1 || b.iside > 4) { m.err = "open boundary side must be 1..4"; return false; }
    }
    if (!(m.dtsec_obc > 0)) { m.err = "dtsecopenbc must be positive"; return false; }
  } else {
    L.skip(7);
  }
  L.skip(3); ok &= rec_i(L, p.nxNBO);                                 // ioNBTOGGLE=1 block
  if (p.nxNBO != 0) { m.err = "nested-boundary output (nxNBO>0) is not supported"; return false; }
  L.skip(7);
  L.skip(3); ok &= rec_i(L, p.ntr);                                   // :172-190
  if (p.ntr > 0) {
    ok &= rec_i(L, p.ecomod); ok &= rec_i(L, p.iotr); ok &= rec_i(L, p.itspftr); ok &= rec_i(L, p.ipwq);
    ok &= rec_i(L, p.nswq);
    if (p.ntr > 30) { m.err = "ntr > ntrmax = 30 (si3d_types.f90:291)"; return false; }
    // srcsnk00 (si3d_ecomod.f90:24-34): conservative tracers; the other models are not restated
    if (p.ecomod != 0) { m.err = "only conservative tracers (ecomod=0) are restated"; return false; }
    if (p.nopen > 0) { m.err = "tracers at open boundaries (openbcTracer) are not restated"; return false; }
  } else {
    L.skip(5);
  }
  L.skip(3); ok &= rec_i(L, p.iopss);                                 // :193-230
  if (p.iopss != 0) { m.err = "point sources (iopss>0) are outside the hot path"; return false; }
  if (!ok) { m.err = "si3d_inp.txt: bad record in output/boundary blocks"; return false; }
  if (p.ifsurfbc != 0) { m.err = "only ifsurfbc=0 (constant surface forcing) is on the hot path"; return false; }
  if (p.iturb != 0 && p.iturb != 1) { m.err = "only iturb = 0 (constant) and 1 (Mellor-Yamada 2.5) are restated"; return false; }
  if (p.ihd > 1) { m.err = "Smagorinsky (ihd>1) is outside the hot path"; return false; }
  if (p.ibathyf < 0) { m.err = "variable layer files (ibathyf<0) are not supported by the oracle"; return false; }

  // si3d_utils.f90:291-306
  m.dt = p.idt; m.dx = p.idx; m.dy = p.idy; m.ddz = p.idz; m.twodt = 2. * m.dt;
  m.dtdx = m.dt / m.dx; m.dtdy = m.dt / m.dy;
  const real g = 9.806;
  m.gdtdx = g * m.dtdx; m.gdtdy = g * m.dtdy; m.gdt2dx2 = m.gdtdx * m.dtdx; m.gdt2dy2 = m.gdtdy * m.dtdy;
  m.twodx = 2. * m.dx; m.twody = 2. * m.dy; m.fourdx = 2. * m.twodx; m.fourdy = 2. * m.twody;
  m.dxdx = m.dx * m.dx; m.dydy = m.dy * m.dy; m.dxdy = m.dx * m.dy;
  m.beta2 = p.beta / 2.;
  m.im = (int)std::lround(p.xl / m.dx) + 1; m.im1 = m.im + 1; m.i1 = 2;
  m.jm = (int)std::lround(p.yl / m.dy) + 1; m.jm1 = m.jm + 1; m.j1 = 2;
  m.nts = (int)(p.tl / m.dt + .5);

  // ZGridDimensions, constant layer thickness (si3d_utils.f90:362-379)
  m.km = (int)std::ceil(p.zl / m.ddz) + 1;
  m.km1 = m.km + 1; m.k1 = 2;
  m.zlevel.assign(m.km1, 0.0);
  m.zlevel[m.k1 - 1] = 0.0;
  for (int k = m.k1 + 1; k <= m.km1; ++k) m.zlevel[k - 1] = m.zlevel[k - 2] + m.ddz;
  m.zlevel[m.k1 - 1] = -100.;
  m.zlevel[0] = -100.;
  return true;
}

// bathy (si3d_utils.f90:595-892)
static bool read_bathy(Model& m, const std::string& dir) {
  Lines L;
  if (!load_lines(dir + "/si3d_bathy", L)) { m.err = "Error opening si3d_bathy"; return false; }
  const std::string& hdr = L.next();
  real a, b, c;
  // '(37X,I5,6X,I5,8X,I5//)'
  if (!parse_num(field(hdr, 37, 5), a) || !parse_num(field(hdr, 48, 5), b) || !parse_num(field(hdr, 61, 5), c)) {
    m.err = "si3d_bathy: bad header"; return false;
  }
  int imm = (int)a, jmm = (int)b, ncols = (int)c;
  L.skip(2);
  if (m.im != imm + 1 || m.jm != jmm + 1) {
    m.err = "Grid size computed from input file does not agree with the header in the bathymetry file";
    return false;
  }
  const int im1 = m.im1, jm1 = m.jm1, im = m.im, jm = m.jm;
  std::vector<real> h4((size_t)im1 * jm1, 0.0);
  auto H4 = [&](int i, int j) -> real& { return h4[(size_t)(j - 1) * im1 + (i - 1)]; };
  int ncols1 = ncols - 1, nc = imm / ncols + 1, ia = -ncols1 + 1;
  for (int nn = 1; nn <= nc; ++nn) {
    ia = ia + ncols;
    int ib = ia + ncols1;
    if (ia > im) break;
    if (ib > im) ib = im;
    for (int j = jm; j >= m.j1; --j) {
      if (L.eof()) { m.err = "si3d_bathy: truncated"; return false; }
      const std::string& s = L.next();
      for (int i = ia; i <= ib; ++i) {          // '(5X,ncolsG5.0)'
        real v;
        if (!parse_num(field(s, 5 + 5 * (i - ia), 5), v)) { m.err = "si3d_bathy: bad value"; return false; }
        H4(i, j) = v;
      }
    }
  }
  for (auto& x : h4) x = x * 0.1 + m.in.datadj;     // dm -> m (:687)
  for (int j = 1; j <= jm1; ++j) { H4(1, j) = 0.0; H4(im1, j) = 0.0; }
  for (int i = 1; i <= im1; ++i) { H4(i, jm1) = 0.0; H4(i, 1) = 0.0; }
  m.mask2d_.assign((size_t)im1 * jm1, 0);
  for (int j = 1; j <= jm1; ++j)
    for (int i = 1; i <= im1; ++i) m.mask2d_[(size_t)(j - 1) * im1 + (i - 1)] = H4(i, j) > 0.0;
  // fictitious rows/columns (:721-727) only matter for outputs; depths at zeta points are H4 itself
  // l-ordering: i outer, j inner (:781-793)
  int l = 0;
  for (int i = 1; i <= im1; ++i)
    for (int j = 1; j <= jm1; ++j)
      if (m.mask2d(i, j)) ++l;
  m.lm = l; m.lm1 = l + 1;
  const int lm1 = m.lm1;
  m.ij2l_.assign((size_t)im1 * jm1, lm1);
  m.l2i.init(lm1, 0); m.l2j.init(lm1, 0);
  l = 0;
  for (int i = 1; i <= im1; ++i)
    for (int j = 1; j <= jm1; ++j)
      if (m.mask2d(i, j)) {
        ++l; m.l2i(l) = i; m.l2j(l) = j; m.ij2l_[(size_t)(j - 1) * im1 + (i - 1)] = l;
      }
  m.lEC.init(lm1, lm1); m.lWC.init(lm1, lm1); m.lNC.init(lm1, lm1); m.lSC.init(lm1, lm1);
  l = 0;
  for (int i = m.i1; i <= im; ++i)
    for (int j = m.j1; j <= jm; ++j) {
      if (!m.mask2d(i, j)) continue;
      ++l;
      m.lEC(l) = m.ij2l(i + 1, j); m.lWC(l) = m.ij2l(i - 1, j);
      m.lNC(l) = m.ij2l(i, j + 1); m.lSC(l) = m.ij2l(i, j - 1);
    }
  // kmz / hhs (:812-863), constant-layer branch
  m.kmz.init(lm1, 0); m.hhs.init(lm1, 0.0);
  for (int j = 1; j <= jm1; ++j)
    for (int i = 1; i <= im1; ++i) {
      if (!m.mask2d(i, j)) continue;
      int ll = m.ij2l(i, j);
      real hs1 = H4(i, j);
      int kk = (int)std::floor(hs1 / m.ddz);
      if ((hs1 - kk * m.ddz) > m.in.dzmin) { kk = kk + 1; m.hhs(ll) = hs1; }
      else m.hhs(ll) = kk * m.ddz;
      m.kmz(ll) = kk + 1;
      if (m.kmz(ll) > m.km) { m.err = "bathymetry deeper than zl: kmz > km"; return false; }
    }
  m.kmz(lm1) = m.km1;
  m.hhu.init(lm1, 0.0); m.hhv.init(lm1, 0.0);
  for (int j = 1; j <= jm; ++j)
    for (int i = 1; i <= im; ++i) {
      if (m.mask2d(i + 1, j) && m.mask2d(i, j)) { int ll = m.ij2l(i, j); m.hhu(ll) = std::min(m.hhs(m.lEC(ll)), m.hhs(ll)); }
      if (m.mask2d(i, j + 1) && m.mask2d(i, j)) { int ll = m.ij2l(i, j); m.hhv(ll) = std::min(m.hhs(m.lNC(ll)), m.hhs(ll)); }
    }
  return true;
}

// si3d_init.txt, InitProc=4 file branch (si3d_procedures.f90:293-318)
// Records '(10X, ntr+1 G11.5)': temperature, then one column per tracer; prof is (km1, ntr + 1)
// with k fastest.
static bool read_init_profile(Model& m, const std::string& dir, std::vector<real>& prof) {
  Lines L;
  if (!load_lines(dir + "/si3d_init.txt", L)) { m.err = "Error opening si3d_init.txt"; return false; }
  L.skip(5);   // '(////)'
  L.skip(1);   // tracer_line '(A)'
  L.skip(1);   // '(A)'
  const int nc = m.in.ntr + 1;
  prof.assign((size_t)m.km1 * nc, 0.0);
  for (int k = 1; k <= m.km1; ++k) {
    if (L.eof()) { m.err = "si3d_init.txt: truncated"; return false; }
    const std::string line = L.next();
    for (int c = 0; c < nc; ++c) {
      real v;
      if (!parse_num(field(line, 10 + 11 * c, 11), v)) { m.err = "si3d_init.txt: bad value"; return false; }
      prof[(size_t)c * m.km1 + k - 1] = v;
    }
  }
  return true;
}

// Harness overlay: per-column wind (uair, vair) on the (i,j) grid.
// File si3d_wind_override.bin: int32 im1, int32 jm1, then im1*jm1 float64 uair and
// im1*jm1 float64 vair, i outer / j inner (the l-ordering traversal).
static bool read_wind_override(Model& m, const std::string& dir) {
  FILE* f = std::fopen((dir + "/si3d_wind_override.bin").c_str(), "rb");
  if (!f) return true;  // optional
  int32_t dims[2];
  bool ok = std::fread(dims, 4, 2, f) == 2 && dims[0] == m.im1 && dims[1] == m.jm1;
  size_t nn = (size_t)m.im1 * m.jm1;
  std::vector<double> uu(nn), vv(nn);
  ok = ok && std::fread(uu.data(), 8, nn, f) == nn && std::fread(vv.data(), 8, nn, f) == nn;
  std::fclose(f);
  if (!ok) { m.err = "si3d_wind_override.bin: bad size"; return false; }
  m.wind_override = true;
  m.uair_ovr.assign(m.lm1, 0.0); m.vair_ovr.assign(m.lm1, 0.0);
  for (int l = 1; l <= m.lm; ++l) {
    size_t c = (size_t)(m.l2i(l) - 1) * m.jm1 + (m.l2j(l) - 1);
    m.uair_ovr[l - 1] = uu[c]; m.vair_ovr[l - 1] = vv[c];
  }
  return true;
}

// init (si3d_procedures.f90:23-181), testcase = 3 -> CASE DEFAULT
static void init_state(Model& m, const std::vector<real>& prof) {
  const int lm1 = m.lm1, km1 = m.km1, k1 = m.k1;
  const real HMIN = 0.0, ZERO = 0.0, sed_h = 0.5;
  m.s.init(lm1, m.in.zetainit); m.sp.init(lm1, m.in.zetainit); m.spp.init(lm1, m.in.zetainit);
  for (F3* a : {&m.uh, &m.uhp, &m.uhpp, &m.u, &m.up, &m.upp, &m.hu, &m.hup, &m.hupp, &m.ex, &m.agx, &m.arx,
                &m.vh, &m.vhp, &m.vhpp, &m.v, &m.vp, &m.vpp, &m.hv, &m.hvp, &m.hvpp, &m.agy, &m.ary,
                &m.h, &m.hp, &m.hpp, &m.sal, &m.salp, &m.salpp, &m.rhop, &m.Av, &m.Dv, &m.wp, &m.HeatSource,
                &m.Bth2, &m.Bth3, &m.Bth4, &m.Bex, &m.Bhaxpp, &m.Bhaypp})
    a->init(km1, lm1, 0.0);
  m.k1z.init(lm1, km1); m.k1u.init(lm1, km1); m.k1v.init(lm1, km1);
  for (int l = 1; l <= m.lm; ++l) {
    int i = m.l2i(l), j = m.l2j(l);
    int kms = m.kmz(l), nwlsp = 0;
    for (int k = k1; k <= kms; ++k) {
      m.hp(k, l) = std::min(m.zl(k + 1), m.hhs(l)) - std::max(m.zl(k), -m.sp(l));
      if (m.hp(k, l) > HMIN) { nwlsp++; if (nwlsp == 1) m.k1z(l) = k; }
      else m.hp(k, l) = ZERO;
    }
    m.hp(kms + 1, l) = sed_h;
    if (m.k1z(l) == km1) { m.s(l) = -m.hhs(l) + HMIN; m.sp(l) = -m.hhs(l) + HMIN; m.spp(l) = -m.hhs(l) + HMIN; }
    if (m.mask2d(i + 1, j)) {
      int kmx = std::min(m.kmz(l), m.kmz(m.lEC(l))), nw = 0;
      for (int k = k1; k <= kmx; ++k) {
        m.hup(k, l) = std::min(m.zl(k + 1), m.hhu(l)) - std::max(m.zl(k), -(m.sp(l) + m.sp(m.lEC(l))) / 2.);
        if (m.hup(k, l) > HMIN) { nw++; if (nw == 1) m.k1u(l) = k; }
        else m.hup(k, l) = ZERO;
      }
    }
    if (m.mask2d(i, j + 1)) {
      int kmy = std::min(m.kmz(l), m.kmz(m.lNC(l))), nw = 0;
      for (int k = k1; k <= kmy; ++k) {
        m.hvp(k, l) = std::min(m.zl(k + 1), m.hhv(l)) - std::max(m.zl(k), -(m.sp(l) + m.sp(m.lNC(l))) / 2.);
        if (m.hvp(k, l) > HMIN) { nw++; if (nw == 1) m.k1v(l) = k; }
        else m.hvp(k, l) = ZERO;
      }
    }
  }
  m.hupp = m.hup; m.hu = m.hup; m.hvpp = m.hvp; m.hv = m.hvp; m.hpp = m.hp; m.h = m.hp;
  for (F1* a : {&m.eagx, &m.eagy, &m.earx, &m.eary, &m.sx, &m.sy, &m.dd, &m.qq}) a->init(lm1, 0.0);
  m.rr.init(lm1, 1.0);
  m.uair.init(lm1, 0.0); m.vair.init(lm1, 0.0); m.cdw.init(lm1, 0.0);
  // InitializeScalarFields file branch: salp(k,:) = profile(k) for every column incl. lm1
  for (int l = 1; l <= lm1; ++l)
    for (int k = 1; k <= km1; ++k) m.salp(k, l) = prof[k - 1];
  m.sal = m.salp; m.salpp = m.salp;
  // non-active tracers, ecomod >= 0 branch: tracer(k,:,nn) = column nn + 1 (:335-351); the
  // sediment-layer values of the Hg and suspended-sediment species do not apply to ecomod = 0
  m.tracer.assign(m.in.ntr, F3());
  for (int nn = 1; nn <= m.in.ntr; ++nn) {
    F3& t = m.tracer[nn - 1];
    t.init(km1, lm1, 0.0);
    for (int l = 1; l <= lm1; ++l)
      for (int k = 1; k <= km1; ++k) t(k, l) = prof[(size_t)nn * km1 + k - 1];
  }
  m.tracerpp = m.tracer;
  for (int l = 1; l <= lm1; ++l)
    for (int k = k1; k <= km1; ++k) {
      real z = (m.zl(k) == -100.) ? 0.5 * m.hp(k, l) : m.zl(k) + 0.5 * m.hp(k, l);
      m.rhop(k, l) = densty_s(m.salp(k, l), 0.00004, z) - 1000.;
    }
  // InitializeTurbulenceModel (si3d_mixing.f90:615-724): CASE(1) sets q2 and q2l and leaves the
  // eddy coefficients at zero until the first fd; CASE(0) (:650-671) sets them
  for (F3* a : {&m.q2, &m.q2p, &m.q2pp, &m.q2l, &m.q2lp, &m.q2lpp}) a->init(km1, lm1, 0.0);
  if (m.in.iturb == 1) { init_turbulence(m); return; }
  for (int l = 1; l <= m.lm; ++l) {
    int kms = m.kmz(l), k1s = m.k1z(l);
    m.Av(k1s, l) = 0.0; m.Dv(k1s, l) = 0.0;
    if (kms > k1s)
      for (int k = k1s + 1; k <= kms; ++k) { m.Av(k, l) = m.in.Av0; m.Dv(k, l) = m.in.Dv0; }
    m.Av(kms + 1, l) = 0.0; m.Dv(kms + 1, l) = 0.0;
  }
}

bool read_inputs(Model& m, const std::string& dir) {
  m.dir = dir;
  if (!read_inp(m, dir)) return false;
  m.date.isec0 = (double)m.in.ihr0 / 100. * 3600.;   // si3d_utils.f90:310
  compute_date(m, 0.0);                               // :43
  if (!read_bathy(m, dir)) return false;
  std::vector<real> prof;
  if (!read_init_profile(m, dir, prof)) return false;
  if (!read_wind_override(m, dir)) return false;
  init_state(m, prof);
  if (!m.obc.empty() && (!read_openbc_files(m, dir) || !openbc0(m))) return false;   // si3d.f90:64
  return write_outputs(m, 0);   // initial frames (si3d.f90:89-100)
}

}  // namespace orc
