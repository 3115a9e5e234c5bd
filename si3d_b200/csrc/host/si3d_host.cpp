// Host side above the C ABI (include/si3d_host.h): the reference's input readers and set-up
// restated in C++, and the time loop driving si3d_gpu_step.
//
// Readers: `input` (si3d_utils.f90:21-315, fixed-column records '(14X,G20.2)'), `bathy`
// (:595-892, header '(37X,I5,6X,I5,8X,I5//)', rows '(5X,ncolsG5.0)' in decimetres),
// InitializeScalarFields' file branch (si3d_procedures.f90:293-318, rows '(10X,G11.5)').
// Set-up: ZGridDimensions (si3d_utils.f90:362-379), the l ordering and neighbour maps
// (:781-806), kmz/hhs/hhu/hhv (:812-880), `init` (si3d_procedures.f90:23-181) and
// InitializeTurbulenceModel CASE(0) (si3d_mixing.f90:650-671).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../../include/si3d_host.h"

namespace {

struct Records {
  std::vector<std::string> rows;
  size_t at = 0;
  bool load(const std::string& path) {
    std::ifstream in(path);
    if (!in) return false;
    for (std::string s; std::getline(in, s);) {
      if (!s.empty() && s.back() == '\r') s.pop_back();
      rows.push_back(s);
    }
    return true;
  }
  bool more() const { return at < rows.size(); }
  std::string take() { return at < rows.size() ? rows[at++] : (at++, std::string()); }
  void skip(int n) { at += n; }
};

// Value of a fixed-width numeric field (blanks ignored, empty = 0, D exponents allowed).
// Integers of a '(14X,20I)' record (separated by blanks or commas); false when fewer than n.
bool int_list(const std::string& rec, int n, std::vector<int>& out) {
  out.clear();
  size_t i = 14;
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

bool numeric(const std::string& row, size_t col, size_t width, double& v) {
  std::string t;
  for (size_t i = col; i < std::min(row.size(), col + width); ++i) {
    char ch = row[i];
    if (ch == ' ' || ch == '\t') continue;
    t.push_back(ch == 'd' || ch == 'D' ? 'e' : ch);
  }
  if (t.empty()) { v = 0; return true; }
  char* e = nullptr;
  v = std::strtod(t.c_str(), &e);
  return e && *e == 0;
}

struct HostModel {
  std::string err;
  si3d_solver_opts opt{};
  // input parameters
  double xl = 0, yl = 0, zl = 0, tl = 0, idx = 0, idy = 0, idz = 0, dzmin = 0, datadj = 0, zetainit = 0, idt = 0;
  double beta = 0, Av0 = 0, Dv0 = 0, Ax0 = 0, Ay0 = 0, f = 0, theta = 1, cd = 0, dtsurfbc = 0, cw = 0, wa = 0, phi = 0;
  int ibathyf = 0, itrap = 1, niter = 2, ismooth = 0, iturb = 0, iadv = 1, itrmom = 1, ihd = 1, ibc = 1, isal = 1,
      itrsca = 0, ifsurfbc = 0, icw = 0, nopen = 0, ntr = 0, iopss = 0, iox = 0, nxNBO = 0, ecomod = 0;
  // grid
  int im = 0, im1 = 0, jm = 0, jm1 = 0, km = 0, km1 = 0, k1 = 2, lm = 0, lm1 = 0, nts = 0;
  std::vector<double> zlevel, hhs, hhu, hhv;
  std::vector<int> l2i, l2j, lEC, lWC, lNC, lSC, kmz;
  std::vector<unsigned char> wet;  // (i,j) mask, j fastest per i (the l traversal order)
  std::vector<int> ij2l;
  // initial state
  std::vector<double> s0, hp0, hup0, hvp0, salp0, Av0f, Dv0f, uair, vair, cdw;
  std::vector<double> tracer0;   // ntr fields of (km1, lm1), column-major
  std::vector<double> q2l0;      // iturb = 1: initial q2l (InitializeTurbulenceModel CASE(1))
  // open boundaries (si3d_utils.f90:124-140 and the openbcNN.txt series, openbc0 :55-91)
  double obc_dtsec = 0;
  std::vector<int> ob_side, ob_type, ob_is, ob_js, ob_ie, ob_je;
  int ob_npts = 0;
  std::vector<double> ob_wse, ob_tmp;   // [nopen][ob_npts]
  // outputs (si3d_utils.f90:72-121, :172-181) and the date of compute_date (:3546-3674)
  int iyr0 = 0, imon0 = 0, iday0 = 0, ihr0 = 0;
  int iop = 0, itspfh = 0, n_planes = 0, ipxml = 0, itspf = 0, iTurbVars = 0, iotr = 0, itspftr = 0;
  std::vector<int> p_out;
  struct Date {
    int iyr = 0, imon = 0, iday = 0, ihr = 0, iyrp = 0, imonp = 0, idayp = 0, ihrp = 0;
    double isec = 0, isecp = 0, isec0 = 0;
    int month[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  } date;
  std::string dir, title;
  bool space_written = false;   // outs writes its header once (first_entry)
  std::shared_ptr<FILE> f_ptrack;
  std::vector<std::shared_ptr<FILE>> f_tracer, f_plane;
  // frame writer: the main thread packs frames into page-locked buffers (asynchronous copies); a
  // writer thread waits for each copy and writes its record, so file output overlaps the steps
  struct Buf { float* p = nullptr; long long cap = 0; };
  struct Job {
    std::shared_ptr<FILE> f;
    std::vector<unsigned char> head;   // record bytes before the frame (or the whole record)
    Buf buf;
    long long count = 0;
    unsigned long long ticket = 0;
  };
  std::mutex wmu;
  std::condition_variable wcv;
  std::deque<Job> jobs;
  std::vector<Buf> free_bufs;
  int in_flight = 0;               // frames queued or being written
  bool stop = false;
  int werr = 0;                    // first writer error
  std::thread writer;
  ~HostModel() {
    if (writer.joinable()) {
      { std::lock_guard<std::mutex> lk(wmu); stop = true; }
      wcv.notify_all();
      writer.join();
    }
    for (Buf& b : free_bufs) si3d_gpu_host_free(b.p);
  }
  std::vector<int> k1z0, k1u0, k1v0;
  // run
  int gpu = -1, n = 0;
  bool W(int i, int j) const { return wet[(size_t)(i - 1) * jm1 + (j - 1)] != 0; }
  int L(int i, int j) const { return ij2l[(size_t)(i - 1) * jm1 + (j - 1)]; }
  double zlv(int k) const { return zlevel[k - 1]; }
  size_t I3(int k, int l) const { return (size_t)(l - 1) * km1 + (k - 1); }
};

std::mutex g_mu;
std::vector<std::unique_ptr<HostModel>> g_models;

HostModel* model(int h) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (h >= 0 && h < (int)g_models.size()) ? g_models[h].get() : nullptr;
}

bool read_parameters(HostModel& M, const std::string& dir) {
  Records R;
  if (!R.load(dir + "/si3d_inp.txt")) { M.err = "cannot open si3d_inp.txt"; return false; }
  bool ok = true;
  auto g = [&](double& v) { ok = ok && numeric(R.take(), 14, 20, v); };
  auto gi = [&](int& v) { double x = 0; ok = ok && numeric(R.take(), 14, 20, x); v = (int)std::lround(x); };
  int dummy = 0;
  R.skip(1); M.title = R.take();                 // title block '(/(A))'
  R.skip(3); gi(M.iyr0); gi(M.imon0); gi(M.iday0); gi(M.ihr0);
  R.skip(3);
  g(M.xl); g(M.yl); g(M.zl); g(M.tl); g(M.idx); g(M.idy); g(M.idz); g(M.dzmin); g(M.datadj); g(M.zetainit);
  g(M.idt); gi(M.ibathyf);
  R.skip(3);
  gi(M.itrap); gi(M.niter); gi(M.ismooth); g(M.beta); gi(M.iturb); g(M.Av0); g(M.Dv0); gi(M.iadv); gi(M.itrmom);
  gi(M.ihd); g(M.Ax0); g(M.Ay0); g(M.f); g(M.theta); gi(M.ibc); gi(M.isal); gi(M.itrsca); g(M.cd); gi(M.ifsurfbc);
  g(M.dtsurfbc); gi(M.icw); g(M.cw); g(M.wa); g(M.phi); gi(dummy); gi(dummy);
  int nnodes = 0;
  R.skip(3); gi(dummy); gi(nnodes); R.skip(2);   // ipt, nnodes, node lists
  R.skip(3); gi(M.iop); gi(M.itspfh); gi(M.n_planes);
  {   // planes '(14X,20I)'
    const std::string rec = R.take();
    M.p_out.clear();
    size_t i = 14;
    while ((int)M.p_out.size() < M.n_planes) {
      while (i < rec.size() && (rec[i] == ' ' || rec[i] == ',' || rec[i] == '\t')) ++i;
      size_t j = i;
      while (j < rec.size() && (std::isdigit((unsigned char)rec[j]) || rec[j] == '-')) ++j;
      if (j == i) { M.err = "si3d_inp.txt: bad output plane list"; return false; }
      M.p_out.push_back(std::atoi(rec.substr(i, j - i).c_str()));
      i = j;
    }
  }
  R.skip(3); gi(M.iox);
  R.skip(3); gi(M.ipxml); gi(M.itspf); gi(M.iTurbVars);
  R.skip(3); gi(M.nopen);
  if (M.nopen > 0) {
    g(M.obc_dtsec);
    for (std::vector<int>* v : {&M.ob_side, &M.ob_type, &M.ob_is, &M.ob_js, &M.ob_ie, &M.ob_je})
      if (!int_list(R.take(), M.nopen, *v)) { M.err = "si3d_inp.txt: bad open-boundary record"; return false; }
    for (int t : M.ob_type)
      if (t != 1) { M.err = "si3d_inp.txt: only water-surface-elevation open boundaries (itype = 1) are built"; return false; }
  } else {
    R.skip(7);
  }
  R.skip(3); gi(M.nxNBO); R.skip(7);
  R.skip(3); gi(M.ntr);                          // tracer block (si3d_utils.f90:172-190)
  if (M.ntr > 0) { gi(M.ecomod); gi(M.iotr); gi(M.itspftr); gi(dummy); gi(dummy); }   // ipwq nswq unused
  else R.skip(5);
  R.skip(3); gi(M.iopss);
  if (!ok) { M.err = "si3d_inp.txt: unreadable record"; return false; }
  if (M.nopen > 0 && M.ntr > 0) { M.err = "si3d_inp.txt: tracers at open boundaries (openbcTracer) are not built"; return false; }
  if (M.iox || M.nxNBO || M.iopss || M.ifsurfbc || (M.iturb != 0 && M.iturb != 1) || M.ihd > 1 || M.ibathyf < 0 ||
      M.ismooth || M.itrmom != 1) {
    M.err = "si3d_inp.txt selects an option outside the semi-implicit core (point sources, heat budget, "
            "turbulence closure, Smagorinsky, smoothing, non-centred advection or variable layers)";
    return false;
  }
  if (nnodes > 0) {
    M.err = "si3d_inp.txt: the time-series writer (outt, nnodes > 0) is not built";
    return false;
  }
  if (M.ipxml > 0 && M.iTurbVars != 0) {
    M.err = "si3d_inp.txt: turbulence variables in the 3-D output need a turbulence closure (iturb > 0)";
    return false;
  }
  if (M.ntr < 0 || M.ntr > 30 || (M.ntr > 0 && M.ecomod != 0)) {
    M.err = "si3d_inp.txt: only 0..30 conservative tracers (ecomod = 0) are supported; water quality, "
            "tracer clouds, size structure and sediment models are not";
    return false;
  }
  M.im = (int)std::lround(M.xl / M.idx) + 1; M.im1 = M.im + 1;
  M.jm = (int)std::lround(M.yl / M.idy) + 1; M.jm1 = M.jm + 1;
  M.nts = (int)(M.tl / M.idt + .5);
  M.km = (int)std::ceil(M.zl / M.idz) + 1;
  M.km1 = M.km + 1;
  M.zlevel.assign(M.km1, 0.0);
  M.zlevel[M.k1 - 1] = 0.0;
  for (int k = M.k1 + 1; k <= M.km1; ++k) M.zlevel[k - 1] = M.zlevel[k - 2] + M.idz;
  M.zlevel[0] = -100.;
  M.zlevel[M.k1 - 1] = -100.;
  return true;
}

bool read_bathymetry(HostModel& M, const std::string& dir) {
  Records R;
  if (!R.load(dir + "/si3d_bathy")) { M.err = "cannot open si3d_bathy"; return false; }
  const std::string head = R.take();
  double a = 0, b = 0, c = 0;
  if (!numeric(head, 37, 5, a) || !numeric(head, 48, 5, b) || !numeric(head, 61, 5, c) || c < 1) {
    M.err = "si3d_bathy: bad header"; return false;
  }
  R.skip(2);
  const int imm = (int)a, jmm = (int)b, ncols = (int)c;
  if (M.im != imm + 1 || M.jm != jmm + 1) { M.err = "si3d_bathy header disagrees with si3d_inp.txt"; return false; }
  // depths at zeta points, decimetres, blocks of ncols i-columns, rows j = jm .. 2
  std::vector<double> dep((size_t)M.im1 * M.jm1, 0.0);
  auto D = [&](int i, int j) -> double& { return dep[(size_t)(i - 1) * M.jm1 + (j - 1)]; };
  for (int ia = 2; ia <= M.im; ia += ncols) {
    const int ib = std::min(ia + ncols - 1, M.im);
    for (int j = M.jm; j >= 2; --j) {
      if (!R.more()) { M.err = "si3d_bathy: truncated"; return false; }
      const std::string row = R.take();
      for (int i = ia; i <= ib; ++i)
        if (!numeric(row, 5 + 5 * (i - ia), 5, D(i, j))) { M.err = "si3d_bathy: bad depth"; return false; }
    }
  }
  M.wet.assign((size_t)M.im1 * M.jm1, 0);
  M.ij2l.assign((size_t)M.im1 * M.jm1, 0);
  int l = 0;
  for (int i = 1; i <= M.im1; ++i)
    for (int j = 1; j <= M.jm1; ++j) {
      const bool border = (i == 1 || i == M.im1 || j == 1 || j == M.jm1);
      const double h4 = border ? 0.0 : D(i, j) * 0.1 + M.datadj;
      D(i, j) = h4;
      if (h4 > 0.0) { M.wet[(size_t)(i - 1) * M.jm1 + (j - 1)] = 1; ++l; }
    }
  M.lm = l; M.lm1 = l + 1;
  const int lm1 = M.lm1;
  for (auto& v : M.ij2l) v = lm1;
  M.l2i.assign(lm1, 0); M.l2j.assign(lm1, 0);
  l = 0;
  for (int i = 1; i <= M.im1; ++i)
    for (int j = 1; j <= M.jm1; ++j)
      if (M.W(i, j)) { ++l; M.l2i[l - 1] = i; M.l2j[l - 1] = j; M.ij2l[(size_t)(i - 1) * M.jm1 + (j - 1)] = l; }
  M.lEC.assign(lm1, lm1); M.lWC.assign(lm1, lm1); M.lNC.assign(lm1, lm1); M.lSC.assign(lm1, lm1);
  for (int q = 1; q <= M.lm; ++q) {
    const int i = M.l2i[q - 1], j = M.l2j[q - 1];
    M.lEC[q - 1] = M.L(i + 1, j); M.lWC[q - 1] = M.L(i - 1, j);
    M.lNC[q - 1] = M.L(i, j + 1); M.lSC[q - 1] = M.L(i, j - 1);
  }
  M.kmz.assign(lm1, 0); M.hhs.assign(lm1, 0.0);
  for (int q = 1; q <= M.lm; ++q) {
    const double hs1 = D(M.l2i[q - 1], M.l2j[q - 1]);
    int kk = (int)std::floor(hs1 / M.idz);
    if ((hs1 - kk * M.idz) > M.dzmin) { kk += 1; M.hhs[q - 1] = hs1; }
    else M.hhs[q - 1] = kk * M.idz;
    M.kmz[q - 1] = kk + 1;
    if (M.kmz[q - 1] > M.km) { M.err = "bathymetry deeper than zl"; return false; }
    if (M.kmz[q - 1] < M.k1) { M.err = "a wet cell shallower than dzmin has no layer"; return false; }
  }
  M.kmz[lm1 - 1] = M.km1;
  M.hhu.assign(lm1, 0.0); M.hhv.assign(lm1, 0.0);
  for (int q = 1; q <= M.lm; ++q) {
    if (M.lEC[q - 1] != lm1) M.hhu[q - 1] = std::min(M.hhs[M.lEC[q - 1] - 1], M.hhs[q - 1]);
    if (M.lNC[q - 1] != lm1) M.hhv[q - 1] = std::min(M.hhs[M.lNC[q - 1] - 1], M.hhs[q - 1]);
  }
  return true;
}

bool read_profile(HostModel& M, const std::string& dir, std::vector<double>& prof) {
  Records R;
  if (!R.load(dir + "/si3d_init.txt")) { M.err = "cannot open si3d_init.txt"; return false; }
  R.skip(7);
  // records '(10X, ntr+1 G11.5)' (si3d_procedures.f90:313-318): temperature, then one column per
  // tracer; prof is (km1, ntr + 1) with k fastest
  const int nc = M.ntr + 1;
  prof.assign((size_t)M.km1 * nc, 0.0);
  for (int k = 0; k < M.km1; ++k) {
    if (!R.more()) { M.err = "si3d_init.txt: truncated"; return false; }
    const std::string rec = R.take();
    for (int c = 0; c < nc; ++c)
      if (!numeric(rec, 10 + 11 * c, 11, prof[(size_t)c * M.km1 + k])) { M.err = "si3d_init.txt: bad value"; return false; }
  }
  return true;
}

bool read_wind(HostModel& M, const std::string& dir) {
  const int lm1 = M.lm1;
  M.uair.assign(lm1, 0.0); M.vair.assign(lm1, 0.0); M.cdw.assign(lm1, 0.0);
  const double pi = 3.1415926535897932;
  for (int q = 0; q < M.lm; ++q) {   // surfbc CASE(0) (si3d_boundaryconditions.f90:4508-4514)
    M.uair[q] = -M.wa * std::sin(pi * M.phi / 180.);
    M.vair[q] = -M.wa * std::cos(pi * M.phi / 180.);
    M.cdw[q] = M.cw;
  }
  FILE* fp = std::fopen((dir + "/si3d_wind_override.bin").c_str(), "rb");
  if (!fp) return true;
  int32_t hd[2] = {0, 0};
  const size_t n2 = (size_t)M.im1 * M.jm1;
  std::vector<double> u(n2), v(n2);
  bool ok = std::fread(hd, 4, 2, fp) == 2 && hd[0] == M.im1 && hd[1] == M.jm1 && std::fread(u.data(), 8, n2, fp) == n2 &&
            std::fread(v.data(), 8, n2, fp) == n2;
  std::fclose(fp);
  if (!ok) { M.err = "si3d_wind_override.bin: size mismatch"; return false; }
  for (int q = 0; q < M.lm; ++q) {
    const size_t c = (size_t)(M.l2i[q] - 1) * M.jm1 + (M.l2j[q] - 1);
    M.uair[q] = u[c]; M.vair[q] = v[c];
  }
  return true;
}

// init (si3d_procedures.f90:23-181), testcase 3 -> CASE DEFAULT, plus the scalar profile and the
// constant eddy coefficients.
void initial_state(HostModel& M, const std::vector<double>& prof) {
  const int lm1 = M.lm1, km1 = M.km1, k1 = M.k1;
  const size_t n3 = (size_t)km1 * lm1;
  M.s0.assign(lm1, M.zetainit);
  M.hp0.assign(n3, 0.0); M.hup0.assign(n3, 0.0); M.hvp0.assign(n3, 0.0);
  M.k1z0.assign(lm1, km1); M.k1u0.assign(lm1, km1); M.k1v0.assign(lm1, km1);
  for (int l = 1; l <= M.lm; ++l) {
    const int kms = M.kmz[l - 1];
    int first = 0;
    for (int k = k1; k <= kms; ++k) {
      double v = std::min(M.zlv(k + 1), M.hhs[l - 1]) - std::max(M.zlv(k), -M.s0[l - 1]);
      if (v > 0.0) { if (!first) { first = 1; M.k1z0[l - 1] = k; } }
      else v = 0.0;
      M.hp0[M.I3(k, l)] = v;
    }
    M.hp0[M.I3(kms + 1, l)] = 0.5;   // sed_h (si3d_types.f90:420)
    if (M.k1z0[l - 1] == km1) M.s0[l - 1] = -M.hhs[l - 1] + 0.0;
    const int lE = M.lEC[l - 1], lN = M.lNC[l - 1];
    if (lE != lm1) {
      const int kmx = std::min(kms, M.kmz[lE - 1]);
      first = 0;
      for (int k = k1; k <= kmx; ++k) {
        double v = std::min(M.zlv(k + 1), M.hhu[l - 1]) - std::max(M.zlv(k), -(M.s0[l - 1] + M.s0[lE - 1]) / 2.);
        if (v > 0.0) { if (!first) { first = 1; M.k1u0[l - 1] = k; } }
        else v = 0.0;
        M.hup0[M.I3(k, l)] = v;
      }
    }
    if (lN != lm1) {
      const int kmy = std::min(kms, M.kmz[lN - 1]);
      first = 0;
      for (int k = k1; k <= kmy; ++k) {
        double v = std::min(M.zlv(k + 1), M.hhv[l - 1]) - std::max(M.zlv(k), -(M.s0[l - 1] + M.s0[lN - 1]) / 2.);
        if (v > 0.0) { if (!first) { first = 1; M.k1v0[l - 1] = k; } }
        else v = 0.0;
        M.hvp0[M.I3(k, l)] = v;
      }
    }
  }
  M.salp0.assign(n3, 0.0);
  for (int l = 1; l <= lm1; ++l)
    for (int k = 1; k <= km1; ++k) M.salp0[M.I3(k, l)] = prof[k - 1];
  // tracer(k, :, nn) = column nn + 1 for every column incl. lm1 (:335-351, ecomod = 0)
  M.tracer0.assign(n3 * M.ntr, 0.0);
  for (int nn = 1; nn <= M.ntr; ++nn)
    for (int l = 1; l <= lm1; ++l)
      for (int k = 1; k <= km1; ++k) M.tracer0[n3 * (nn - 1) + M.I3(k, l)] = prof[(size_t)nn * km1 + k - 1];
  M.Av0f.assign(n3, 0.0); M.Dv0f.assign(n3, 0.0);
  if (M.iturb == 1) {
    // InitializeTurbulenceModel CASE(1) (si3d_mixing.f90:679-719): q2 = q2_min everywhere, q2l
    // = q2 times the mixing length kappa z sqrt(1 - z / htot) below each column's top layer (htot
    // sums hp over every layer, the sediment layer included); the eddy coefficients stay zero
    // until the first fd
    M.q2l0.assign(n3, 0.0);
    for (int l = 1; l <= M.lm; ++l) {
      const int kms = M.kmz[l - 1], k1s = M.k1z0[l - 1];
      double htot = 0.0;
      for (int k = 1; k <= km1; ++k) htot += M.hp0[M.I3(k, l)];
      if (kms <= k1s) continue;
      double z0 = 0.0;
      for (int k = k1s + 1; k <= kms; ++k) {
        z0 = z0 + M.hp0[M.I3(k - 1, l)];
        const double mixl = 0.41 * z0 * std::sqrt(std::max(1. - (z0 / htot), 0.0));
        M.q2l0[M.I3(k, l)] = 2.e-6 * mixl;
      }
    }
    return;
  }
  for (int l = 1; l <= M.lm; ++l) {
    const int kms = M.kmz[l - 1], k1s = M.k1z0[l - 1];
    for (int k = k1s + 1; k <= kms; ++k) { M.Av0f[M.I3(k, l)] = M.Av0; M.Dv0f[M.I3(k, l)] = M.Dv0; }
    // Av(k1s) and Av(kms+1) stay zero (si3d_mixing.f90:661-669)
  }
}


// compute_date (si3d_utils.f90:3546-3674): REAL variables as double, NINT rounding half away from
// zero, the month table kept between calls as the reference's SAVEd local.
void compute_date(HostModel& M, double itime_sec) {
  HostModel::Date& D = M.date;
  auto leap = [](int y) { return y % 4 == 0; };
  if (itime_sec == 0) {
    D.iyrp = M.iyr0; D.imonp = M.imon0; D.idayp = M.iday0; D.ihrp = M.ihr0; D.isecp = D.isec0;
    D.iyr = M.iyr0; D.imon = M.imon0; D.iday = M.iday0; D.ihr = M.ihr0; D.isec = D.isec0;
    if (leap(D.iyrp)) D.month[1] = 29;
    return;
  }
  D.isecp += itime_sec;
  if (D.isecp < 86400) {
    D.isec = D.isecp;
    D.ihrp = (int)std::lround(D.isec / 3600. * 100.);
    D.ihr = D.ihrp;
    return;
  }
  D.idayp = (int)(D.idayp + D.isecp / 86400);
  D.isecp = std::fmod(D.isecp, 86400.);
  D.isec = D.isecp;
  D.ihrp = (int)std::lround(D.isec / 3600. * 100.);
  D.ihr = D.ihrp;
  if (D.imonp == 2) D.month[1] = leap(D.iyrp) ? 29 : 28;
  if (D.idayp <= D.month[D.imonp - 1]) {
    D.iday = D.idayp;
    return;
  }
  const int months = (int)(itime_sec / 2500000 + 1);
  for (int j = 1; j <= months; ++j) {
    D.idayp -= D.month[D.imonp - 1];
    if (++D.imonp == 13) {
      D.imonp = 1;
      ++D.iyrp;
      D.month[1] = leap(D.iyrp) ? 29 : 28;
    }
    if (D.idayp <= D.month[D.imonp - 1]) {
      D.iday = D.idayp;
      break;
    }
  }
  D.imon = D.imonp;
  D.iyr = D.iyrp;
}

// Fortran unformatted sequential record: byte length, payload, byte length (4-byte integers).
bool put_record(HostModel& M, FILE* f, const void* head, size_t nh, const void* body, size_t nb) {
  const int32_t len = (int32_t)(nh + nb);
  bool ok = std::fwrite(&len, 4, 1, f) == 1 && (nh == 0 || std::fwrite(head, 1, nh, f) == nh) &&
            (nb == 0 || std::fwrite(body, 1, nb, f) == nb) && std::fwrite(&len, 4, 1, f) == 1;
  ok = ok && std::fflush(f) == 0;
  if (!ok) M.err = "output: write failed";
  return ok;
}

std::shared_ptr<FILE> open_output(HostModel& M, const std::string& name) {
  FILE* f = std::fopen((M.dir + "/" + name).c_str(), "wb");
  if (!f) { M.err = "output: cannot open " + name; return nullptr; }
  return std::shared_ptr<FILE>(f, [](FILE* q) { std::fclose(q); });
}

constexpr int kMaxFramesInFlight = 4;

void writer_loop(HostModel* M) {
  for (;;) {
    HostModel::Job j;
    {
      std::unique_lock<std::mutex> lk(M->wmu);
      M->wcv.wait(lk, [&] { return M->stop || !M->jobs.empty(); });
      if (M->jobs.empty()) return;
      j = std::move(M->jobs.front());
      M->jobs.pop_front();
    }
    int rc = j.ticket ? si3d_gpu_output_wait(M->gpu, j.ticket) : 0;
    if (!rc && !put_record(*M, j.f.get(), j.head.data(), j.head.size(), j.buf.p, (size_t)j.count * 4)) rc = SI3D_EDIMS;
    {
      std::lock_guard<std::mutex> lk(M->wmu);
      if (rc && !M->werr) M->werr = rc;
      if (j.buf.p) M->free_bufs.push_back(j.buf);
      --M->in_flight;
    }
    M->wcv.notify_all();
  }
}

void enqueue(HostModel& M, HostModel::Job&& j) {
  {
    std::lock_guard<std::mutex> lk(M.wmu);
    if (!M.writer.joinable()) M.writer = std::thread(writer_loop, &M);
    ++M.in_flight;
    M.jobs.push_back(std::move(j));
  }
  M.wcv.notify_all();
}

// Wait until every queued record is written; returns the writer's first error.
int drain(HostModel& M) {
  std::unique_lock<std::mutex> lk(M.wmu);
  M.wcv.wait(lk, [&] { return M.in_flight == 0; });
  return M.werr;
}

bool header_records(HostModel& M, const std::shared_ptr<FILE>& f, int frames, long long points) {
  for (int32_t v : {(int32_t)frames, (int32_t)points}) {
    HostModel::Job j;
    j.f = f;
    j.head.resize(4);
    std::memcpy(j.head.data(), &v, 4);
    enqueue(M, std::move(j));
  }
  return true;
}

// One frame: packed on the device and copied asynchronously into a page-locked buffer; the record
// (time stamp n, year, month, day, hour, si3d_utils.f90:2540-2541, then the frame) is written by
// the writer thread once the copy has landed.
int frame_record(HostModel& M, const std::shared_ptr<FILE>& f, int n, int kind, int arg) {
  long long cnt = 0;
  int rc = si3d_gpu_output_frame(M.gpu, kind, arg, n == 0, nullptr, 0, &cnt);
  if (rc) return rc;
  HostModel::Buf buf;
  {
    std::unique_lock<std::mutex> lk(M.wmu);
    M.wcv.wait(lk, [&] { return M.in_flight < kMaxFramesInFlight; });
    if (M.werr) return M.werr;
    for (size_t i = 0; i < M.free_bufs.size(); ++i)
      if (M.free_bufs[i].cap >= cnt) { buf = M.free_bufs[i]; M.free_bufs.erase(M.free_bufs.begin() + i); break; }
  }
  if (!buf.p) {
    void* p = nullptr;
    if ((rc = si3d_gpu_host_alloc(std::max<long long>(cnt, 1) * 4, &p))) return rc;
    buf.p = static_cast<float*>(p);
    buf.cap = std::max<long long>(cnt, 1);
  }
  HostModel::Job j;
  j.f = f;
  j.buf = buf;
  rc = si3d_gpu_output_frame_async(M.gpu, kind, arg, n == 0, buf.p, buf.cap, &j.count, &j.ticket);
  if (rc) {
    std::lock_guard<std::mutex> lk(M.wmu);
    M.free_bufs.push_back(buf);
    return rc;
  }
  j.head.resize(20);
  const int32_t iv[4] = {n, M.date.iyr, M.date.imon, M.date.iday};
  const float hour = (float)M.date.ihr;
  std::memcpy(j.head.data(), iv, 16);
  std::memcpy(j.head.data() + 16, &hour, 4);
  enqueue(M, std::move(j));
  return 0;
}

// The output calls of the time loop (si3d.f90:430-438; with n = 0 the initial ones, :89-100):
// outh (planes), outz (tracers), outp (ptrack file).  Files go to the run directory.
// outs (si3d_utils.f90:2605-2760) with ipxml < 0: on its first call the XML header of the Gr viewer's
// binary space files, and the two binary files opened empty.  The reference writes nothing more: its
// frame writer outs_bin (:2763) is not called anywhere, so the binary files stay empty.  runNumber
// is the wall-clock date and time (date_and_time), as in the reference.
int write_space_xml(HostModel& M) {
  FILE* f = std::fopen((M.dir + "/spacefile.xml").c_str(), "w");
  if (!f) { M.err = "output: cannot open spacefile.xml"; return SI3D_EDIMS; }
  for (const char* b : {"spacefile2d.bin", "spacefile3d.bin"}) {
    FILE* g = std::fopen((M.dir + "/" + b).c_str(), "wb");
    if (!g) { std::fclose(f); M.err = std::string("output: cannot open ") + b; return SI3D_EDIMS; }
    std::fclose(g);
  }
  // int_to_char(v, 0): the value left-justified between quotes
  auto quoted = [](long long v) { return "\"" + std::to_string(v) + "\""; };
  std::fprintf(f, "<?xml version=\"1.0\"?>\n \n<!-- Si3D Output for Gr -->\n");
  std::fprintf(f, "<!-- xml header file for binary spacefiles -->\n");
  std::fprintf(f, "<!-- Run Parameters:  dt =%5.2f s  dz =%5.2f m  im =%5d  jm =%5d\n", M.idt, M.idz, M.im, M.jm);
  std::fprintf(f, "     itrsca =%2d  itrap =%2d  cd = %7.4f  ismooth =%2d  beta =%6.3f  niter =%2d\n", M.itrsca, M.itrap,
               M.cd, M.ismooth, M.beta, M.niter);
  std::fprintf(f, "     itrmom =%2d  f =%7.4f  wa =%8.1f -->\n \n", M.itrmom, M.f, M.wa);
  std::fprintf(f, "<gov.usgs.gr>\n   <obj class=\"gov.usgs.sfhydro.si3d.Si3dOutput\"\n");
  std::string title = M.title;
  while (!title.empty() && title.back() == ' ') title.pop_back();
  std::fprintf(f, "        runTitle=\"%s\"\n", title.c_str());
  std::time_t now = std::time(nullptr);
  std::tm lt{};
  localtime_r(&now, &lt);
  std::fprintf(f, "        runNumber=\"%04d%02d%02d%02d%02d\"\n", lt.tm_year + 1900, lt.tm_mon + 1, lt.tm_mday, lt.tm_hour,
               lt.tm_min);
  // start of the output: itspf rounded up to a multiple of ipxml * idt (idt2 < 0 for ipxml < 0)
  const long long idt2 = (long long)M.ipxml * (long long)M.idt;
  HostModel::Date saved = M.date;
  if (M.itspf == 0) {
    compute_date(M, 0.0);
  } else {
    long long itspf1 = (M.itspf / idt2) * idt2;
    if (M.itspf % idt2 != 0) itspf1 += idt2;
    compute_date(M, (double)itspf1);
  }
  const int ihr2 = (int)(M.date.isec / 3600);
  int isec2 = (int)(M.date.isec - ihr2 * 3600);
  const int imin2 = isec2 / 60;
  isec2 = isec2 - imin2 * 60;
  std::fprintf(f, "        startTime=\"%4d/%02d/%02d %02d:%02d:%02d\" timeStepInSeconds=%s>\n", M.date.iyr, M.date.imon,
               M.date.iday, ihr2, imin2, isec2, quoted(idt2).c_str());
  M.date = saved;
  compute_date(M, 0.0);   // reset to the start of the run, as outs does
  M.date = saved;
  std::fprintf(f, " \n      <obj class=\"gov.usgs.gr.GrObjectContainer\" title=\"2-D x-y Variables\">\n");
  std::fprintf(f, "         <dataseries class=\"gov.usgs.gr.data.RafDataSeries\"\n");
  std::fprintf(f, "            file=\"spacefile2d.bin\"\n");
  std::fprintf(f, "            title=\"2-D Variables\" numDimensions=%s>\n", quoted(1).c_str());
  std::fprintf(f, "            <dim num=\"0\" title=\"Zeta\" units=\"meters\" unitScale=\"0.0001\"/>\n \n");
  std::fprintf(f, "         </dataseries>\n      </obj>\n \n");
  std::fprintf(f, "      <obj class=\"gov.usgs.gr.GrObjectContainer\" title=\"3-D Variables\">\n");
  std::fprintf(f, "         <dataseries class=\"gov.usgs.gr.data.RafDataSeries\"\n");
  std::fprintf(f, "            file=\"spacefile3d.bin\"\n");
  std::fprintf(f, "            title=\"3-D Variables\" numDimensions=%s>\n", quoted(4).c_str());
  std::fprintf(f, "            <dim num=\"0\" title=\"u\" units=\"m/s\" unitScale=\"0.0001\"/>\n");
  std::fprintf(f, "            <dim num=\"1\" title=\"v\" units=\"m/s\" unitScale=\"0.0001\"/>\n");
  std::fprintf(f, "            <dim num=\"2\" title=\"w\" units=\"m/s\" unitScale=\"0.00001\"/>\n");
  std::fprintf(f, "            <dim num=\"3\" title=\"dz\" units=\"m**2/s\" unitScale=\"0.0001\"/>\n \n");
  std::fprintf(f, "         </dataseries>\n      </obj>\n   </obj>\n</gov.usgs.gr>\n \n");
  std::fclose(f);
  M.space_written = true;
  return 0;
}

int write_outputs(HostModel& M, int n) {
  int rc = 0;
  const int apxml = std::abs(M.ipxml);
  if (M.iop > 0 && (n == 0 || (n >= M.itspfh && n % std::max(M.iop, 1) == 0))) {
    if (n == 0) {
      M.f_plane.clear();
      for (int kp : M.p_out) {
        if (kp < M.k1) { M.err = "output plane is not in the domain"; return SI3D_EDIMS; }
        auto f = open_output(M, "plane_" + std::to_string(kp));
        long long cnt = 0;
        if (!f) return SI3D_EDIMS;
        if ((rc = si3d_gpu_output_frame(M.gpu, SI3D_OUT_PLANE, kp, 1, nullptr, 0, &cnt))) return rc;
        if (!header_records(M, f, (M.nts - M.itspfh) / std::max(M.iop, 1), cnt / 8)) return SI3D_EDIMS;
        M.f_plane.push_back(f);
      }
    }
    for (size_t j = 0; j < M.p_out.size(); ++j)
      if ((rc = frame_record(M, M.f_plane[j], n, SI3D_OUT_PLANE, M.p_out[j]))) return rc;
  }
  long long pts = 0;
  for (int l = 0; l < M.lm; ++l) pts += M.kmz[l] + 2 - M.k1;
  if (M.iotr > 0 && M.ntr > 0 && (n == 0 || n % std::max(M.iotr, 1) == 0)) {
    if (n == 0) {
      M.f_tracer.clear();
      for (int t = 1; t <= M.ntr; ++t) {
        auto f = open_output(M, "tracer_" + std::to_string(t));
        if (!f || !header_records(M, f, (M.nts - M.itspftr) / std::max(M.iotr, 1), pts)) return SI3D_EDIMS;
        M.f_tracer.push_back(f);
      }
    }
    for (int t = 1; t <= M.ntr; ++t)
      if ((rc = frame_record(M, M.f_tracer[t - 1], n, SI3D_OUT_TRACER, t))) return rc;
  }
  // outs, called at n = 0 and every step (MOD(n, MAX(ipxml, 1)) with ipxml < 0), writes once
  if (M.ipxml < 0 && !M.space_written && (rc = write_space_xml(M))) return rc;
  if (M.ipxml > 0 && (n == 0 || (n >= M.itspf && n % std::max(apxml, 1) == 0))) {
    if (n == 0) {
      M.f_ptrack = open_output(M, "si3d_3D");
      if (!M.f_ptrack || !header_records(M, M.f_ptrack, (M.nts - M.itspf) / std::max(apxml, 1), pts))
        return SI3D_EDIMS;
    }
    if ((rc = frame_record(M, M.f_ptrack, n, SI3D_OUT_PTRACK, 0))) return rc;
  }
  return 0;
}

}  // namespace

extern "C" {

// The series of each open boundary: openbcNN.txt with five header records, the record count in
// '(10X,I7)', then '(10X,(ntr+2)G11.2)' records of which the first two values (elevation,
// temperature) are used (openbc0, si3d_boundaryconditions.f90:55-91).
bool read_openbc(HostModel& M, const std::string& dir) {
  std::vector<std::vector<double>> w(M.nopen), t(M.nopen);
  int npts = -1;
  for (int nn = 1; nn <= M.nopen; ++nn) {
    char name[32];
    std::snprintf(name, sizeof name, "openbc%02d.txt", nn);
    Records R;
    if (!R.load(dir + "/" + name)) { M.err = std::string("cannot open ") + name; return false; }
    R.skip(5);
    double np = 0;
    if (!numeric(R.take(), 10, 7, np) || np < 3) { M.err = std::string(name) + ": bad record count"; return false; }
    for (int j = 0; j < (int)np; ++j) {
      if (!R.more()) { M.err = std::string(name) + ": truncated"; return false; }
      const std::string row = R.take();
      double a = 0, b = 0;
      if (!numeric(row, 10, 11, a) || !numeric(row, 21, 11, b)) { M.err = std::string(name) + ": bad value"; return false; }
      w[nn - 1].push_back(a);
      t[nn - 1].push_back(b);
    }
    npts = npts < 0 ? (int)np : std::min(npts, (int)np);
  }
  M.ob_npts = npts;
  for (int nn = 0; nn < M.nopen; ++nn) {
    M.ob_wse.insert(M.ob_wse.end(), w[nn].begin(), w[nn].begin() + npts);
    M.ob_tmp.insert(M.ob_tmp.end(), t[nn].begin(), t[nn].begin() + npts);
  }
  return true;
}

int si3d_host_open(const char* run_dir, const si3d_solver_opts* opts, int* hm, char* err, int errlen) {
  auto M = std::make_unique<HostModel>();
  if (opts) M->opt = *opts;
  else { M->opt.pcg_test = 5; M->opt.pcg_tol = 1e-12; M->opt.pcg_itmax = 200; M->opt.srelpr = 2.220446049250313e-16; }
  const std::string dir = run_dir ? run_dir : ".";
  std::vector<double> prof;
  bool ok = read_parameters(*M, dir) && read_bathymetry(*M, dir) && read_profile(*M, dir, prof) && read_wind(*M, dir) &&
            (M->nopen == 0 || read_openbc(*M, dir));
  if (!ok) {
    if (err && errlen > 0) { std::strncpy(err, M->err.c_str(), errlen - 1); err[errlen - 1] = 0; }
    return SI3D_EDIMS;
  }
  initial_state(*M, prof);
  M->dir = dir;
  M->date.isec0 = (double)M->ihr0 / 100. * 3600.;   // si3d_utils.f90:310
  compute_date(*M, 0.0);                              // :43
  std::lock_guard<std::mutex> lk(g_mu);
  g_models.push_back(std::move(M));
  *hm = (int)g_models.size() - 1;
  return 0;
}

int si3d_host_dims(int h, int* dims) {
  HostModel* M = model(h);
  if (!M) return SI3D_EHANDLE;
  dims[0] = M->im1; dims[1] = M->jm1; dims[2] = M->km1; dims[3] = M->lm; dims[4] = M->km; dims[5] = M->nts;
  return 0;
}

int si3d_host_get_map(int h, const char* name, int* out) {
  HostModel* M = model(h);
  if (!M) return SI3D_EHANDLE;
  const std::string n = name ? name : "";
  const std::vector<int>* v = n == "l2i" ? &M->l2i : n == "l2j" ? &M->l2j : n == "lEC" ? &M->lEC : n == "lWC" ? &M->lWC
                            : n == "lNC" ? &M->lNC : n == "lSC" ? &M->lSC : n == "kmz" ? &M->kmz : nullptr;
  if (!v) return SI3D_ENAME;
  std::memcpy(out, v->data(), sizeof(int) * v->size());
  return 0;
}

int si3d_host_get_zlevel(int h, double* out) {
  HostModel* M = model(h);
  if (!M) return SI3D_EHANDLE;
  std::memcpy(out, M->zlevel.data(), sizeof(double) * M->zlevel.size());
  return 0;
}

int si3d_host_attach_gpu(int h, int device, int* gpu_handle) {
  HostModel* M = model(h);
  if (!M) return SI3D_EHANDLE;
  si3d_grid g{};
  g.im1 = M->im1; g.jm1 = M->jm1; g.km1 = M->km1; g.k1 = M->k1; g.lm = M->lm;
  g.l2i = M->l2i.data(); g.l2j = M->l2j.data();
  g.lEC = M->lEC.data(); g.lWC = M->lWC.data(); g.lNC = M->lNC.data(); g.lSC = M->lSC.data();
  g.kmz = M->kmz.data(); g.hhs = M->hhs.data(); g.hhu = M->hhu.data(); g.hhv = M->hhv.data();
  g.zlevel = M->zlevel.data();
  si3d_params p{};
  p.dt = M->idt; p.dx = M->idx; p.dy = M->idy;
  p.Av0 = M->Av0; p.Dv0 = M->Dv0; p.Ax0 = M->Ax0; p.Ay0 = M->Ay0; p.f = M->f; p.theta = M->theta; p.cd = M->cd;
  p.cw = M->cw; p.beta = M->beta;
  p.iadv = M->iadv; p.itrmom = M->itrmom; p.ihd = M->ihd; p.ibc = M->ibc; p.isal = M->isal; p.itrap = M->itrap;
  p.niter = M->niter; p.ismooth = M->ismooth;
  p.pcg_test = M->opt.pcg_test; p.pcg_tol = M->opt.pcg_tol; p.pcg_itmax = M->opt.pcg_itmax; p.srelpr = M->opt.srelpr;
  p.ordering = M->opt.ordering == SI3D_ORDER_NATURAL ? SI3D_ORDER_NATURAL : SI3D_ORDER_REDBLACK;
  p.x0_mode = M->opt.x0_mode; p.precision = M->opt.precision;
  p.ntr = M->ntr;
  p.iturb = M->iturb;
  int gh = -1;
  int rc = si3d_gpu_init(&g, &p, device, &gh);
  if (rc) return rc;
  // initial fields (init: s = sp = spp; hpp = hp = h; k1 indices; sal = salp = salpp; Av/Dv)
  const char* same_s[] = {"s", "sp", "spp"};
  for (const char* nm : same_s) if ((rc = si3d_gpu_set_field(gh, nm, M->s0.data()))) return rc;
  if (M->nopen > 0) {
    // openbc0 (si3d.f90:64, after init): the boundary cells' sp takes the series' first value
    std::vector<double> sp0 = M->s0;
    for (int nn = 0; nn < M->nopen; ++nn) {
      const bool x = M->ob_side[nn] == 1 || M->ob_side[nn] == 3;
      const int a = x ? M->ob_js[nn] : M->ob_is[nn], e = x ? M->ob_je[nn] : M->ob_ie[nn];
      for (int q = a; q <= e; ++q) {
        const int i = x ? M->ob_is[nn] : q, j = x ? q : M->ob_js[nn];
        if (i < 1 || j < 1 || i > M->im1 || j > M->jm1 || !M->W(i, j)) return SI3D_EDIMS;
        sp0[M->L(i, j) - 1] = M->ob_wse[(size_t)nn * M->ob_npts];
      }
    }
    if ((rc = si3d_gpu_set_field(gh, "sp", sp0.data()))) return rc;
    if ((rc = si3d_gpu_set_open_boundaries(gh, M->nopen, M->ob_side.data(), M->ob_type.data(), M->ob_is.data(),
                                           M->ob_js.data(), M->ob_ie.data(), M->ob_je.data(), M->obc_dtsec,
                                           M->ob_npts, M->ob_wse.data(), M->ob_tmp.data())))
      return rc;
  }
  const char* same_h[] = {"h", "hp", "hpp"};
  for (const char* nm : same_h) if ((rc = si3d_gpu_set_field(gh, nm, M->hp0.data()))) return rc;
  const char* same_hu[] = {"hu", "hup", "hupp"};
  for (const char* nm : same_hu) if ((rc = si3d_gpu_set_field(gh, nm, M->hup0.data()))) return rc;
  const char* same_hv[] = {"hv", "hvp", "hvpp"};
  for (const char* nm : same_hv) if ((rc = si3d_gpu_set_field(gh, nm, M->hvp0.data()))) return rc;
  const char* same_t[] = {"sal", "salp", "salpp"};
  for (const char* nm : same_t) if ((rc = si3d_gpu_set_field(gh, nm, M->salp0.data()))) return rc;
  for (int nn = 1; nn <= M->ntr; ++nn) {   // tracerpp = tracer (:352)
    const double* t0 = M->tracer0.data() + (size_t)(nn - 1) * M->km1 * M->lm1;
    const std::string a = "tracer" + std::to_string(nn), b = "tracerpp" + std::to_string(nn);
    if ((rc = si3d_gpu_set_field(gh, a.c_str(), t0))) return rc;
    if ((rc = si3d_gpu_set_field(gh, b.c_str(), t0))) return rc;
  }
  if (M->iturb == 1) {
    const std::vector<double> qmin((size_t)M->km1 * M->lm1, 2.e-6);
    for (const char* nm : {"q2", "q2p", "q2pp"}) if ((rc = si3d_gpu_set_field(gh, nm, qmin.data()))) return rc;
    for (const char* nm : {"q2l", "q2lp", "q2lpp"}) if ((rc = si3d_gpu_set_field(gh, nm, M->q2l0.data()))) return rc;
  }
  if ((rc = si3d_gpu_set_field(gh, "Av", M->Av0f.data()))) return rc;
  if ((rc = si3d_gpu_set_field(gh, "Dv", M->Dv0f.data()))) return rc;
  if ((rc = si3d_gpu_set_field(gh, "uair", M->uair.data()))) return rc;
  if ((rc = si3d_gpu_set_field(gh, "vair", M->vair.data()))) return rc;
  if ((rc = si3d_gpu_set_field(gh, "cdw", M->cdw.data()))) return rc;
  std::vector<double> one(M->lm1, 1.0);
  if ((rc = si3d_gpu_set_field(gh, "rr", one.data()))) return rc;
  if ((rc = si3d_gpu_set_ifield(gh, "k1z", M->k1z0.data()))) return rc;
  if ((rc = si3d_gpu_set_ifield(gh, "k1u", M->k1u0.data()))) return rc;
  if ((rc = si3d_gpu_set_ifield(gh, "k1v", M->k1v0.data()))) return rc;
  if ((rc = si3d_gpu_density(gh))) return rc;   // rhop from the initial profile (:363-373)
  M->gpu = gh;
  M->n = 0;
  if ((rc = write_outputs(*M, 0))) return rc;   // the initial frames (si3d.f90:89-100)
  if ((rc = drain(*M))) return rc;
  if (gpu_handle) *gpu_handle = gh;
  return 0;
}

int si3d_host_run(int h, int nsteps, si3d_step_stats* stats) {
  HostModel* M = model(h);
  if (!M) return SI3D_EHANDLE;
  if (M->gpu < 0) return SI3D_EHANDLE;
  for (int s = 0; s < nsteps; ++s) {
    const int n = M->n + 1;
    compute_date(*M, M->idt);   // si3d.f90:333
    int rc = si3d_gpu_step(M->gpu, n, stats ? &stats[s] : nullptr);
    if (rc) return rc;
    M->n = n;
    if ((rc = write_outputs(*M, n))) return rc;
  }
  return drain(*M);   // every record of these steps is in its file when the call returns
}

int si3d_host_step_count(int h) {
  HostModel* M = model(h);
  return M ? M->n : SI3D_EHANDLE;
}

void si3d_host_close(int h) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (h < 0 || h >= (int)g_models.size() || !g_models[h]) return;
  drain(*g_models[h]);   // the writer still needs the device handle for its last copies
  if (g_models[h]->gpu >= 0) si3d_gpu_finalize(g_models[h]->gpu);
  g_models[h].reset();
}

}  // extern "C"
