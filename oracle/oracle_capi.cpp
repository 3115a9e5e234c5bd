// C entry points of the CPU oracle, loaded by tests/ and bench.py through ctypes —
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#include "oracle.hpp"

using namespace orc;

namespace {

F3* field3(Model& m, const std::string& n) {
  static const std::map<std::string, F3 Model::*> t = {
      {"uh", &Model::uh},     {"uhp", &Model::uhp},   {"uhpp", &Model::uhpp}, {"u", &Model::u},
      {"up", &Model::up},     {"upp", &Model::upp},   {"hu", &Model::hu},     {"hup", &Model::hup},
      {"hupp", &Model::hupp}, {"ex", &Model::ex},     {"agx", &Model::agx},   {"arx", &Model::arx},
      {"vh", &Model::vh},     {"vhp", &Model::vhp},   {"vhpp", &Model::vhpp}, {"v", &Model::v},
      {"vp", &Model::vp},     {"vpp", &Model::vpp},   {"hv", &Model::hv},     {"hvp", &Model::hvp},
      {"hvpp", &Model::hvpp}, {"agy", &Model::agy},   {"ary", &Model::ary},   {"h", &Model::h},
      {"hp", &Model::hp},     {"hpp", &Model::hpp},   {"sal", &Model::sal},   {"salp", &Model::salp},
      {"salpp", &Model::salpp}, {"rhop", &Model::rhop}, {"Av", &Model::Av},   {"Dv", &Model::Dv},
      {"wp", &Model::wp},     {"Bth2", &Model::Bth2}, {"Bth3", &Model::Bth3}, {"Bth4", &Model::Bth4},
      {"Bex", &Model::Bex},   {"q2", &Model::q2},     {"q2p", &Model::q2p},   {"q2pp", &Model::q2pp},
      {"q2l", &Model::q2l},   {"q2lp", &Model::q2lp}, {"q2lpp", &Model::q2lpp}};
  auto it = t.find(n);
  if (it != t.end()) return &(m.*(it->second));
  // "tracer<nt>" and "tracerpp<nt>", nt = 1..ntr
  for (auto [pre, vec] : {std::pair<const char*, std::vector<F3>*>{"tracerpp", &m.tracerpp},
                          std::pair<const char*, std::vector<F3>*>{"tracer", &m.tracer}}) {
    const size_t np = std::strlen(pre);
    if (n.size() > np && n.compare(0, np, pre) == 0 && n.find_first_not_of("0123456789", np) == std::string::npos) {
      const int nt = std::atoi(n.c_str() + np);
      return (nt >= 1 && nt <= (int)vec->size()) ? &(*vec)[nt - 1] : nullptr;
    }
  }
  return nullptr;
}

F1* field2(Model& m, const std::string& n) {
  static const std::map<std::string, F1 Model::*> t = {
      {"s", &Model::s},       {"sp", &Model::sp},     {"spp", &Model::spp},   {"eagx", &Model::eagx},
      {"earx", &Model::earx}, {"eagy", &Model::eagy}, {"eary", &Model::eary}, {"sx", &Model::sx},
      {"sy", &Model::sy},     {"dd", &Model::dd},     {"qq", &Model::qq},     {"rr", &Model::rr},
      {"uair", &Model::uair}, {"vair", &Model::vair}, {"cdw", &Model::cdw},   {"hhs", &Model::hhs},
      {"hhu", &Model::hhu},   {"hhv", &Model::hhv}};
  auto it = t.find(n);
  return it == t.end() ? nullptr : &(m.*(it->second));
}

I1* fieldi(Model& m, const std::string& n) {
  static const std::map<std::string, I1 Model::*> t = {
      {"l2i", &Model::l2i}, {"l2j", &Model::l2j}, {"lEC", &Model::lEC}, {"lWC", &Model::lWC},
      {"lNC", &Model::lNC}, {"lSC", &Model::lSC}, {"kmz", &Model::kmz}, {"k1z", &Model::k1z},
      {"k1u", &Model::k1u}, {"k1v", &Model::k1v}};
  auto it = t.find(n);
  return it == t.end() ? nullptr : &(m.*(it->second));
}

}  // namespace

extern "C" {

void* orc_create(const char* dir, int pcg_test, double pcg_tol, int pcg_itmax, int ordering, int x0_mode,
                 double srelpr, char* err, int errlen) {
  Model* m = new Model();
  m->opt.pcg_test = pcg_test;
  m->opt.pcg_tol = pcg_tol;
  m->opt.pcg_itmax = pcg_itmax;
  m->opt.ordering = ordering;
  m->opt.x0_mode = x0_mode;
  m->opt.srelpr = srelpr;
  if (!read_inputs(*m, dir)) {
    if (err && errlen > 0) { std::strncpy(err, m->err.c_str(), errlen - 1); err[errlen - 1] = 0; }
    delete m;
    return nullptr;
  }
  return m;
}

void orc_destroy(void* h) { delete static_cast<Model*>(h); }

const char* orc_error(void* h) { return static_cast<Model*>(h)->err.c_str(); }

int orc_run(void* h, int nsteps) { return run_steps(*static_cast<Model*>(h), nsteps) ? 0 : -1; }

int orc_stage(void* h, const char* stage, int istep) {
  return run_stage(*static_cast<Model*>(h), stage, istep) ? 0 : -1;
}

int orc_set_int(void* h, const char* name, const int* in) {
  Model& m = *static_cast<Model*>(h);
  if (I1* f = fieldi(m, name)) { std::memcpy(f->v.data(), in, sizeof(int) * f->v.size()); return 1; }
  return -1;
}

// im1, jm1, km1, lm, km, k1, nts, n, ntr
int orc_dims(void* h, int* out) {
  Model& m = *static_cast<Model*>(h);
  out[0] = m.im1; out[1] = m.jm1; out[2] = m.km1; out[3] = m.lm; out[4] = m.km; out[5] = m.k1;
  out[6] = m.nts; out[7] = m.n; out[8] = m.in.ntr;
  return 0;
}

int orc_zlevel(void* h, double* out) {
  Model& m = *static_cast<Model*>(h);
  std::memcpy(out, m.zlevel.data(), sizeof(double) * m.km1);
  return 0;
}

// 3-D fields come back (km1, lm1) column-major; 2-D fields have lm1 entries.
int orc_get(void* h, const char* name, double* out) {
  Model& m = *static_cast<Model*>(h);
  if (F3* f = field3(m, name)) { std::memcpy(out, f->v.data(), sizeof(double) * f->v.size()); return 3; }
  if (F1* f = field2(m, name)) { std::memcpy(out, f->v.data(), sizeof(double) * f->v.size()); return 2; }
  return -1;
}

int orc_set(void* h, const char* name, const double* in) {
  Model& m = *static_cast<Model*>(h);
  if (F3* f = field3(m, name)) { std::memcpy(f->v.data(), in, sizeof(double) * f->v.size()); return 3; }
  if (F1* f = field2(m, name)) { std::memcpy(f->v.data(), in, sizeof(double) * f->v.size()); return 2; }
  return -1;
}

int orc_get_int(void* h, const char* name, int* out) {
  Model& m = *static_cast<Model*>(h);
  if (I1* f = fieldi(m, name)) { std::memcpy(out, f->v.data(), sizeof(int) * f->v.size()); return 1; }
  return -1;
}

int orc_nsolves(void* h) { return (int)static_cast<Model*>(h)->solves.size(); }

// per solve: ints = n, istep, iter, iters, ier; reals = stptst, emin, emax
int orc_solve_log(void* h, int* ints, double* reals) {
  Model& m = *static_cast<Model*>(h);
  for (size_t i = 0; i < m.solves.size(); ++i) {
    const SolveLog& s = m.solves[i];
    ints[5 * i + 0] = s.n; ints[5 * i + 1] = s.istep; ints[5 * i + 2] = s.iter; ints[5 * i + 3] = s.iters;
    ints[5 * i + 4] = s.ier;
    reals[3 * i + 0] = s.stptst; reals[3 * i + 1] = s.emin; reals[3 * i + 2] = s.emax;
  }
  return (int)m.solves.size();
}

// Standalone NSPCG mic1 + cg on Purdue arrays (n x 5 column-major, 1-based, 0 = none).
int orc_pcg(int n, const double* coef, const int* jcoef, const double* rhs, double* u, int pcg_test, double tol,
            int itmax, int ordering, double srelpr, int* iters, double* stptst, double* emin, double* emax,
            double* alphas, double* betas) {
  std::vector<real> c(coef, coef + (size_t)5 * n), b(rhs, rhs + n), x(u, u + n);
  std::vector<int> j(jcoef, jcoef + (size_t)5 * n);
  Opts o;
  o.pcg_test = pcg_test; o.pcg_tol = tol; o.pcg_itmax = itmax; o.ordering = ordering; o.srelpr = srelpr;
  std::vector<int> col;
  if (ordering == 1) {
    col = redblack_colors(n, c, j);
    if (col.empty()) return -8;
  }
  PcgResult r = nspcg_mic_cg(n, c, j, b, x, o, ordering == 1 ? &col : nullptr);
  std::memcpy(u, x.data(), sizeof(double) * n);
  *iters = r.iters; *stptst = r.stptst; *emin = r.emin; *emax = r.emax;
  if (alphas) for (size_t i = 0; i < r.alphas.size(); ++i) alphas[i] = r.alphas[i];
  if (betas) for (size_t i = 0; i < r.betas.size(); ++i) betas[i] = r.betas[i];
  return r.ier;
}

// trid for unit tests: aa is (3, n) column-major for rows k1..km mapped to 1..n.
int orc_trid(int n, const double* aa, const double* g, const double* r, double* ag, double* ar) {
  orc::trid(aa, g, r, ag, ar, 1, n, n);
  return 0;
}

int orc_trid1(int n, const double* aa, const double* d, double* x) {
  orc::trid1(aa, d, x, 1, n, n);
  return 0;
}

double orc_densty(double t, double s, double z) { return orc::densty_s(t, s, z); }

}  // extern "C"
