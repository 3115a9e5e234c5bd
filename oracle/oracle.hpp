// CPU oracle for the pSi3D per-timestep semi-implicit core — TEST INFRASTRUCTURE ONLY.
//
// This is a plain, single-threaded FP64 restatement ("the reference with REAL -> REAL(8)")
// of the Fortran routines on the hot path, written routine by routine with file:line
// citations into the reference (si3d.f90, si3d_procedures.f90, si3d_utils.f90,
// si3d_boundaryconditions.f90, si3d_mixing.f90, nspcg.f).  Arrays keep the reference's
// Fortran layout: 3-D fields are (km1, lm1) column-major with k fastest, every index is
// 1-based, and column lm1 is the dry sentinel.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this code,
// and only as the checker or the timed CPU baseline.  The product (si3d_b200) never links it.
//
// Parity pinning: the reference ships no tests, golden vectors or outputs for this path, and
// it cannot be compiled here (no Fortran compiler; GOTM is not vendored).  Parity is
// therefore UNPINNED by reference golden data; the oracle is pinned instead by analytic
// known-answer tests (lake at rest, closed-basin volume invariant, surface-seiche period,
// manufactured PCG solutions, dense tridiagonal solves) under tests/.
#pragma once
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

namespace orc {

using real = double;

// Solver/harness options that the reference hard-codes (si3d_procedures.f90:1989-1995)
// plus the harness overlay (ordering, x0 mode, srelpr).
struct Opts {
  int pcg_test = 5;          // NSPCG stopping test: 2 or 5 (nspcg.f:25956-26100)
  double pcg_tol = 1e-12;    // rparm(1) (zeta)
  int pcg_itmax = 200;       // iparm(2)
  int ordering = 0;          // 0 natural (iperm=0), 1 red-black (NSPCG iperm=1 via prbndx)
  int x0_mode = 0;           // 0 previous step sp (si3d_procedures.f90:1970), 1 zero
  double srelpr = 2.220446049250313e-16;  // nspcg.f:33208 double-precision value
};

struct SolveLog {
  int n, istep, iter, iters, ier;
  double stptst, emin, emax;
};

// Input parameters read by `input` (si3d_utils.f90:21-315).
struct Inp {
  std::string title;
  int iyr0 = 0, imon0 = 0, iday0 = 0, ihr0 = 0;
  real xl = 0, yl = 0, zl = 0, tl = 0, idx = 0, idy = 0, idz = 0, dzmin = 0, datadj = 0,
       zetainit = 0, idt = 0;
  int ibathyf = 0;
  int itrap = 1, niter = 2, ismooth = 0;
  real beta = 0.05;
  int iturb = 0;
  real Av0 = 0, Dv0 = 0;
  int iadv = 1, itrmom = 1, ihd = 1;
  real Ax0 = 0, Ay0 = 0, f = 0, theta = 1;
  int ibc = 1, isal = 1, itrsca = 0;
  real cd = 0;
  int ifsurfbc = 0;
  real dtsurfbc = 0;
  int icw = 0;
  real cw = 0, wa = 0, phi = 0;
  int idbg = 0, num_threads = 1;
  int ipt = 0, nnodes = 0, iop = 0, itspfh = 0, n_planes = 0, iox = 0, ipxml = 0, itspf = 0,
      iTurbVars = 0, nopen = 0, nxNBO = 0, ntr = 0, iopss = 0;
  // tracer block (si3d_utils.f90:172-181), read when ntr > 0
  int ecomod = 0, iotr = 0, itspftr = 0, ipwq = 0, nswq = 0;
  std::vector<int> p_out;   // output planes (si3d_utils.f90:80-83)
};

// One open boundary (si3d_utils.f90:124-140): side (1 W, 2 N, 3 E, 4 S), type (1 = water-surface
// elevation specified, the only type restated), the cell range, and the series read from its
// openbcNN.txt file (openbc0, si3d_boundaryconditions.f90:55-91): wse and the scalar (temperature).
struct OpenBC {
  int iside = 0, itype = 0, isbc = 0, jsbc = 0, iebc = 0, jebc = 0;
  std::vector<double> wse, sal;
};

// Calendar of compute_date (si3d_utils.f90:3546-3674); REAL variables as double.
struct Date {
  int iyr = 0, imon = 0, iday = 0, ihr = 0, iyrp = 0, imonp = 0, idayp = 0, ihrp = 0;
  double isec = 0, isecp = 0, isec0 = 0;
  int month[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};   // SAVEd between calls
};

struct F3 {  // (km1, lm1) column-major, 1-based
  std::vector<real> v;
  int km1 = 0, lm1 = 0;
  void init(int km1_, int lm1_, real val = 0) { km1 = km1_; lm1 = lm1_; v.assign((size_t)km1 * lm1, val); }
  real& operator()(int k, int l) { return v[(size_t)(l - 1) * km1 + (k - 1)]; }
  real operator()(int k, int l) const { return v[(size_t)(l - 1) * km1 + (k - 1)]; }
};
struct F1 {  // 1-based vector
  std::vector<real> v;
  void init(int n, real val = 0) { v.assign(n, val); }
  real& operator()(int i) { return v[i - 1]; }
  real operator()(int i) const { return v[i - 1]; }
};
struct I1 {
  std::vector<int> v;
  void init(int n, int val = 0) { v.assign(n, val); }
  int& operator()(int i) { return v[i - 1]; }
  int operator()(int i) const { return v[i - 1]; }
};

struct Model {
  Inp in;
  Opts opt;
  // grid (si3d_types.f90:77-82, si3d_utils.f90:300-306, 318-382)
  real dt, dx, dy, ddz, twodt, dtdx, dtdy, gdtdx, gdtdy, gdt2dx2, gdt2dy2, twodx, twody,
      fourdx, fourdy, dxdx, dydy, dxdy, beta2;
  int im, im1, i1, jm, jm1, j1, km, km1, k1, nts, lm, lm1;
  real tz = 1;
  std::vector<real> zlevel;  // 1-based through zl(k)
  real zl(int k) const { return zlevel[k - 1]; }
  // masks and maps (si3d_utils.f90:595-892)
  std::vector<uint8_t> mask2d_;  // (i,j) 1-based, im1 x jm1, i fastest
  bool mask2d(int i, int j) const { return mask2d_[(size_t)(j - 1) * im1 + (i - 1)] != 0; }
  std::vector<int> ij2l_;
  int ij2l(int i, int j) const { return ij2l_[(size_t)(j - 1) * im1 + (i - 1)]; }
  I1 l2i, l2j, lEC, lWC, lNC, lSC, kmz, k1z, k1u, k1v;
  F1 hhs, hhu, hhv;
  // 2-D state
  F1 s, sp, spp, eagx, earx, eagy, eary, sx, sy, dd, qq, rr, uair, vair, cdw;
  // 3-D state
  F3 uh, uhp, uhpp, u, up, upp, hu, hup, hupp, ex, agx, arx;
  F3 vh, vhp, vhpp, v, vp, vpp, hv, hvp, hvpp, agy, ary;
  F3 h, hp, hpp, sal, salp, salpp, rhop, Av, Dv, wp, HeatSource;
  // thread-private scratch that the reference keeps across calls (si3d.f90:299-316;
  // InitThreads si3d_procedures.f90:4838-4841 zero-initialises them)
  F3 Bth2, Bth3, Bth4, Bex, Bhaxpp, Bhaypp;
  // Mellor-Yamada 2.5 state (iturb = 1): 2 TKE and 2 TKE x length scale at n+1, n (or n+1/2), n-1
  F3 q2, q2p, q2pp, q2l, q2lp, q2lpp;
  // non-active tracers (si3d_utils.f90:571-574): tracer and tracerpp per tracer, ntr of each
  std::vector<F3> tracer, tracerpp;
  // binary output files (outp, outz, outh) written into the run directory, and the date stamp
  std::string dir;
  Date date;
  bool space_written = false;   // outs' first_entry
  std::shared_ptr<FILE> f_ptrack;
  std::vector<std::shared_ptr<FILE>> f_tracer, f_plane;
  // open boundaries (nopen > 0): records, series spacing dtsecOpenBC (s), hours of the current step
  std::vector<OpenBC> obc;
  double dtsec_obc = 0;
  double thrs = 0;
  // per-column wind override (harness overlay; surfbc CASE 0 otherwise)
  bool wind_override = false;
  std::vector<real> uair_ovr, vair_ovr;  // l-indexed (1..lm)
  // bookkeeping
  int n = 0;
  int istep = 1, lastiter = 0, iter = 0;
  std::vector<SolveLog> solves;
  std::string err;
  bool failed = false;
};

// I/O and setup
bool read_inputs(Model& m, const std::string& dir);  // input + ZGridDimensions + bathy + init
// open boundaries (oracle_obc.cpp)
bool read_openbc_files(Model& m, const std::string& dir);   // the openbcNN.txt series
bool openbc0(Model& m);                                      // checks and sp at t = 0
bool openbc_uvh(Model& m);                                   // s on the boundary cells at thrs
void mod_exmom_openbc(Model& m, int ieq);                    // ex of the faces at the boundaries
void mod_qq_openbc(Model& m);                                // qq and sx/sy of the zeta system
void mod_vel_openbc(Model& m);                               // vh/uh and wp of the boundary cells
void openbc_sca(Model& m);                                   // temperature of the boundary cells
double parab(double frstpt, double x, const std::vector<double>& fx, double dx);
void compute_date(Model& m, double itime_sec);
// Mellor-Yamada 2.5 (oracle_turb.cpp)
void init_turbulence(Model& m);
void settrap_2eq(Model& m);
void settrap2_2eq(Model& m);
void save_2eq(Model& m, int istep);
void update_mixing(Model& m, int istep);
bool write_outputs(Model& m, int n);   // outh, outz, outp as the time loop calls them for step n
// time loop
bool run_steps(Model& m, int nsteps);
// one routine (momentum, matcon, solve, vel, scalar, vel2, fd, settrap, settrap2, save)
bool run_stage(Model& m, const std::string& stage, int istep);
// routines used by unit tests
void trid(const real* aa /*3 x km1, 1-based in k*/, const real* g, const real* r, real* ag, real* ar,
          int k1, int km, int n);
void trid1(const real* aa, const real* dsal, real* sal, int k1, int km, int n);
real densty_s(real temperature, real salinity, real elevation);

// NSPCG mic1 + cg restatement.  coef/jcoef are ndim x 5 column-major (Purdue storage,
// diagonal in column 1, 1-based column indices, 0 = no entry).  u holds x0 on entry.
struct PcgResult {
  int iters = 0, ier = 0;
  real stptst = 0, emin = 0, emax = 0;
  std::vector<real> alphas, betas;
};
PcgResult nspcg_mic_cg(int n, const std::vector<real>& coef, const std::vector<int>& jcoef,
                       const std::vector<real>& rhs, std::vector<real>& u, const Opts& opt,
                       const std::vector<int>* color /* 1 red, 2 black; null = natural */);
// prbndx-equivalent 2-colouring of the matrix graph (nspcg.f:25337-25460): returns
// colours (1 red / 2 black) or empty when the matrix lacks property A.
std::vector<int> redblack_colors(int n, const std::vector<real>& coef, const std::vector<int>& jcoef);

}  // namespace orc
