// Declarations shared by the stage kernels and the C-ABI orchestration (si3d_gpu.cu).
#pragma once
#include "common.cuh"

namespace si3d {

// One colour of the red-black ordered zeta system (see k_zeta.cu), with vectors and coefficients
// of type T (double for the plain solve, float for the inner solve of iterative refinement).
template <typename T>
struct PcgColorT {
  int n;                 // nodes of this colour; arrays hold n + 1 entries (entry n = 0)
  const int* l;          // [n] reference column index (1-based)
  const int4* nbr;       // [n] W, S, N, E as indices into the other colour (absent -> other.n)
  T *sx, *sy, *rhs, *u, *r, *z, *p, *p2, *q, *dinv, *diag, *rs;   // p/p2: double-buffered search direction
};
using PcgColor = PcgColorT<double>;

// Device-resident CG scalars (NSPCG common blocks itcom1/itcom3 that itcg and pstops use).
struct PcgScal {
  double alpha, beta, alphao, rzdot, dkm1, pap, bnorm, stptst, zeta, srelpr, udnm, emin, emax;
  int in, itmax, ntest, done, ier, q1, hist_cap, negpiv;
  unsigned int cnt[4];
  // adaptive eigenvalue estimates of stopping test 2 (chgcon, itcom2/itcom3 of NSPCG)
  double tl1, tl2, bl1, bl2;
  int maxadp, minadp, chg_ier;
};

template <typename T>
struct PcgDevT {
  PcgColorT<T> R, B;
  PcgScal* sc;
  double *part0, *part1, *part2, *part3;   // block partials, part_n entries each, contiguous
  int part_n;
  double *hist_alpha, *hist_beta;
  double* tri;   // Lanczos tridiagonal of chgcon, 2 x (itmax + 2), column-major (test 2)
  // the iteration reads the gathered diagonal (matcon's rr) instead of forming it from sx and sy:
  // set for handles with open boundaries, whose cut faces leave rr larger than that sum
  bool diag_stored = false;
};
using PcgDev = PcgDevT<double>;
using PcgDevF = PcgDevT<float>;

// Launch shapes of the column stages that the autotuner picks per handle (results do not depend on
// them): layer lanes per column of the cell-parallel kernels (2, 4, 8) and threads per block of the
// column-sequential kernels (64, 128, 256).
struct Tune {
  int mom_cl = 8, mom_nt = 128, sal_cl = 8, sal_nt = 128;
};

// Static indices of one u (v) face column of the momentum stage, computed once from the grid maps
// so that the kernels start from one coalesced load instead of a chain of dependent lookups:
// a = (l, lE, lW, lN), b = (lS, lX2, kmx, mW_last), c = (mS_last, 0, 0, 0), where lX2 is lSC(lEC(l))
// (lWC(lNC(l)) for v), kmx the face depth, and mW_last / mS_last the last layer of the west / south
// neighbouring face's diffusion coefficient (-1 when that face contributes none).
struct FaceMeta {
  int4 a, b, c;
};

int momentum_init(int km1);
// Raises the continuity kernels' shared-memory limit for columns deeper than 95 levels.
int transport_init(int km1);
struct ObcDev;
// `obc` (nobc boundaries): open boundaries whose face columns' explicit term is recomputed between
// the cell and the column kernels
void launch_momentum(const Dev& d, int ieq, const FaceMeta* meta, int ncols, const Tune& tu, cudaStream_t st,
                     const ObcDev* obc = nullptr, int nobc = 0);
void launch_matcon(const Dev& d, cudaStream_t st);

void pcg_setup(const Dev& d, const PcgDev& P, int x0_mode, const double* dz, const double* hist, int* negpiv,
               cudaStream_t st);
void pcg_iteration(const PcgDev& P, int par, cudaStream_t st);
void pcg_finish(const Dev& d, const PcgDev& P, double* hist, cudaStream_t st);
// Graph-capturable solve pieces: scalars initialised by a kernel, statistics kept on the device.
void pcg_init_scalars(PcgScal* sc, const PcgScal& init, cudaStream_t st);
void pcg_record_stats(const PcgScal* sc, int ier0, int* iters_ier, double* relres, int slot, cudaStream_t st);
int pcg_max_blocks(int nR, int nB);
// Iterative refinement: FP64 residual r = rhs - A u and its squared norm into P.sc->stptst
// (the host compares it with bnorm); FP32 inner-system set-up from the FP64 residual; the
// FP32 iteration; the FP64 correction u += e.
void ir_residual(const PcgDev& P, cudaStream_t st);
void ir_inner_setup(const PcgDev& P, const PcgDevF& F, cudaStream_t st);
void pcg_iteration_f(const PcgDevF& F, int par, cudaStream_t st);
void ir_correct(const PcgDev& P, const PcgDevF& F, cudaStream_t st);

// Whole solve in one cooperative launch (k_pcg_persistent.cu).  The barrier state is reset by
// every launch.
// Grid barrier record, zeroed before every cooperative launch.  `absent` (blocks the barrier waits
// for beyond the grid) and `limit` (polls before a wait gives up; 0 = the built-in limit) are zero in
// every solve; a test sets them through si3d_gpu_test_wait_limit to make a wait run out.
struct GridBar {
  unsigned long long count;        // arrivals since the launch (never reset within it)
  unsigned int abort, absent;
  unsigned long long limit, pad;
};
int pcg_loop_blocks(int device, int nR, int nB, int max_per_sm, bool fp32);

// Natural-order MIC-CG (the reference's own ordering, SI3D_ORDER_NATURAL), k_pcg_persistent.cu.
// The unknowns are the wet columns in l order.  Each row keeps its four neighbours and their
// coefficients; `order` packs, 3 bits per slot, the codes (0 W, 1 S, 2 N, 3 E, 4 none) of the row's
// off-diagonal columns in the order NSPCG's move1 leaves them (upper columns first), which fixes
// the order of the sums in the SpMV and the backward sweep.  The triangular sweeps of the
// preconditioner are recurrences along l; they run level by level (a row's level is one more than
// its lower neighbours'), the rows of a level in parallel.
struct NatDev {
  int n = 0, nlev = 0, nt = 0;   // rows, levels, upper columns per row (move1's nt)
  const int* lvl_off = nullptr;   // [nlev + 1]
  const int* lvl_row = nullptr;   // [n] rows (0-based) by ascending level
  const int* lrow = nullptr;      // [n] 1-based column index l of each row (= row + 1)
  const int4* nbr = nullptr;      // [n] W, S, N, E rows (n = none)
  const int* order = nullptr;     // [n] move1 column order, packed
  double *cd = nullptr, *cW = nullptr, *cS = nullptr, *cN = nullptr, *cE = nullptr;   // [n + 1]
  double *b = nullptr, *u = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
  double *piv = nullptr, *dinv = nullptr;
  PcgScal* sc = nullptr;
  double *hist_alpha = nullptr, *hist_beta = nullptr, *tri = nullptr;
};
// One open boundary with a specified water-surface elevation (k_openbc.cu).  side: 1 W, 2 N, 3 E,
// 4 S.  Per boundary cell (1-based column indices): the cell, its interior neighbour, the column
// whose sx (W, E) or sy (N, S) couples the two; per boundary row, the face column whose momentum
// the reference recomputes (`mom`, nface entries).
struct ObcDev {
  int side = 0, n = 0, nface = 0;
  const int* cells = nullptr;
  const int* inner = nullptr;
  const int* face = nullptr;
  const int* mom = nullptr;
};
void obc_set_s(const Dev& d, const ObcDev& B, double v, cudaStream_t st);
void obc_exmom(const Dev& d, const ObcDev& B, int ieq, cudaStream_t st);
void obc_qq(const Dev& d, const ObcDev& B, cudaStream_t st);
void obc_vel(const Dev& d, const ObcDev& B, cudaStream_t st);
void obc_sca(const Dev& d, const ObcDev& B, double salbc, cudaStream_t st);

// rows and x0 from matcon's sx, sy, qq (x0 modes as the red-black gather); the solve (one block);
// zeta back to the columns
void nat_setup(const Dev& d, const NatDev& N, int x0_mode, const double* dz, cudaStream_t st);
int nat_solve(const NatDev& N, bool test2, cudaStream_t st);
void nat_finish(const Dev& d, const NatDev& N, cudaStream_t st);
// `init` (host memory, optional) replaces the zeroed barrier record of this launch
// One basin's share of an ensemble's batched FP64 solve (k_pcg_loop_ens): its system, its own
// barrier record, and the blocks [first, first + nblk) of the launch that solve it.
struct PcgEnsItem {
  PcgDev P;
  GridBar* bar;
  int first, nblk;
};
int pcg_loop_ens_blocks(int device);   // co-resident blocks of the batched launch
// the batched launch over nitems basins (items and bars in device memory; bars zeroed first)
int pcg_loop_ens(const PcgEnsItem* items, int nitems, int nblocks, GridBar* bars, cudaStream_t st);
int pcg_loop(const PcgDev& P, GridBar* bar, int nblocks, bool test2, cudaStream_t st,
             const GridBar* init = nullptr);   // test2: stopping test 2
int pcg_loop_f(const PcgDevF& F, GridBar* bar, int nblocks, cudaStream_t st, const GridBar* init = nullptr);

void launch_slayer_h(const Dev& d, cudaStream_t st);
void launch_vel(const Dev& d, const int* ce, int nce, const int* cn, int ncn, cudaStream_t st);
void launch_exsal_imsal(const Dev& d, const Tune& tu, cudaStream_t st);
// Non-active tracers (k_tracer.cu): exTracer + ImTracer for ntr tracers at once.  Tracer nt
// (0-based) of a pool is the layer-major field at pool + nt * stride.  `cpp` holds tracerpp, `tr`
// receives tracer; layers without a solve keep the tracer pool's values, or tracerpp's when
// keep_pp (the two are then equal and the tracer pool is stale).  `fx` holds the face fluxes of
// the tracers of one flux group but the last tracer (3 min(ntr - 1, kTracerFluxGroup) fields of
// km1 x P); `scr` one km1 x P field per group of kTracerGroup tracers of the column solve.
constexpr int kTracerGroup = 8;
constexpr int kTracerFluxGroup = 4;
void launch_tracers(const Dev& d, const double* cpp, double* tr, bool keep_pp, int ntr, long long stride,
                    double* fx, double* scr, cudaStream_t st);
void launch_vel2(const Dev& d, cudaStream_t st);
void launch_settrap(const Dev& d, cudaStream_t st);
void launch_settrap2(const Dev& d, cudaStream_t st);
void launch_save(const Dev& d, int istep, cudaStream_t st);

void launch_density_init(const Dev& d, cudaStream_t st);

// Mellor-Yamada 2.5 (k_turb.cu): the closure at the end of fd (scr4: four km1 x P scratch fields),
// the half levels of settrap (mode 1) / settrap2 (mode 2), and save's time levels.
void launch_turbulence(const Dev& d, double* scr4, cudaStream_t st);
void launch_turb_half(const Dev& d, int mode, cudaStream_t st);
void launch_turb_save(const Dev& d, int istep, cudaStream_t st);

// Output frames (k_output.cu): nf fields (layer-major FP64) at every point k1..kmz(l) + 1 of every
// wet column, point offsets poff (lm + 1 entries), optionally preceded by the coordinates i, j, k,
// as 4-byte floats into `out`; and one horizontal plane's frame over its column list.
void launch_pack_points(const Dev& d, const double* const* fields, int nf, const int* poff, const int* l2i,
                        const int* l2j, bool coords, float* out, cudaStream_t st);
void launch_pack_plane(const Dev& d, const int* cols, int n, int kp, bool first, const int* l2i, const int* l2j,
                       float* out, cudaStream_t st);

void launch_column_tridiag(int n, int nsys, const double* a, const double* b, const double* c, const double* g,
                           const double* r, double* ag, double* ar, double* scratch, cudaStream_t st);

}  // namespace si3d
