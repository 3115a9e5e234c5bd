// Aggregation multigrid for the FP32 inner solves of iterative refinement (precision
// SI3D_MIXED_MG).
//
// The zeta matrix is a mass term plus a graph Laplacian over the wet cells of the (im1, jm1)
// grid: (A x)_l = m_l x_l + sum over the faces f of l of c_f (x_l - x_nbr).  Every level of the
// hierarchy stores that form as an image: cell (r, c) of a rows x cols level at
// (r + 1) * pitch + c + kMgColOff, with a zero frame (one ghost row before and two after, four
// ghost columns before and at least five after) so that stencils and 2 x 2 aggregates never test
// bounds.  The offset of four columns puts every group of four cells 4q .. 4q + 3 of a row on a
// 16-byte boundary (the level passes move them as one float4), and with it every aggregate pair of
// the coarser level on an 8-byte boundary; a pass over whole groups also touches frame and land
// cells, which hold zero in every array and stay zero.  Per cell: the mass, the face to the next
// column (fc) and to the next row (fr), the inverse diagonal, the right-hand side b and the
// iterate z.  Level 0 is the zeta system itself (row = i - 1, column = j - 1 of the wet column);
// level k + 1 aggregates 2 x 2 cells of level k: masses add, the faces that cross between two
// aggregates add and are scaled by one half (the scaled piecewise-constant coarse operator; the
// unscaled Galerkin product over-weights the Laplacian of smooth modes by about two).  Land and
// frame cells carry zero mass and faces and stay zero.
//
// The preconditioner is one symmetric V-cycle: red-black Gauss-Seidel (red then black) from a zero
// guess on the way down, the residual summed over each aggregate, the coarsest level swept red,
// black, red, and on the way up the coarse correction enters through the black
// half-sweep (black then red), so the cycle is a symmetric positive-definite operator and plain CG
// applies.
#pragma once
#include "kernels.h"

namespace si3d {

constexpr int kMgMaxLevels = 10;
constexpr int kMgCoarsest = 8192;   // cells of the coarsest level at most
// Levels at least: each level divides the face-to-mass ratio of the operator by four, and the
// coarsest level, swept once, must be mass-dominated; 4 coarsenings bring the ratio of the 50 m,
// 30 s, 60 m deep workloads (about 210 at the leapfrog solve) below one.
constexpr int kMgMinLevels = 5;

// x / d for 0 <= x < 2^31 as (x * m) >> p with p = 31 + ceil(log2 d), m = ceil(2^p / d).
struct FastDiv {
  unsigned long long m;
  int p, d;
};

constexpr int kMgColOff = 4;   // buffer column of interior column 0

struct MgLevel {
  int rows, cols, pitch, nq;   // nq = (cols + 3) / 4 groups of four cells per row
  FastDiv div_cols, div_q;
  float *z, *b, *fc, *fr, *mass, *dinv;
};

// Floats per row of a level with `cols` columns: the four leading ghost columns, nq whole groups,
// and at least five trailing ghost columns (the east neighbours of the last group and the
// aggregate pairs the coarser level reads), rounded up to 32 floats.
inline int mg_pitch(int cols) { return ((4 * ((cols + 3) / 4) + kMgColOff + 5 + 31) / 32) * 32; }

constexpr int kMgMaxOuter = 40;      // FP64 refinement passes at most (then ier = 1)

struct MgDev {
  int nlev = 0;
  MgLevel lv[kMgMaxLevels];
  // level-0 FP32 CG vectors of the inner solve (e = u; lv[0].b is its residual)
  float *u = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr;
  // the FP64 system on the level-0 image: solution, right-hand side, faces and diagonal
  double *u64 = nullptr, *b64 = nullptr, *fc64 = nullptr, *fr64 = nullptr, *dg64 = nullptr;
  const int* pixL = nullptr;   // wet column l -> level-0 offset (index l - 1)
  // block partials: (r, r) [nb], (r, z) black + red [2 nb], (p, q) [nb], FP64 (r, r) and (b, b) [2 nb]
  double* part = nullptr;
  // in: zeta (outer tolerance), srelpr, itmax (inner); out: in (inner iterations, all passes),
  // stptst (outer), bnorm, ier, q1 (outer passes), done
  PcgScal* sc = nullptr;
};

FastDiv fast_div(int d);
size_t mg_level_elems(int rows, int cols);   // floats of one array of a rows x cols level
int mg_loop_blocks(int device, int cells0, int max_per_sm);
// the FP64 system, level 0 and the coarser levels from matcon's sx, sy, qq and the initial guess
void mg_setup(const Dev& d, const MgDev& M, int x0_mode, const double* dz, const double* hist, cudaStream_t st);
int mg_solve(const MgDev& M, GridBar* bar, int nblocks, cudaStream_t st, const GridBar* init = nullptr);     // the cooperative solve
void mg_finish(const Dev& d, const MgDev& M, double* hist, cudaStream_t st);  // s(l) = u (and hist)

}  // namespace si3d
