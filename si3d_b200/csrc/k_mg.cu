// Mixed-precision zeta solve with aggregation-multigrid preconditioned FP32 inner solves (hierarchy
// and V-cycle: mg.h), the whole solve in one cooperative launch: FP64 iterative refinement around
// FP32 MG-PCG.  Phases are separated by grid barriers (coop.cuh) and every block reduces the block
// partials itself in the same fixed order, so all blocks take the same decisions.
//
// Outer (FP64) pass: u += e (from the second pass on; e is the FP32 correction), then the residual
// r = b - A u and ||r|| (and ||b|| on the first pass); stop when ||r|| < ||b|| zeta (test 5);
// otherwise the inner solve starts from e = 0 with right-hand side r rounded to FP32 and stops when
// its residual has dropped by max(1e-5, what the outer test still needs).
//
// Inner (FP32 MG-PCG) iteration (a barrier after each phase):
//   U       e += alpha p, r -= alpha q (from the second iteration on), (r, r), and the first
//           (red) half-sweep of level 0 from z = 0, which is z = dinv r;
//           the stopping test on the inner residual right after its barrier
//   down    per level k < L - 1: black half-sweep; residual summed over 2 x 2 aggregates into
//           level k + 1's b, whose red cells get their first half-sweep z = dinv b.  On levels
//           >= 2 the black half-sweep is not run as a phase: the restriction forms the black
//           values it reads from their red neighbours (the same expression)
//   coarse  black half-sweep of the coarsest level
//   up      per level k = L - 2 .. 0: black half-sweep with the neighbours' values plus the coarse
//           correction of their aggregate; red half-sweep; at level 0 both add to (r, z).  The
//           red half-sweeps of the coarsest level and of levels >= 2 are not run as phases: the
//           black half-sweep of the next finer level forms each red aggregate it reads from that
//           aggregate's black neighbours (the same expression, so the same values)
//   PQ      beta, p = z + beta p and q = A p (neighbours' p formed on the fly), (p, q)
// With L >= 3 levels that is 2 L + 5 barriers an inner iteration (15 for the five levels of the
// 2000 x 1000 system, where a V-cycle with every half-sweep a phase has 19).
//
// Every level pass walks groups of four consecutive cells of a row (one float4 of each array,
// 16-byte aligned by the image layout, mg.h): a thread keeps several groups' loads in flight with a
// quarter of the load instructions and index arithmetic of a cell-by-cell pass.  Frame and land
// cells inside a group hold zero in every array and compute zero, so no cell is tested.
#include <algorithm>

#include "../../include/si3d_gpu.h"
#include "common.cuh"
#include "coop.cuh"
#include "mg.h"

namespace si3d {

FastDiv fast_div(int d) {
  FastDiv f{};
  int s = 0;
  while ((1LL << s) < (long long)d) ++s;
  f.p = 31 + s;
  f.m = ((1ULL << f.p) + (unsigned long long)d - 1ULL) / (unsigned long long)d;
  f.d = d;
  return f;
}

size_t mg_level_elems(int rows, int cols) { return (size_t)(rows + 3) * (size_t)mg_pitch(cols); }

namespace {

using namespace coop;

constexpr int PB = 256;               // threads per block of the setup kernels
constexpr float kFaceScale = 0.5f;    // coarse faces: half the sum of the crossing fine faces
constexpr int CO = kMgColOff;
constexpr int UG = 2;                 // groups of four cells a thread keeps in flight in the level-0 CG passes
constexpr int UH = 2;                 // groups in flight in the half-sweeps
// Levels from kSweptFrom on (and the coarsest) skip their red half-sweep of the way up: the finer
// level's black half-sweep forms the red values it reads from their black neighbours (swept_z).
// Cheap on the small levels, it saves a grid barrier a level; on levels 0 and 1 the recomputation
// costs more than the barrier.
constexpr int kSweptFrom = 2;
constexpr int kSpreadFrom = 2;   // levels whose items are dealt round robin (first_item_spread)
constexpr int MQ = 512;               // threads per block of the cooperative solve (one block per SM)

__device__ __forceinline__ int fdiv(const FastDiv& f, int x) {
  return (int)(((unsigned long long)(unsigned int)x * f.m) >> f.p);
}

// ---------------------------------------------------------------- per-solve setup
// Level 0 and the FP64 system from the assembled zeta system of wet column l (matcon's sx, sy, qq):
// the faces the system couples, the diagonal it applies (1 + sx + sx(W) + sy + sy(S), as the red-black
// system does), mass = diagonal - faces, and the initial guess (x0 modes of the red-black gather).
__global__ void k_mg_setup(Dev d, MgDev M, int x0_mode, const double* __restrict__ dz,
                           const double* __restrict__ hist) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int lm1 = d.g.lm1;
  const int o = M.pixL[l - 1];
  const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
  const double sxi = d.s.sx[l - 1], syi = d.s.sy[l - 1];
  const double sxW = (lW != lm1) ? d.s.sx[lW - 1] : 0.0;
  const double syS = (lS != lm1) ? d.s.sy[lS - 1] : 0.0;
  const double diag = d.s.rr[l - 1];   // matcon's 1 + sx + sx(W) + sy + sy(S), before any face cut
  const double fN = (lN != lm1) ? syi : 0.0;   // face to (i, j + 1): the next column
  const double fE = (lE != lm1) ? sxi : 0.0;   // face to (i + 1, j): the next row
  M.fc64[o] = fN;
  M.fr64[o] = fE;
  M.dg64[o] = diag;
  M.b64[o] = d.s.qq[l - 1];
  double x0;
  switch (x0_mode) {
    case 1: x0 = 0.0; break;
    case 3: x0 = d.s.s[l - 1]; break;
    case 4: x0 = d.s.s[l - 1] + (hist ? hist[l - 1] : 0.0); break;
    default: x0 = d.s.sp[l - 1]; if (x0_mode == 2 && dz) x0 = x0 + dz[l - 1];
  }
  M.u64[o] = x0;
  const MgLevel& L = M.lv[0];
  L.fc[o] = (float)fN;
  L.fr[o] = (float)fE;
  L.mass[o] = (float)(diag - fN - fE - sxW - syS);
  L.dinv[o] = (float)(1.0 / diag);
}

// zeta back to the columns: s(l) = u; with `hist`, also this solve's correction to the zeta it
// started from (s before the write), per column, for the next step's guess of the same solve.
__global__ void k_mg_scatter(Dev d, MgDev M, double* __restrict__ hist) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const double u = M.u64[M.pixL[l - 1]];
  if (hist) hist[l - 1] = u - d.s.s[l - 1];
  d.s.s[l - 1] = u;
}

// Level k + 1 from level k: 2 x 2 aggregates (frame cells read as zero).
__global__ void k_mg_coarsen(MgLevel F, MgLevel G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= G.rows * G.cols) return;
  const int R = t / G.cols, Cc = t - R * G.cols;
  const int fp = F.pitch;
  const int o00 = (2 * R + 1) * fp + 2 * Cc + CO, o01 = o00 + 1, o10 = o00 + fp, o11 = o10 + 1;
  const float mass = (F.mass[o00] + F.mass[o01]) + (F.mass[o10] + F.mass[o11]);
  const float fc = kFaceScale * (F.fc[o01] + F.fc[o11]);
  const float fr = kFaceScale * (F.fr[o10] + F.fr[o11]);
  const float fcW = kFaceScale * (F.fc[o00 - 1] + F.fc[o10 - 1]);
  const float frS = kFaceScale * (F.fr[o00 - fp] + F.fr[o01 - fp]);
  const int O = (R + 1) * G.pitch + Cc + CO;
  G.fc[O] = fc;
  G.fr[O] = fr;
  G.mass[O] = mass;
  const float diag = mass + fc + fr + fcW + frS;
  G.dinv[O] = diag > 0.f ? 1.f / diag : 0.f;
}

// ---------------------------------------------------------------- V-cycle pieces
__device__ __forceinline__ float4 ld4(const float* p, int o) { return *reinterpret_cast<const float4*>(p + o); }
__device__ __forceinline__ float2 ld2(const float* p, int o) { return *reinterpret_cast<const float2*>(p + o); }
__device__ __forceinline__ void st4(float* p, int o, float4 v) { *reinterpret_cast<float4*>(p + o) = v; }
__device__ __forceinline__ void st2(float* p, int o, float2 v) { *reinterpret_cast<float2*>(p + o) = v; }
__device__ __forceinline__ float sel(int j, float a0, float a1) { return j ? a1 : a0; }

// Group t of a level: row r, group q, buffer offset of its first cell (column 4q).
__device__ __forceinline__ int group_at(const MgLevel& L, int t, int& r, int& q) {
  r = fdiv(L.div_q, t);
  q = t - r * L.nq;
  return (r + 1) * L.pitch + 4 * q + CO;
}

// Gauss-Seidel value of cell (R, C) of level G from its neighbours' current z, dinv (b + sum of
// face * neighbour z), in the half-sweep's operation order.  Every load is unconditional (the rows
// are clamped into the frame), so a thread issues all of them at once; frame and land cells
// (dinv = b = faces = 0) give zero.  R in [-1, rows + 1], C in [-1, 4 nq + 3].
__device__ __forceinline__ float gs_value(const MgLevel& G, int R, int C) {
  const int gp = G.pitch, o = (R + 1) * gp + C + CO;
  const int oS = (max(R - 1, -1) + 1) * gp + C + CO, oN = (min(R + 1, G.rows + 1) + 1) * gp + C + CO;
  const float s1 = G.b[o] + G.fc[o] * G.z[o + 1] + G.fc[o - 1] * G.z[o - 1] + G.fr[o] * G.z[oN] + G.fr[oS] * G.z[oS];
  return G.dinv[o] * s1;
}

// z of cell (R, C) of level G as it stands after G's red half-sweep of the way up, when that sweep
// was not run: red cells are formed from their black neighbours exactly as the sweep would form
// them; black cells are read.
__device__ __forceinline__ float swept_z(const MgLevel& G, int R, int C) {
  const float v = gs_value(G, R, C), z = G.z[(R + 1) * G.pitch + C + CO];
  return ((R + C) & 1) == 0 ? v : z;
}

// Gauss-Seidel half-sweep over the cells of colour `col` ((r + c) & 1 == col) of level L:
// z = dinv (b + sum of face * neighbour z).  PROLONG: each neighbour's value is its z plus the
// correction of its aggregate in the coarser level G; with SWEPT, G's red half-sweep was not run and
// the red aggregates are formed on the fly (swept_z).  DOT: returns this thread's sum of b * z.
// A group of four cells of row r holds two cells of the colour, at j0 = (r + col) & 1 and j0 + 2.
template <bool PROLONG, bool DOT, int U, bool SWEPT = false>
__device__ __forceinline__ double half_sweep(const MgLevel& L, const MgLevel& G, int col, int g0, int stride) {
  double rz = 0.0;
  const int n = L.rows * L.nq, pt = L.pitch;
  for (int t0 = g0; t0 < n; t0 += U * stride) {
    int x[U], jc[U];
    bool ok[U];
    float zv[U][2], bq[U][2];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int t = t0 + k * stride;
      ok[k] = t < n;
      int r = 0, q = 0;
      x[k] = ok[k] ? group_at(L, t, r, q) : pt + CO;   // an interior group, loaded and dropped
      const int j = (r + col) & 1;
      jc[k] = j;
      const int o = x[k];
      const float4 zm = ld4(L.z, o), zs = ld4(L.z, o - pt), zn = ld4(L.z, o + pt);
      const float zw0 = L.z[o - 1], ze3 = L.z[o + 4];
      const float4 bb = ld4(L.b, o), dv = ld4(L.dinv, o), fc = ld4(L.fc, o), fr = ld4(L.fr, o), fs = ld4(L.fr, o - pt);
      const float fw0 = L.fc[o - 1];
      // the two cells of the colour: column jj = j (m = 0) and j + 2 (m = 1)
      // row values at columns -1 .. 4 of the group
      const float zr[6] = {zw0, zm.x, zm.y, zm.z, zm.w, ze3};
      const float fcr[5] = {fw0, fc.x, fc.y, fc.z, fc.w};   // fcr[c + 1] = face from column c to c + 1
      const float zsv[4] = {zs.x, zs.y, zs.z, zs.w}, znv[4] = {zn.x, zn.y, zn.z, zn.w};
      const float bv[4] = {bb.x, bb.y, bb.z, bb.w}, dvv[4] = {dv.x, dv.y, dv.z, dv.w};
      const float frn[4] = {fr.x, fr.y, fr.z, fr.w}, frs[4] = {fs.x, fs.y, fs.z, fs.w};
      float gW[2] = {0.f, 0.f}, gE[2] = {0.f, 0.f}, gS[2] = {0.f, 0.f}, gN[2] = {0.f, 0.f};
      if (PROLONG) {
        // aggregates of the neighbours: row r >> 1 at coarse columns 2q - 1 .. 2q + 2, rows
        // (r - 1) >> 1 and (r + 1) >> 1 at 2q, 2q + 1
        float gc[4];   // coarse columns 2q - 1 .. 2q + 2 of row r >> 1
        float2 gs, gn;
        if (SWEPT) {
          // rows (r - 1) >> 1 and (r + 1) >> 1: one of them is row r >> 1 itself
          const int g1 = r >> 1, go = (r & 1) ? g1 + 1 : g1 - 1;
#pragma unroll
          for (int i = 0; i < 4; ++i) gc[i] = swept_z(G, g1, 2 * q - 1 + i);
          const float2 gm = make_float2(gc[1], gc[2]);
          const float2 gx = make_float2(swept_z(G, go, 2 * q), swept_z(G, go, 2 * q + 1));
          gs = (r & 1) ? gm : gx;
          gn = (r & 1) ? gx : gm;
        } else {
          const int gp = G.pitch;
          const int gr = ((r >> 1) + 1) * gp + 2 * q + CO;
          const float2 gm = ld2(G.z, gr);
          gc[0] = G.z[gr - 1]; gc[1] = gm.x; gc[2] = gm.y; gc[3] = G.z[gr + 2];
          gs = ld2(G.z, (((r - 1) >> 1) + 1) * gp + 2 * q + CO);
          gn = ld2(G.z, (((r + 1) >> 1) + 1) * gp + 2 * q + CO);
        }
        // cell jj = 2m + j: west neighbour's aggregate gc[((jj - 1) >> 1) + 1], east gc[((jj + 1) >> 1) + 1],
        // south / north (jj >> 1) = m
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          gW[m] = sel(j, gc[m], gc[m + 1]);          // jj = 2m: column m ; jj = 2m + 1: column m + 1
          gE[m] = sel(j, gc[m + 1], gc[m + 2]);
          gS[m] = m ? gs.y : gs.x;
          gN[m] = m ? gn.y : gn.x;
        }
      }
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        // column jj = 2m + j, selected between the even (j = 0) and odd (j = 1) candidates
        float zw = sel(j, zr[2 * m], zr[2 * m + 1]);
        float ze = sel(j, zr[2 * m + 2], zr[2 * m + 3]);
        float zs1 = sel(j, zsv[2 * m], zsv[2 * m + 1]);
        float zn1 = sel(j, znv[2 * m], znv[2 * m + 1]);
        if (PROLONG) { zw += gW[m]; ze += gE[m]; zs1 += gS[m]; zn1 += gN[m]; }
        const float b1 = sel(j, bv[2 * m], bv[2 * m + 1]);
        const float fce = sel(j, fcr[2 * m + 1], fcr[2 * m + 2]), fcw = sel(j, fcr[2 * m], fcr[2 * m + 1]);
        const float fn = sel(j, frn[2 * m], frn[2 * m + 1]), fsv = sel(j, frs[2 * m], frs[2 * m + 1]);
        const float s1 = b1 + fce * ze + fcw * zw + fn * zn1 + fsv * zs1;
        zv[k][m] = sel(j, dvv[2 * m], dvv[2 * m + 1]) * s1;
        bq[k][m] = b1;
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      if (!ok[k]) continue;
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        L.z[x[k] + 2 * m + jc[k]] = zv[k][m];
        if (DOT) rz += (double)bq[k][m] * (double)zv[k][m];
      }
    }
  }
  return rz;
}

// b of level G = the residual b - A z of level F summed over each 2 x 2 aggregate; z of G = dinv b,
// which is the first half-sweep from zero for its red cells (its black cells are swept before
// they are read).  An item is one group of four columns in the two fine rows of a coarse row: the
// coarse pair 2q, 2q + 1.  BLK: F's black half-sweep of the way down was not run; the black values
// the residuals read (ten of the twenty in the item's window) are formed here from their red
// neighbours, as that half-sweep forms them (gs_value).
template <bool BLK>
__device__ __forceinline__ void restrict_residual(const MgLevel& F, const MgLevel& G, int g0, int stride) {
  const int n = G.rows * F.nq, fp = F.pitch;
  for (int t = g0; t < n; t += stride) {
    const int R = fdiv(F.div_q, t);
    const int q = t - R * F.nq;
    const int x0 = (2 * R + 1) * fp + 4 * q + CO, x1 = x0 + fp;
    // z on fine rows 2R - 1 .. 2R + 2 (i) and columns 4q - 1 .. 4q + 4 (j); cell (i, j) is black when
    // i + j is odd
    float zw[4][6];
    {
      const float4 zA = ld4(F.z, x0 - fp), z0 = ld4(F.z, x0), z1 = ld4(F.z, x1), zB = ld4(F.z, x1 + fp);
      const float z0w = F.z[x0 - 1], z0e = F.z[x0 + 4], z1w = F.z[x1 - 1], z1e = F.z[x1 + 4];
      const float win[4][6] = {{0.f, zA.x, zA.y, zA.z, zA.w, 0.f},
                               {z0w, z0.x, z0.y, z0.z, z0.w, z0e},
                               {z1w, z1.x, z1.y, z1.z, z1.w, z1e},
                               {0.f, zB.x, zB.y, zB.z, zB.w, 0.f}};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const bool used = (i == 1 || i == 2) || (j >= 1 && j <= 4);
          zw[i][j] = (BLK && used && ((i + j) & 1)) ? gs_value(F, 2 * R - 1 + i, 4 * q - 1 + j) : win[i][j];
        }
      }
    }
    const float4 b0 = ld4(F.b, x0), b1 = ld4(F.b, x1), m0 = ld4(F.mass, x0), m1 = ld4(F.mass, x1);
    const float4 c0 = ld4(F.fc, x0), c1 = ld4(F.fc, x1);
    const float c0w = F.fc[x0 - 1], c1w = F.fc[x1 - 1];
    const float4 rA = ld4(F.fr, x0 - fp), r0 = ld4(F.fr, x0), r1 = ld4(F.fr, x1);
    const int O = (R + 1) * G.pitch + 2 * q + CO;
    const float2 dg = ld2(G.dinv, O);
    float res[2][4];
    {
      const float bv[2][4] = {{b0.x, b0.y, b0.z, b0.w}, {b1.x, b1.y, b1.z, b1.w}};
      const float mv[2][4] = {{m0.x, m0.y, m0.z, m0.w}, {m1.x, m1.y, m1.z, m1.w}};
      const float fcr[2][5] = {{c0w, c0.x, c0.y, c0.z, c0.w}, {c1w, c1.x, c1.y, c1.z, c1.w}};
      const float frs[2][4] = {{rA.x, rA.y, rA.z, rA.w}, {r0.x, r0.y, r0.z, r0.w}};
      const float frn[2][4] = {{r0.x, r0.y, r0.z, r0.w}, {r1.x, r1.y, r1.z, r1.w}};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const float fcw = fcr[h][jj], fce = fcr[h][jj + 1], fs = frs[h][jj], fn = frn[h][jj];
          const float diag = mv[h][jj] + fcw + fce + fs + fn;
          const float az = diag * zw[h + 1][jj + 1] - fce * zw[h + 1][jj + 2] - fcw * zw[h + 1][jj] -
                           fn * zw[h + 2][jj + 1] - fs * zw[h][jj + 1];
          res[h][jj] = bv[h][jj] - az;
        }
      }
    }
    // aggregate (R, 2q + a): fine cells (2R, 2a), (2R, 2a + 1), (2R + 1, 2a), (2R + 1, 2a + 1), in that order
    float acc[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      float s1 = 0.f;
      s1 += res[0][2 * a];
      s1 += res[0][2 * a + 1];
      s1 += res[1][2 * a];
      s1 += res[1][2 * a + 1];
      acc[a] = s1;
    }
    st2(G.b, O, make_float2(acc[0], acc[1]));
    st2(G.z, O, make_float2(dg.x * acc[0], dg.y * acc[1]));
  }
}

// ---------------------------------------------------------------- the inner solve
// FP32 MG-PCG on level 0 from e = 0 (M.u) with right-hand side r (level 0's b), until
// ||r|| < bnorm * zeta or itmax iterations.  Returns false when a barrier gave up (the caller returns
// at once); otherwise its = the iterations taken and ier = 0, 1 (itmax) or -6 / -7 (breakdown).
// A thread's first item of a level pass.  On levels 0 and 1 a block takes MQ consecutive items
// (b * MQ + thread, then + blocks * MQ), which keeps its accesses in few DRAM pages.  On the coarser
// levels (a few thousand items) the items are dealt to the blocks in runs of 32 (one warp's worth,
// so a warp's accesses stay coalesced), round robin, so that they spread over every SM instead of
// filling the first blocks: thread (warp w, lane i) of block b takes (w * blocks + b) * 32 + i.
__device__ __forceinline__ int first_item_dense() { return (int)blockIdx.x * MQ + (int)threadIdx.x; }
__device__ __forceinline__ int first_item_spread() {
  return ((int)(threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) * 32 + (int)(threadIdx.x & 31);
}

__device__ bool mg_pcg(const MgDev& M, const MgLevel* s_lv, int nlev, GridBar* bar, PcgScal* SC, BarSt* s_flag,
                       double* sh, double zeta, double bnorm, int itmax, int& its, int& ier) {
  const int nb = gridDim.x, stride = nb * MQ, g0 = first_item_dense(), g0s = first_item_spread();
  auto gk = [&](int k) { return k < kSpreadFrom ? g0 : g0s; };
  double* const rr_part = M.part;
  double* const rz_part = M.part + nb;
  double* const pq_part = M.part + 3 * nb;
  double alpha = 0.0, beta = 0.0, rz_old = 1.0;
  int it = 0;
  ier = 0;
  const MgLevel& L0 = s_lv[0];
  const int n0q = L0.rows * L0.nq, pt = L0.pitch;
  for (;;) {
    // ---- U: u += alpha p, r -= alpha q; (r, r); z = dinv r, the red half-sweep of level 0 from zero
    // (written for the black cells too: the black half-sweep replaces them before they are read)
    {
      const float a = (float)alpha;
      const float* __restrict__ pn = (it & 1) ? M.p1 : M.p0;
      double rr = 0.0;
      for (int t0 = g0; t0 < n0q; t0 += UG * stride) {
        int o[UG];
        bool ok[UG];
        float4 rv[UG], zv[UG], uv[UG];
#pragma unroll
        for (int k = 0; k < UG; ++k) {
          const int t = t0 + k * stride;
          ok[k] = t < n0q;
          int r = 0, q = 0;
          o[k] = ok[k] ? group_at(L0, t, r, q) : pt + CO;
          rv[k] = ld4(L0.b, o[k]);
          const float4 dv = ld4(L0.dinv, o[k]);
          if (it > 0) {
            const float4 u4 = ld4(M.u, o[k]), p4 = ld4(pn, o[k]), q4 = ld4(M.q, o[k]);
            uv[k] = make_float4(u4.x + a * p4.x, u4.y + a * p4.y, u4.z + a * p4.z, u4.w + a * p4.w);
            rv[k] = make_float4(rv[k].x - a * q4.x, rv[k].y - a * q4.y, rv[k].z - a * q4.z, rv[k].w - a * q4.w);
          }
          zv[k] = make_float4(dv.x * rv[k].x, dv.y * rv[k].y, dv.z * rv[k].z, dv.w * rv[k].w);
        }
#pragma unroll
        for (int k = 0; k < UG; ++k) {
          if (!ok[k]) continue;
          if (it > 0) {
            st4(M.u, o[k], uv[k]);
            st4(L0.b, o[k], rv[k]);
          }
          st4(L0.z, o[k], zv[k]);
          rr += (double)rv[k].x * (double)rv[k].x;
          rr += (double)rv[k].y * (double)rv[k].y;
          rr += (double)rv[k].z * (double)rv[k].z;
          rr += (double)rv[k].w * (double)rv[k].w;
        }
      }
      double w[1] = {rr};
      bsum<1, MQ>(w, sh);
      if (threadIdx.x == 0) rr_part[blockIdx.x] = w[0];
    }
    if (!grid_barrier(bar, SC, s_flag)) return false;
    {
      double w[1];
      all_partials<1, MQ>(rr_part, nb, 0, w, sh);
      const double tl = sqrt(w[0]);
      if (tl < bnorm * zeta) break;
      if (it >= itmax) { ier = 1; break; }
    }
    // ---- down: black half-sweep, restriction (on levels >= kSweptFrom the restriction forms the
    // black values it reads, and the black half-sweep is not run as a phase)
    for (int k = 0; k < nlev - 1; ++k) {
      if (k >= kSweptFrom) {
        restrict_residual<true>(s_lv[k], s_lv[k + 1], gk(k), stride);
      } else {
        half_sweep<false, false, UH>(s_lv[k], s_lv[k], 1, gk(k), stride);
        if (!grid_barrier(bar, SC, s_flag)) return false;
        restrict_residual<false>(s_lv[k], s_lv[k + 1], gk(k), stride);
      }
      if (!grid_barrier(bar, SC, s_flag)) return false;
    }
    // ---- coarsest level: black half-sweep (its red half-sweep is formed where it is read)
    half_sweep<false, false, UH>(s_lv[nlev - 1], s_lv[nlev - 1], 1, gk(nlev - 1), stride);
    if (!grid_barrier(bar, SC, s_flag)) return false;
    // ---- up: black half-sweep with the coarse correction, red half-sweep; (r, z) at level 0.  The
    // red half-sweeps of levels >= kSweptFrom (and of the coarsest) are not run: the black half-sweep
    // of the next finer level forms the red aggregates it reads (swept_z), one barrier fewer each.
    for (int k = nlev - 2; k >= 0; --k) {
      const bool swept = k + 1 >= kSweptFrom || k + 1 == nlev - 1;
      if (k == 0) {
        double w[1] = {swept ? half_sweep<true, true, 1, true>(s_lv[0], s_lv[1], 1, g0, stride)
                             : half_sweep<true, true, UH>(s_lv[0], s_lv[1], 1, g0, stride)};
        bsum<1, MQ>(w, sh);
        if (threadIdx.x == 0) rz_part[blockIdx.x] = w[0];
      } else if (swept) {
        half_sweep<true, false, 1, true>(s_lv[k], s_lv[k + 1], 1, gk(k), stride);
      } else {
        half_sweep<true, false, UH>(s_lv[k], s_lv[k + 1], 1, gk(k), stride);
      }
      if (!grid_barrier(bar, SC, s_flag)) return false;
      if (k >= kSweptFrom) continue;
      if (k == 0) {
        double w[1] = {half_sweep<false, true, UH>(s_lv[0], s_lv[0], 0, g0, stride)};
        bsum<1, MQ>(w, sh);
        if (threadIdx.x == 0) rz_part[nb + blockIdx.x] = w[0];
      } else {
        half_sweep<false, false, UH>(s_lv[k], s_lv[k], 0, gk(k), stride);
      }
      if (!grid_barrier(bar, SC, s_flag)) return false;
    }
    {
      double w[1];
      all_partials<1, MQ>(rz_part, 2 * nb, 0, w, sh);
      if (!(w[0] > 0.0)) { ier = -7; break; }
      beta = (it == 0) ? 0.0 : w[0] / rz_old;
      rz_old = w[0];
    }
    // ---- PQ: p = z + beta p, q = A p, (p, q)
    {
      const float bt = (float)beta;
      const bool first = it == 0;
      const float* __restrict__ po = (it & 1) ? M.p1 : M.p0;
      float* __restrict__ pw = (it & 1) ? M.p0 : M.p1;
      double pq = 0.0;
      for (int t0 = g0; t0 < n0q; t0 += UG * stride) {
        int o[UG];
        bool ok[UG];
        float4 pc[UG], qv[UG];
#pragma unroll
        for (int k = 0; k < UG; ++k) {
          const int t = t0 + k * stride;
          ok[k] = t < n0q;
          int r = 0, q = 0;
          const int x = ok[k] ? group_at(L0, t, r, q) : pt + CO;
          o[k] = x;
          // p at columns -1 .. 4 of the row and at the four cells of the rows south and north
          float4 zm = ld4(L0.z, x), zs = ld4(L0.z, x - pt), zn = ld4(L0.z, x + pt);
          float zw = L0.z[x - 1], ze = L0.z[x + 4];
          if (!first) {
            const float4 om = ld4(po, x), os = ld4(po, x - pt), on = ld4(po, x + pt);
            const float ow = po[x - 1], oe = po[x + 4];
            zm = make_float4(zm.x + bt * om.x, zm.y + bt * om.y, zm.z + bt * om.z, zm.w + bt * om.w);
            zs = make_float4(zs.x + bt * os.x, zs.y + bt * os.y, zs.z + bt * os.z, zs.w + bt * os.w);
            zn = make_float4(zn.x + bt * on.x, zn.y + bt * on.y, zn.z + bt * on.z, zn.w + bt * on.w);
            zw = zw + bt * ow;
            ze = ze + bt * oe;
          }
          const float4 fc = ld4(L0.fc, x), fr = ld4(L0.fr, x), fs = ld4(L0.fr, x - pt), ms = ld4(L0.mass, x);
          const float fw0 = L0.fc[x - 1];
          const float pr[6] = {zw, zm.x, zm.y, zm.z, zm.w, ze};
          const float ps[4] = {zs.x, zs.y, zs.z, zs.w}, pn4[4] = {zn.x, zn.y, zn.z, zn.w};
          const float fcr[5] = {fw0, fc.x, fc.y, fc.z, fc.w};
          const float frn[4] = {fr.x, fr.y, fr.z, fr.w}, frs[4] = {fs.x, fs.y, fs.z, fs.w};
          const float mv[4] = {ms.x, ms.y, ms.z, ms.w};
          float qq[4];
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const float fcw = fcr[jj], fce = fcr[jj + 1];
            const float diag = mv[jj] + fcw + fce + frs[jj] + frn[jj];
            qq[jj] = diag * pr[jj + 1] - fce * pr[jj + 2] - fcw * pr[jj] - frn[jj] * pn4[jj] - frs[jj] * ps[jj];
          }
          pc[k] = zm;
          qv[k] = make_float4(qq[0], qq[1], qq[2], qq[3]);
        }
#pragma unroll
        for (int k = 0; k < UG; ++k) {
          if (!ok[k]) continue;
          st4(pw, o[k], pc[k]);
          st4(M.q, o[k], qv[k]);
          pq += (double)pc[k].x * (double)qv[k].x;
          pq += (double)pc[k].y * (double)qv[k].y;
          pq += (double)pc[k].z * (double)qv[k].z;
          pq += (double)pc[k].w * (double)qv[k].w;
        }
      }
      double w[1] = {pq};
      bsum<1, MQ>(w, sh);
      if (threadIdx.x == 0) pq_part[blockIdx.x] = w[0];
    }
    if (!grid_barrier(bar, SC, s_flag)) return false;
    {
      double w[1];
      all_partials<1, MQ>(pq_part, nb, 0, w, sh);
      if (!(w[0] > 0.0)) { ier = -6; break; }
      alpha = rz_old / w[0];
    }
    ++it;
  }
  its = it;
  return true;
}

// ---------------------------------------------------------------- the whole solve
__global__ void __launch_bounds__(MQ, 1) k_mg_solve(MgDev M, GridBar* bar) {
  __shared__ double sh[(MQ / 32) * 2 + 2];
  __shared__ BarSt s_flag;
  __shared__ MgLevel s_lv[kMgMaxLevels];
  if (threadIdx.x == 0) s_flag.epoch = 0;
  const int nlev = M.nlev;
  if (threadIdx.x < nlev) s_lv[threadIdx.x] = M.lv[threadIdx.x];
  __syncthreads();
  PcgScal* SC = M.sc;
  const int nb = gridDim.x, stride = nb * MQ, g0 = first_item_dense();
  double* const res_part = M.part + 4 * nb;   // (r, r) [nb], (b, b) [nb] of the FP64 system
  const double zeta = SC->zeta, srelpr = SC->srelpr;
  const int itmax = SC->itmax;
  const MgLevel& L0 = s_lv[0];
  const int n0 = L0.rows * L0.cols, pt = L0.pitch;
  double bn = 1.0, stp = 1.0;
  int outer = 0, total = 0, ier = 0;
  for (;;) {
    if (outer > 0) {
      // ---- u += e (FP64)
      for (int t = g0; t < n0; t += stride) {
        const int r = fdiv(L0.div_cols, t), c = t - r * L0.cols;
        const int o = (r + 1) * pt + c + CO;
        M.u64[o] = M.u64[o] + (double)M.u[o];
      }
      if (!grid_barrier(bar, SC, &s_flag)) return;
    }
    // ---- r = b - A u (FP64), ||r||^2 (and ||b||^2 on the first pass); inner rhs r and e = 0
    {
      double v[2] = {0.0, 0.0};
      for (int t0 = g0; t0 < n0; t0 += 2 * stride) {
        int o[2];
        bool ok[2];
        double rv[2], bv[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int t = t0 + k * stride;
          ok[k] = t < n0;
          const int r = ok[k] ? fdiv(L0.div_cols, t) : 0;
          const int c = ok[k] ? t - r * L0.cols : 0;
          const int x = (r + 1) * pt + c + CO;
          o[k] = x;
          double y = M.dg64[x] * M.u64[x];
          y = y + (-M.fr64[x - pt]) * M.u64[x - pt];
          y = y + (-M.fc64[x - 1]) * M.u64[x - 1];
          y = y + (-M.fc64[x]) * M.u64[x + 1];
          y = y + (-M.fr64[x]) * M.u64[x + pt];
          bv[k] = M.b64[x];
          rv[k] = bv[k] - y;
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          if (!ok[k]) continue;
          v[0] += rv[k] * rv[k];
          v[1] += bv[k] * bv[k];
          L0.b[o[k]] = (float)rv[k];
          M.u[o[k]] = 0.f;
        }
      }
      bsum<2, MQ>(v, sh);
      if (threadIdx.x == 0) { res_part[blockIdx.x] = v[0]; res_part[nb + blockIdx.x] = v[1]; }
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
    double w[2];
    all_partials<2, MQ>(res_part, nb, nb, w, sh);
    if (outer == 0) bn = fmax(sqrt(w[1]), srelpr);   // bnorm of stopping test 5 (nmcalc)
    const double rn = sqrt(w[0]);
    stp = rn / bn;
    if (rn < bn * zeta) break;
    if (outer >= kMgMaxOuter) { ier = 1; break; }
    // ---- inner FP32 MG-PCG
    int its = 0, iier = 0;
    if (!mg_pcg(M, s_lv, nlev, bar, SC, &s_flag, sh, fmax(1e-5, 0.5 * zeta * bn / rn), rn, itmax, its, iier)) return;
    total += its;
    ++outer;
    if (iier < 0) { ier = iier; break; }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SC->in = total;
    SC->stptst = stp;
    SC->bnorm = bn;
    SC->ier = ier;
    SC->q1 = outer;
    SC->done = 1;
  }
}

}  // namespace

int mg_loop_blocks(int device, int cells0, int max_per_sm) {
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_solve, MQ, 0);
  int per_sm = std::max(occ, 1);
  if (max_per_sm > 0) per_sm = std::min(per_sm, max_per_sm);
  const int need = std::max(1, (cells0 + MQ - 1) / MQ);
  return std::max(1, std::min(sms * per_sm, need));
}

void mg_setup(const Dev& d, const MgDev& M, int x0_mode, const double* dz, const double* hist, cudaStream_t st) {
  k_mg_setup<<<(d.g.lm + PB - 1) / PB, PB, 0, st>>>(d, M, x0_mode, dz, hist);
  for (int k = 0; k + 1 < M.nlev; ++k) {
    const int n = M.lv[k + 1].rows * M.lv[k + 1].cols;
    k_mg_coarsen<<<(n + PB - 1) / PB, PB, 0, st>>>(M.lv[k], M.lv[k + 1]);
  }
}

int mg_solve(const MgDev& M, GridBar* bar, int nblocks, cudaStream_t st, const GridBar* init) {
  if (init) {
    if (cudaMemcpyAsync(bar, init, sizeof(GridBar), cudaMemcpyHostToDevice, st) != cudaSuccess) return -1;
  } else if (cudaMemsetAsync(bar, 0, sizeof(GridBar), st) != cudaSuccess) {
    return -1;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(MQ);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_mg_solve, M, bar) == cudaSuccess ? 0 : -1;
}

void mg_finish(const Dev& d, const MgDev& M, double* hist, cudaStream_t st) {
  k_mg_scatter<<<(d.g.lm + PB - 1) / PB, PB, 0, st>>>(d, M, hist);
}

}  // namespace si3d
