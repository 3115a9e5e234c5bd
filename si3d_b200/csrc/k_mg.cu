// Aggregation-multigrid preconditioned CG for the FP32 inner solves of iterative refinement
// (hierarchy and V-cycle: mg.h).  One cooperative launch runs a whole inner solve; its phases are
// separated by grid barriers (coop.cuh) and every block reduces the block partials itself in the
// same fixed order, so all blocks take the same alpha, beta and stopping decision.
//
// Phases of one iteration (a barrier after each):
//   U       u += alpha p, r -= alpha q (from the second iteration on), (r, r), and the first
//           (red) half-sweep of level 0 from z = 0, which is z = dinv r;
//           the stopping test (test 5 on the inner residual) right after its barrier
//   down    per level k < L - 1: black half-sweep; residual summed over 2 x 2 aggregates into
//           level k + 1's b, whose red cells get their first half-sweep z = dinv b
//   coarse  black then red half-sweep of the coarsest level, by block 0 alone
//   up      per level k = L - 2 .. 0: black half-sweep with the neighbours' values plus the coarse
//           correction of their aggregate; red half-sweep; at level 0 both add to (r, z)
//   PQ      beta, p = z + beta p and q = A p (neighbours' p formed on the fly), (p, q)
// With L levels that is 4 L - 1 barriers an iteration.
#include <algorithm>

#include "../../include/si3d_gpu.h"
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

size_t mg_level_elems(int rows, int cols) {
  const int pitch = ((cols + 3 + 31) / 32) * 32;
  return (size_t)(rows + 3) * (size_t)pitch;
}

namespace {

using namespace coop;

constexpr int PB = 256;               // threads per block of the setup kernels
constexpr float kFaceScale = 0.5f;    // coarse faces: half the sum of the crossing fine faces
constexpr int UN = 4;                 // cells a thread keeps in flight in the level loops

__device__ __forceinline__ int fdiv(const FastDiv& f, int x) {
  return (int)(((unsigned long long)(unsigned int)x * f.m) >> f.p);
}

// ---------------------------------------------------------------- per-solve setup
// Level 0 from the FP64 red-black system: the faces the system couples, the diagonal it applies
// (1 + sx + sx(W) + sy + sy(S)), and mass = diagonal - faces.
__global__ void k_mg_coef0(PcgDev P, MgDev M, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  const PcgColor& O = color ? P.R : P.B;
  if (i >= C.n) return;
  const int o = (color ? M.pixB : M.pixR)[i];
  const int4 q = C.nbr[i];   // W, S, N, E in the other colour (absent: O.n, the zero slot)
  const double sxi = C.sx[i], syi = C.sy[i], sxW = O.sx[q.x], syS = O.sy[q.y];
  const double diag = 1.0 + sxi + sxW + syi + syS;
  const double fN = (q.z != O.n) ? syi : 0.0;   // face to (i, j + 1): the next column
  const double fE = (q.w != O.n) ? sxi : 0.0;   // face to (i + 1, j): the next row
  const MgLevel& L = M.lv[0];
  L.fc[o] = (float)fN;
  L.fr[o] = (float)fE;
  L.mass[o] = (float)(diag - fN - fE - sxW - syS);
  L.dinv[o] = (float)(1.0 / diag);
}

// Level k + 1 from level k: 2 x 2 aggregates (frame cells read as zero).
__global__ void k_mg_coarsen(MgLevel F, MgLevel G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= G.rows * G.cols) return;
  const int R = t / G.cols, Cc = t - R * G.cols;
  const int fp = F.pitch;
  const int o00 = (2 * R + 1) * fp + 2 * Cc + 1, o01 = o00 + 1, o10 = o00 + fp, o11 = o10 + 1;
  const float mass = (F.mass[o00] + F.mass[o01]) + (F.mass[o10] + F.mass[o11]);
  const float fc = kFaceScale * (F.fc[o01] + F.fc[o11]);
  const float fr = kFaceScale * (F.fr[o10] + F.fr[o11]);
  const float fcW = kFaceScale * (F.fc[o00 - 1] + F.fc[o10 - 1]);
  const float frS = kFaceScale * (F.fr[o00 - fp] + F.fr[o01 - fp]);
  const int O = (R + 1) * G.pitch + Cc + 1;
  G.fc[O] = fc;
  G.fr[O] = fr;
  G.mass[O] = mass;
  const float diag = mass + fc + fr + fcW + frS;
  G.dinv[O] = diag > 0.f ? 1.f / diag : 0.f;
}

// Inner right-hand side: the FP64 outer residual rounded to FP32; the correction starts at zero.
__global__ void k_mg_inner_setup(PcgDev P, MgDev M, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i >= C.n) return;
  const int o = (color ? M.pixB : M.pixR)[i];
  M.lv[0].b[o] = (float)C.r[i];
  M.u[o] = 0.f;
}

__global__ void k_mg_correct(PcgDev P, MgDev M, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i >= C.n) return;
  C.u[i] = C.u[i] + (double)M.u[(color ? M.pixB : M.pixR)[i]];
}

// ---------------------------------------------------------------- V-cycle pieces
// Gauss-Seidel half-sweep over the cells of colour `col` ((r + c) & 1 == col) of level L:
// z = dinv (b + sum of face * neighbour z).  PROLONG: each neighbour's value is its z plus the
// correction of its aggregate in the coarser level G.  DOT: returns this thread's sum of b * z.
template <bool PROLONG, bool DOT>
__device__ __forceinline__ double half_sweep(const MgLevel& L, const MgLevel& G, int col, int g0, int stride) {
  double rz = 0.0;
  const int n = L.rows * L.hw, pt = L.pitch;
  for (int h0 = g0; h0 < n; h0 += UN * stride) {
    int o[UN];
    bool ok[UN];
    float s[UN], dv[UN], bb[UN];
#pragma unroll
    for (int k = 0; k < UN; ++k) {
      const int h = h0 + k * stride;
      int r = fdiv(L.div_hw, h);
      int c = 2 * (h - r * L.hw) + ((r + col) & 1);
      ok[k] = (h < n) && (c < L.cols);
      if (!ok[k]) { r = 0; c = 0; }   // an interior cell, loaded and dropped
      o[k] = (r + 1) * pt + c + 1;
      float zw = L.z[o[k] - 1], ze = L.z[o[k] + 1], zs = L.z[o[k] - pt], zn = L.z[o[k] + pt];
      if (PROLONG) {
        const int gp = G.pitch;
        const int row = ((r >> 1) + 1) * gp;
        zw += G.z[row + ((c - 1) >> 1) + 1];
        ze += G.z[row + ((c + 1) >> 1) + 1];
        zs += G.z[(((r - 1) >> 1) + 1) * gp + (c >> 1) + 1];
        zn += G.z[(((r + 1) >> 1) + 1) * gp + (c >> 1) + 1];
      }
      bb[k] = L.b[o[k]];
      s[k] = bb[k] + L.fc[o[k]] * ze + L.fc[o[k] - 1] * zw + L.fr[o[k]] * zn + L.fr[o[k] - pt] * zs;
      dv[k] = L.dinv[o[k]];
    }
#pragma unroll
    for (int k = 0; k < UN; ++k) {
      if (!ok[k]) continue;
      const float z = dv[k] * s[k];
      L.z[o[k]] = z;
      if (DOT) rz += (double)bb[k] * (double)z;
    }
  }
  return rz;
}

// b of level G = the residual b - A z of level F summed over each 2 x 2 aggregate; the red cells of
// G then take their first half-sweep from zero, z = dinv b.
__device__ __forceinline__ void restrict_residual(const MgLevel& F, const MgLevel& G, int g0, int stride) {
  const int n = G.rows * G.cols, fp = F.pitch;
  for (int t0 = g0; t0 < n; t0 += 2 * stride) {
    float acc[2];
    int O[2];
    bool ok[2], red[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int t = t0 + k * stride;
      ok[k] = t < n;
      int R = ok[k] ? fdiv(G.div_cols, t) : 0;
      int Cc = ok[k] ? t - R * G.cols : 0;
      O[k] = (R + 1) * G.pitch + Cc + 1;
      red[k] = ((R + Cc) & 1) == 0;
      const int o00 = (2 * R + 1) * fp + 2 * Cc + 1;
      float a = 0.f;
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const int o = o00 + (ch >> 1) * fp + (ch & 1);
        const float fcw = F.fc[o - 1], fce = F.fc[o], frs = F.fr[o - fp], frn = F.fr[o];
        const float diag = F.mass[o] + fcw + fce + frs + frn;
        const float az = diag * F.z[o] - fce * F.z[o + 1] - fcw * F.z[o - 1] - frn * F.z[o + fp] - frs * F.z[o - fp];
        a += F.b[o] - az;
      }
      acc[k] = a;
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (!ok[k]) continue;
      G.b[O[k]] = acc[k];
      if (red[k]) G.z[O[k]] = G.dinv[O[k]] * acc[k];
    }
  }
}

// ---------------------------------------------------------------- the inner solve
__global__ void __launch_bounds__(QB, 2) k_mg_loop(MgDev M, GridBar* bar) {
  __shared__ double sh[8 + 1];
  __shared__ int s_flag;
  __shared__ MgLevel s_lv[kMgMaxLevels];
  const int nlev = M.nlev;
  if (threadIdx.x < nlev) s_lv[threadIdx.x] = M.lv[threadIdx.x];
  __syncthreads();
  PcgScal* SC = M.sc;
  const int nb = gridDim.x, stride = nb * QB, g0 = blockIdx.x * QB + threadIdx.x;
  double* const rr_part = M.part;
  double* const rz_part = M.part + nb;
  double* const pq_part = M.part + 3 * nb;
  const double zeta = SC->zeta, bnorm = SC->bnorm;
  const int itmax = SC->itmax;
  double alpha = 0.0, beta = 0.0, rz_old = 1.0, stptst = 1.0;
  int it = 0, ier = 0;
  const MgLevel& L0 = s_lv[0];
  const int n0 = L0.rows * L0.cols, pt = L0.pitch;
  for (;;) {
    // ---- U: u += alpha p, r -= alpha q; (r, r); red half-sweep of level 0 from zero
    {
      const float a = (float)alpha;
      const float* __restrict__ pn = (it & 1) ? M.p1 : M.p0;
      double rr = 0.0;
      for (int t0 = g0; t0 < n0; t0 += UN * stride) {
        int o[UN];
        bool ok[UN], red[UN];
        float rv[UN], dv[UN], uv[UN], pv[UN], qv[UN];
#pragma unroll
        for (int k = 0; k < UN; ++k) {
          const int t = t0 + k * stride;
          ok[k] = t < n0;
          const int r = ok[k] ? fdiv(L0.div_cols, t) : 0;
          const int c = ok[k] ? t - r * L0.cols : 0;
          o[k] = (r + 1) * pt + c + 1;
          red[k] = ((r + c) & 1) == 0;
          rv[k] = L0.b[o[k]];
          dv[k] = L0.dinv[o[k]];
          if (it > 0) { uv[k] = M.u[o[k]]; pv[k] = pn[o[k]]; qv[k] = M.q[o[k]]; }
        }
#pragma unroll
        for (int k = 0; k < UN; ++k) {
          if (!ok[k]) continue;
          float r = rv[k];
          if (it > 0) {
            M.u[o[k]] = uv[k] + a * pv[k];
            r = r - a * qv[k];
            L0.b[o[k]] = r;
          }
          rr += (double)r * (double)r;
          if (red[k]) L0.z[o[k]] = dv[k] * r;
        }
      }
      double w[1] = {rr};
      bsum<1>(w, sh);
      if (threadIdx.x == 0) rr_part[blockIdx.x] = w[0];
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
    {
      double w[1];
      all_partials<1>(rr_part, nb, 0, w, sh);
      const double tl = sqrt(w[0]);
      stptst = tl / bnorm;
      if (tl < bnorm * zeta) break;
      if (it >= itmax) { ier = 1; break; }
    }
    // ---- down: black half-sweep, restriction
    for (int k = 0; k < nlev - 1; ++k) {
      half_sweep<false, false>(s_lv[k], s_lv[k], 1, g0, stride);
      if (!grid_barrier(bar, SC, &s_flag)) return;
      restrict_residual(s_lv[k], s_lv[k + 1], g0, stride);
      if (!grid_barrier(bar, SC, &s_flag)) return;
    }
    // ---- coarsest level: black, red (one block)
    if (blockIdx.x == 0) {
      const MgLevel& Lc = s_lv[nlev - 1];
      half_sweep<false, false>(Lc, Lc, 1, threadIdx.x, QB);
      __syncthreads();
      half_sweep<false, false>(Lc, Lc, 0, threadIdx.x, QB);
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
    // ---- up: black half-sweep with the coarse correction, red half-sweep; (r, z) at level 0
    for (int k = nlev - 2; k >= 0; --k) {
      if (k == 0) {
        double w[1] = {half_sweep<true, true>(s_lv[0], s_lv[1], 1, g0, stride)};
        bsum<1>(w, sh);
        if (threadIdx.x == 0) rz_part[blockIdx.x] = w[0];
      } else {
        half_sweep<true, false>(s_lv[k], s_lv[k + 1], 1, g0, stride);
      }
      if (!grid_barrier(bar, SC, &s_flag)) return;
      if (k == 0) {
        double w[1] = {half_sweep<false, true>(s_lv[0], s_lv[0], 0, g0, stride)};
        bsum<1>(w, sh);
        if (threadIdx.x == 0) rz_part[nb + blockIdx.x] = w[0];
      } else {
        half_sweep<false, false>(s_lv[k], s_lv[k], 0, g0, stride);
      }
      if (!grid_barrier(bar, SC, &s_flag)) return;
    }
    {
      double w[1];
      all_partials<1>(rz_part, 2 * nb, 0, w, sh);
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
      for (int t0 = g0; t0 < n0; t0 += UN * stride) {
        int o[UN];
        bool ok[UN];
        float pc[UN], qv[UN];
#pragma unroll
        for (int k = 0; k < UN; ++k) {
          const int t = t0 + k * stride;
          ok[k] = t < n0;
          const int r = ok[k] ? fdiv(L0.div_cols, t) : 0;
          const int c = ok[k] ? t - r * L0.cols : 0;
          const int x = (r + 1) * pt + c + 1;
          o[k] = x;
          float p0 = L0.z[x], pW = L0.z[x - 1], pE = L0.z[x + 1], pS = L0.z[x - pt], pN = L0.z[x + pt];
          if (!first) {
            p0 += bt * po[x]; pW += bt * po[x - 1]; pE += bt * po[x + 1]; pS += bt * po[x - pt]; pN += bt * po[x + pt];
          }
          const float fcw = L0.fc[x - 1], fce = L0.fc[x], frs = L0.fr[x - pt], frn = L0.fr[x];
          const float diag = L0.mass[x] + fcw + fce + frs + frn;
          pc[k] = p0;
          qv[k] = diag * p0 - fce * pE - fcw * pW - frn * pN - frs * pS;
        }
#pragma unroll
        for (int k = 0; k < UN; ++k) {
          if (!ok[k]) continue;
          pw[o[k]] = pc[k];
          M.q[o[k]] = qv[k];
          pq += (double)pc[k] * (double)qv[k];
        }
      }
      double w[1] = {pq};
      bsum<1>(w, sh);
      if (threadIdx.x == 0) pq_part[blockIdx.x] = w[0];
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
    {
      double w[1];
      all_partials<1>(pq_part, nb, 0, w, sh);
      if (!(w[0] > 0.0)) { ier = -6; break; }
      alpha = rz_old / w[0];
    }
    ++it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SC->in = it;
    SC->stptst = stptst;
    SC->ier = ier;
    SC->done = 1;
  }
}

}  // namespace

int mg_loop_blocks(int device, int cells0, int max_per_sm) {
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_loop, QB, 0);
  int per_sm = std::max(occ, 1);
  if (max_per_sm > 0) per_sm = std::min(per_sm, max_per_sm);
  const int need = std::max(1, (cells0 + QB - 1) / QB);
  return std::max(1, std::min(sms * per_sm, need));
}

void mg_setup(const PcgDev& P, const MgDev& M, cudaStream_t st) {
  if (P.R.n > 0) k_mg_coef0<<<(P.R.n + PB - 1) / PB, PB, 0, st>>>(P, M, 0);
  if (P.B.n > 0) k_mg_coef0<<<(P.B.n + PB - 1) / PB, PB, 0, st>>>(P, M, 1);
  for (int k = 0; k + 1 < M.nlev; ++k) {
    const int n = M.lv[k + 1].rows * M.lv[k + 1].cols;
    k_mg_coarsen<<<(n + PB - 1) / PB, PB, 0, st>>>(M.lv[k], M.lv[k + 1]);
  }
}

void mg_inner_setup(const PcgDev& P, const MgDev& M, cudaStream_t st) {
  if (P.R.n > 0) k_mg_inner_setup<<<(P.R.n + PB - 1) / PB, PB, 0, st>>>(P, M, 0);
  if (P.B.n > 0) k_mg_inner_setup<<<(P.B.n + PB - 1) / PB, PB, 0, st>>>(P, M, 1);
}

void mg_correct(const PcgDev& P, const MgDev& M, cudaStream_t st) {
  if (P.R.n > 0) k_mg_correct<<<(P.R.n + PB - 1) / PB, PB, 0, st>>>(P, M, 0);
  if (P.B.n > 0) k_mg_correct<<<(P.B.n + PB - 1) / PB, PB, 0, st>>>(P, M, 1);
}

int mg_loop(const MgDev& M, GridBar* bar, int nblocks, cudaStream_t st) {
  if (cudaMemsetAsync(bar, 0, sizeof(GridBar), st) != cudaSuccess) return -1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(QB);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_mg_loop, M, bar) == cudaSuccess ? 0 : -1;
}

}  // namespace si3d
