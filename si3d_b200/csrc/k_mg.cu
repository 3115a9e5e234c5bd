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
//           level k + 1's b, whose red cells get their first half-sweep z = dinv b
//   coarse  black then red half-sweep of the coarsest level, by block 0 alone
//   up      per level k = L - 2 .. 0: black half-sweep with the neighbours' values plus the coarse
//           correction of their aggregate; red half-sweep; at level 0 both add to (r, z)
//   PQ      beta, p = z + beta p and q = A p (neighbours' p formed on the fly), (p, q)
// With L levels that is 4 L - 1 barriers an inner iteration.
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

size_t mg_level_elems(int rows, int cols) {
  const int pitch = ((cols + 3 + 31) / 32) * 32;
  return (size_t)(rows + 3) * (size_t)pitch;
}

namespace {

using namespace coop;

constexpr int PB = 256;               // threads per block of the setup kernels
constexpr float kFaceScale = 0.5f;    // coarse faces: half the sum of the crossing fine faces
constexpr int UN = 4;                 // cells a thread keeps in flight in the level loops
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
// FP32 MG-PCG on level 0 from e = 0 (M.u) with right-hand side r (level 0's b), until
// ||r|| < bnorm * zeta or itmax iterations.  Returns false when a barrier gave up (the caller returns
// at once); otherwise its = the iterations taken and ier = 0, 1 (itmax) or -6 / -7 (breakdown).
__device__ bool mg_pcg(const MgDev& M, const MgLevel* s_lv, int nlev, GridBar* bar, PcgScal* SC, BarSt* s_flag,
                       double* sh, double zeta, double bnorm, int itmax, int& its, int& ier) {
  const int nb = gridDim.x, stride = nb * MQ, g0 = blockIdx.x * MQ + threadIdx.x;
  double* const rr_part = M.part;
  double* const rz_part = M.part + nb;
  double* const pq_part = M.part + 3 * nb;
  double alpha = 0.0, beta = 0.0, rz_old = 1.0;
  int it = 0;
  ier = 0;
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
    // ---- down: black half-sweep, restriction
    for (int k = 0; k < nlev - 1; ++k) {
      half_sweep<false, false>(s_lv[k], s_lv[k], 1, g0, stride);
      if (!grid_barrier(bar, SC, s_flag)) return false;
      restrict_residual(s_lv[k], s_lv[k + 1], g0, stride);
      if (!grid_barrier(bar, SC, s_flag)) return false;
    }
    // ---- coarsest level: black, red (one block)
    if (blockIdx.x == 0) {
      const MgLevel& Lc = s_lv[nlev - 1];
      half_sweep<false, false>(Lc, Lc, 1, threadIdx.x, MQ);
      __syncthreads();
      half_sweep<false, false>(Lc, Lc, 0, threadIdx.x, MQ);
    }
    if (!grid_barrier(bar, SC, s_flag)) return false;
    // ---- up: black half-sweep with the coarse correction, red half-sweep; (r, z) at level 0
    for (int k = nlev - 2; k >= 0; --k) {
      if (k == 0) {
        double w[1] = {half_sweep<true, true>(s_lv[0], s_lv[1], 1, g0, stride)};
        bsum<1, MQ>(w, sh);
        if (threadIdx.x == 0) rz_part[blockIdx.x] = w[0];
      } else {
        half_sweep<true, false>(s_lv[k], s_lv[k + 1], 1, g0, stride);
      }
      if (!grid_barrier(bar, SC, s_flag)) return false;
      if (k == 0) {
        double w[1] = {half_sweep<false, true>(s_lv[0], s_lv[0], 0, g0, stride)};
        bsum<1, MQ>(w, sh);
        if (threadIdx.x == 0) rz_part[nb + blockIdx.x] = w[0];
      } else {
        half_sweep<false, false>(s_lv[k], s_lv[k], 0, g0, stride);
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
  const int nb = gridDim.x, stride = nb * MQ, g0 = blockIdx.x * MQ + threadIdx.x;
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
        const int o = (r + 1) * pt + c + 1;
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
          const int x = (r + 1) * pt + c + 1;
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
