// Free-surface system assembly and the MIC-preconditioned CG zeta solve.
//
// matcon (si3d_procedures.f90:1749-1867) builds sx, sy, dd, qq, rr per column.  SolverSparse
// (:1870-2065) hands the 5-point system to NSPCG's mic1 + cg (nspcg.f:1441, :8328, :8967).  The
// GPU form runs NSPCG's own red-black variant of that method (iperm = 1): the unknowns are split
// by the prbndx colouring (nspcg.f:25337) into a red and a black list, each kept in l order, so
// MIC(0) with property A (icfp, nspcg.f:20789-20806) reduces to a diagonal update of the black
// pivots, and one application of M^-1 = a black pass followed by a red pass (icfstp/icbsp,
// nspcg.f:22875, :22729) — two fully parallel sweeps instead of the natural ordering's
// sequential recurrences.
//
// Data layout: every PCG vector lives in two colour arrays (n_c + 1 entries; entry n_c is a
// permanent zero used by absent neighbours).  Each node stores its four neighbours (W, S, N, E) as
// indices into the other colour's arrays (int4, one 16-byte load).  At 2000 x 1000 cells the whole
// working set (u, r, z, p, q, sx, sy, 1/d) is about 90 MB, so after the first iteration the solve
// streams from the 126 MB L2 rather than from HBM.
//
// One CG iteration = 4 kernels: black M^-1 pass, red M^-1 pass (+ (r,z) reduction -> beta and the
// stopping test), black p/q update, red p/q update (+ (p,q) reduction -> alpha).  The u += alpha p
// and r -= alpha q updates of itcg are fused into the next iteration's M^-1 passes.  Global sums
// use fixed-order block partials reduced by the last block to finish (no spin-waits), so results
// are deterministic.  Scalars stay on the device; every kernel returns at once when `done` is set,
// which lets the host run batches of iterations without a round trip per iteration.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace si3d {

// ------------------------------------------------------------------ matcon
__global__ void k_matcon(Dev d) {
  double* __restrict__ f_uhpp = d.f.uhpp;
  double* __restrict__ f_vhpp = d.f.vhpp;
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const double tz = d.tz;
  const double cx = d.p.gdt2dx2 * tz * tz, cy = d.p.gdt2dy2 * tz * tz;
  const double dtdx1 = d.p.dtdx * tz, dtdy1 = d.p.dtdy * tz, dt1 = d.p.dt * tz;
  const int lm1 = d.g.lm1;
  const int lE = NB(d.g.lEC, l), lN = NB(d.g.lNC, l), lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l);
  // sx, sy of this column and of its W/S neighbours (the latter recomputed identically so the
  // kernel needs no second pass; Bsx(Bend+1) = Bsy(Bend+1) = 0 for the dry sentinel).
  auto sxof = [&](int m) -> double {
    if (m == lm1) return 0.0;
    return (NB(d.g.lEC, m) != lm1) ? cx * 1000. * d.s.earx[m - 1] : 0.0;
  };
  auto syof = [&](int m) -> double {
    if (m == lm1) return 0.0;
    return (NB(d.g.lNC, m) != lm1) ? cy * 1000. * d.s.eary[m - 1] : 0.0;
  };
  const double sxl = (lE != lm1) ? cx * 1000. * d.s.earx[l - 1] : 0.0;
  const double syl = (lN != lm1) ? cy * 1000. * d.s.eary[l - 1] : 0.0;
  d.s.sx[l - 1] = sxl;
  d.s.sy[l - 1] = syl;
  const int kms = NB(d.g.kmz, l);
  const double rdx = 1.0 / d.p.dx, rdy = 1.0 / d.p.dy;   // divisions by the grid constants as products
  double sum = 0;
  #pragma unroll 4
  for (int k = d.g.k1; k <= kms; ++k)
    sum += (f_uhpp[IX(d, k, l)] - f_uhpp[IX(d, k, lW)]) * rdx +
           (f_vhpp[IX(d, k, l)] - f_vhpp[IX(d, k, lS)]) * rdy;
  const double ddv = dt1 * sum;
  d.s.dd[l - 1] = ddv;
  d.s.qq[l - 1] = d.s.spp[l - 1] - dtdx1 * (d.s.eagx[l - 1] - d.s.eagx[lW - 1]) -
                  dtdy1 * (d.s.eagy[l - 1] - d.s.eagy[lS - 1]) - ddv;
  d.s.rr[l - 1] = 1 + sxl + sxof(lW) + syl + syof(lS);
}

void launch_matcon(const Dev& d, cudaStream_t st) {
  const int B = 256;
  k_matcon<<<(d.g.lm + B - 1) / B, B, 0, st>>>(d);
}

// ------------------------------------------------------------------ red-black PCG
namespace {

constexpr int PB = 256;  // threads per block of the PCG kernels

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (ln == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = (ln < (int)(blockDim.x >> 5)) ? sh[ln] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

// Fixed-order reduction of `n` block partials by the calling (last) block.
__device__ __forceinline__ double reduce_partials(const double* part, int n, double* sh) {
  double v = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  return block_sum(v, sh);
}

// Returns true in every thread of the block that finished last.
__device__ __forceinline__ bool last_block(unsigned int* counter) {
  __shared__ bool amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int prev = atomicAdd(counter, 1u);
    amlast = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (amlast) {
    __threadfence();
    if (threadIdx.x == 0) *counter = 0u;
  }
  return amlast;
}

}  // namespace

// Gather the assembled system into colour order: sx, sy, rhs and the initial guess.
__global__ void k_pcg_gather(Dev d, PcgDev P, int color, int x0_mode, const double* __restrict__ dz,
                             const double* __restrict__ hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i > C.n) return;
  if (i == C.n) {  // the permanent zero slot
    C.sx[i] = 0.0; C.sy[i] = 0.0; C.u[i] = 0.0; C.r[i] = 0.0; C.z[i] = 0.0; C.p[i] = 0.0; C.p2[i] = 0.0;
    C.q[i] = 0.0;
    C.rhs[i] = 0.0; C.dinv[i] = 0.0; C.diag[i] = 0.0;
    return;
  }
  const int l = C.l[i];
  C.sx[i] = d.s.sx[l - 1];
  C.sy[i] = d.s.sy[l - 1];
  C.rhs[i] = d.s.qq[l - 1];
  // matcon's rr: 1 + sx + sx(W) + sy + sy(S), formed before open boundaries cut their faces
  C.diag[i] = d.s.rr[l - 1];
  // x0: sp (the reference), zero, sp + learned increment, s (the latest accepted solution),
  // or s + this solve's correction one step earlier
  double x0;
  switch (x0_mode) {
    case 1: x0 = 0.0; break;
    case 3: x0 = d.s.s[l - 1]; break;
    case 4: x0 = d.s.s[l - 1] + (hist ? hist[i] : 0.0); break;
    default: x0 = d.s.sp[l - 1]; if (x0_mode == 2 && dz) x0 = x0 + dz[l - 1];
  }
  C.u[i] = x0;
  C.z[i] = 0.0; C.p[i] = 0.0; C.p2[i] = 0.0; C.q[i] = 0.0;
}

// Red pivots are the diagonal itself (no lower neighbours in red-black order).
__global__ void k_pcg_factor_red(PcgDev P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  if (i >= R.n) return;
  const int4 nb = R.nbr[i];
  const double diag = R.diag[i];
  R.dinv[i] = 1.0 / diag;
  // row sum of the upper triangle T (icfp wksp, nspcg.f:20786-20789), columns W, S, N, E
  const double tW = -B.sx[nb.x], tS = -B.sy[nb.y], tN = -R.sy[i], tE = -R.sx[i];
  R.rs[i] = (((0.0 + tW) + tS) + tN) + tE;
}

// Black pivots: d(j) -= t(k,j)/d(k) * (omega*rowsum_T(k) - (omega-1)*t(k,j)) for every red
// neighbour k in increasing l order (W, S, N, E), omega = 1 (icfp, nspcg.f:20797-20806).
__global__ void k_pcg_factor_black(PcgDev P, int* __restrict__ negpiv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  if (j >= B.n) return;
  const int4 nb = B.nbr[j];
  double dj = B.diag[j];
  const double omega = 1.0;
  const int ks[4] = {nb.x, nb.y, nb.z, nb.w};
  const double t[4] = {-R.sx[nb.x], -R.sy[nb.y], -B.sy[j], -B.sx[j]};
  for (int c = 0; c < 4; ++c) {
    const int k = ks[c];
    if (k == R.n) continue;  // absent neighbour: NSPCG skips jcol == k
    const double term = t[c] / R.diag[k];
    dj = dj - term * (omega * R.rs[k] - (omega - 1.0) * t[c]);
  }
  if (dj < 0.0) atomicOr(negpiv, 1);    // negative pivot: ier = 5 (pfact1, nspcg.f:6654)
  if (dj == 0.0) atomicOr(negpiv, 2);   // zero pivot: ier = -12
  B.dinv[j] = 1.0 / dj;
}

// r = rhs - A u in both colours (itcg start, nspcg.f:9024-9026); order of mult1 after move1:
// diagonal, then W, S, N, E.
__global__ void k_pcg_resid0(PcgDev P, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  const PcgColor& O = color ? P.R : P.B;
  if (i >= C.n) return;
  const int4 nb = C.nbr[i];
  const double diag = C.diag[i];
  double y = diag * C.u[i];
  y = y + (-O.sx[nb.x]) * O.u[nb.x];
  y = y + (-O.sy[nb.y]) * O.u[nb.y];
  y = y + (-C.sy[i]) * O.u[nb.z];
  y = y + (-C.sx[i]) * O.u[nb.w];
  C.r[i] = C.rhs[i] - y;
}

// bnorm = max(sqrt(rhs.rhs), srelpr) for stopping test 5 (nmcalc, nspcg.f:24248-24252)
__global__ void k_pcg_bnorm(PcgDev P) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nR = P.R.n, nB = P.B.n;
  double v = 0;
  if (i < nR) v = P.R.rhs[i] * P.R.rhs[i];
  else if (i < nR + nB) v = P.B.rhs[i - nR] * P.B.rhs[i - nR];
  const double bs = block_sum(v, sh);
  if (threadIdx.x == 0) P.part0[blockIdx.x] = bs;
  if (last_block(&P.sc->cnt[3])) {
    const double tot = reduce_partials(P.part0, gridDim.x, sh);
    if (threadIdx.x == 0) P.sc->bnorm = fmax(sqrt(tot), P.sc->srelpr);
  }
}

// Each thread of the iteration kernels handles NPT nodes of one colour (node = block base +
// r * PB + thread, so every r-slice is a coalesced access and the NPT slices are independent
// loads in flight).  Fewer, fuller blocks keep the last-block reductions short.
constexpr int NPT = 4;

// Black half of z = M^-1 r, fused with u += alpha p and r -= alpha q (itcg :9031, :9088).
// `par` selects the current p buffer (p is double-buffered across iterations).
template <typename T>
__global__ void __launch_bounds__(PB) k_pcg_black_solve(PcgDevT<T> P, int par) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const PcgColorT<T> &R = P.R, &B = P.B;
  const T* __restrict__ Bp = par ? B.p2 : B.p;
  const T alpha = (T)P.sc->alpha;
  double rr = 0, rz = 0, uu = 0, zz = 0;
#pragma unroll
  for (int q = 0; q < NPT; ++q) {
    const int j = blockIdx.x * (PB * NPT) + q * PB + threadIdx.x;
    if (j < B.n) {
      const int4 nb = B.nbr[j];
      const T uj = B.u[j] + alpha * Bp[j];
      const T rj = B.r[j] - alpha * B.q[j];
      B.u[j] = uj;
      B.r[j] = rj;
      // icfstp: the red rows scatter into this black row in l order W, S, N, E
      const int ks[4] = {nb.x, nb.y, nb.z, nb.w};
      const T t[4] = {-R.sx[nb.x], -R.sy[nb.y], -B.sy[j], -B.sx[j]};
      T x = rj;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int k = ks[c];
        const T rk = R.r[k] - alpha * R.q[k];
        const T xfk = rk * R.dinv[k];
        x = x - t[c] * xfk;
      }
      const T dj = B.dinv[j];
      x = x * dj;                // icfstp: x(i) = x(i)*d(i)
      x = x / dj;                // icsp:   x(i) = x(i)/d(i)
      const T zj = x * dj;  // icbsp on a row with no upper entries
      B.z[j] = zj;
      rr += (double)rj * (double)rj; rz += (double)rj * (double)zj; uu += (double)uj * (double)uj;
      zz += (double)zj * (double)zj;
    }
  }
  double s;
  s = block_sum(rr, sh); if (threadIdx.x == 0) P.part0[blockIdx.x] = s;
  s = block_sum(rz, sh); if (threadIdx.x == 0) P.part1[blockIdx.x] = s;
  if (P.sc->ntest == 2) {
    s = block_sum(uu, sh); if (threadIdx.x == 0) P.part2[blockIdx.x] = s;
    s = block_sum(zz, sh); if (threadIdx.x == 0) P.part3[blockIdx.x] = s;
  }
}

// Red half of z = M^-1 r (+ u/r updates), then the (r,z) reduction, the stopping test and beta.
template <typename T>
__global__ void __launch_bounds__(PB) k_pcg_red_solve(PcgDevT<T> P, int par, int nblk_black) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const PcgColorT<T> &R = P.R, &B = P.B;
  const T* __restrict__ Rp = par ? R.p2 : R.p;
  const T alpha = (T)P.sc->alpha;
  double rr = 0, rz = 0, uu = 0, zz = 0;
#pragma unroll
  for (int q = 0; q < NPT; ++q) {
    const int k = blockIdx.x * (PB * NPT) + q * PB + threadIdx.x;
    if (k < R.n) {
      const int4 nb = R.nbr[k];
      const T uk = R.u[k] + alpha * Rp[k];
      const T rk = R.r[k] - alpha * R.q[k];
      R.u[k] = uk;
      R.r[k] = rk;
      const T dk = R.dinv[k];
      T x = rk * dk;   // icfstp
      x = x / dk;           // icsp
      // icbsp: sum = x - t(k,W) z_W - t(k,S) z_S - t(k,N) z_N - t(k,E) z_E
      x = x - (-B.sx[nb.x]) * B.z[nb.x];
      x = x - (-B.sy[nb.y]) * B.z[nb.y];
      x = x - (-R.sy[k]) * B.z[nb.z];
      x = x - (-R.sx[k]) * B.z[nb.w];
      const T zk = x * dk;
      R.z[k] = zk;
      rr += (double)rk * (double)rk; rz += (double)rk * (double)zk; uu += (double)uk * (double)uk;
      zz += (double)zk * (double)zk;
    }
  }
  const int off = nblk_black;
  double s;
  s = block_sum(rr, sh); if (threadIdx.x == 0) P.part0[off + blockIdx.x] = s;
  s = block_sum(rz, sh); if (threadIdx.x == 0) P.part1[off + blockIdx.x] = s;
  if (P.sc->ntest == 2) {
    s = block_sum(uu, sh); if (threadIdx.x == 0) P.part2[off + blockIdx.x] = s;
    s = block_sum(zz, sh); if (threadIdx.x == 0) P.part3[off + blockIdx.x] = s;
  }
  if (!last_block(&P.sc->cnt[0])) return;
  const int ntot = off + gridDim.x;
  const double rrt = reduce_partials(P.part0, ntot, sh);
  __syncthreads();
  const double rzt = reduce_partials(P.part1, ntot, sh);
  __syncthreads();
  double uut = 0, zzt = 0;
  if (P.sc->ntest == 2) {
    uut = reduce_partials(P.part2, ntot, sh);
    __syncthreads();
    zzt = reduce_partials(P.part3, ntot, sh);
  }
  if (threadIdx.x != 0) return;
  PcgScal* S = P.sc;
  S->dkm1 = S->rzdot;
  S->rzdot = rzt;
  if (!(rzt > 0.0)) { S->ier = -7; S->done = 1; return; }
  // pstops (nspcg.f:25956-26100)
  const double tiny = 500.0 * S->srelpr;
  bool halt = false;
  if (S->ntest == 5) {
    const double tl = sqrt(rrt), tr = S->bnorm;
    S->stptst = tl / tr;
    halt = tl < tr * S->zeta;
  } else {
    if (S->in < 1) {
      S->q1 = 0;
      S->udnm = 1.0;
      S->stptst = sqrt(rzt);
      halt = S->stptst < tiny;
    } else {
      if (!S->q1 && !((S->in > 5) && (S->in % 5 != 0))) {
        const double uold = S->udnm;
        S->udnm = sqrt(uut);
        if (S->udnm < tiny) S->udnm = 1.0;
        if ((S->in > 5) && (fabs(S->udnm - uold) < S->udnm * S->zeta)) S->q1 = 1;
      }
      double eminl = S->emin;
      if (eminl < tiny) eminl = tiny;
      const double tl = sqrt(zzt), tr = S->udnm * eminl;
      S->stptst = tl / tr;
      halt = tl < tr * S->zeta;
    }
  }
  if (halt) { S->done = 1; return; }
  if (!(S->in < S->itmax)) { S->ier = 1; S->done = 1; return; }
  if (S->in != 0) S->beta = S->rzdot / S->dkm1;
}

// p = z + beta p and q = A p on both colours in one launch (blocks [0, nblk_red) take red
// nodes, the rest black).  The other colour's new p is formed on the fly from its z and old p,
// with the same expression, so both colours see identical values; p is double-buffered.
// Then (p,q), alpha and the iteration count (itcg :9064-9086).
template <typename T, bool DIAG>
__global__ void __launch_bounds__(PB) k_pcg_apply(PcgDevT<T> P, int par, int nblk_red) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const bool red = blockIdx.x < (unsigned)nblk_red;
  const PcgColorT<T>& C = red ? P.R : P.B;
  const PcgColorT<T>& O = red ? P.B : P.R;
  const T* __restrict__ Cp = par ? C.p2 : C.p;
  const T* __restrict__ Op = par ? O.p2 : O.p;
  T* __restrict__ Cn = par ? C.p : C.p2;
  const int blk = red ? blockIdx.x : blockIdx.x - nblk_red;
  const T beta = (T)P.sc->beta;
  double pq = 0;
#pragma unroll
  for (int q = 0; q < NPT; ++q) {
    const int i = blk * (PB * NPT) + q * PB + threadIdx.x;
    if (i < C.n) {
      const int4 nb = C.nbr[i];
      const T pi = C.z[i] + beta * Cp[i];
      const T pW = O.z[nb.x] + beta * Op[nb.x];
      const T pS = O.z[nb.y] + beta * Op[nb.y];
      const T pN = O.z[nb.z] + beta * Op[nb.z];
      const T pE = O.z[nb.w] + beta * Op[nb.w];
      const T sxW = O.sx[nb.x], syS = O.sy[nb.y];
      const T diag = DIAG ? C.diag[i] : (T)1 + C.sx[i] + sxW + C.sy[i] + syS;
      T y = diag * pi;
      y = y + (-sxW) * pW;
      y = y + (-syS) * pS;
      y = y + (-C.sy[i]) * pN;
      y = y + (-C.sx[i]) * pE;
      Cn[i] = pi;
      C.q[i] = y;
      pq += (double)pi * (double)y;
    }
  }
  const double s = block_sum(pq, sh);
  if (threadIdx.x == 0) P.part0[blockIdx.x] = s;
  if (!last_block(&P.sc->cnt[1])) return;
  const double pap = reduce_partials(P.part0, gridDim.x, sh);
  if (threadIdx.x != 0) return;
  PcgScal* S = P.sc;
  S->alphao = S->alpha;
  S->pap = pap;
  S->alpha = S->rzdot / pap;
  if (!(pap > 0.0)) { S->ier = -6; S->done = 1; return; }
  if (S->in < S->hist_cap) { P.hist_alpha[S->in] = S->alpha; P.hist_beta[S->in] = S->beta; }
  S->in += 1;
}

// zeta back to column order: s(l) = zeta(l) (SolverSparse :2035-2040)
// With `hist`, also this solve's correction to the zeta it started from (s before the write), in
// colour order, for the next step's guess of the same solve.
__global__ void k_pcg_scatter(Dev d, PcgDev P, int color, double* __restrict__ hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i >= C.n) return;
  const int l = C.l[i];
  const double u = C.u[i];
  if (hist) hist[i] = u - d.s.s[l - 1];
  d.s.s[l - 1] = u;
}

void pcg_setup(const Dev& d, const PcgDev& P, int x0_mode, const double* dz, const double* hist, int* negpiv,
               cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  k_pcg_gather<<<(nR + 1 + PB - 1) / PB, PB, 0, st>>>(d, P, 0, x0_mode, dz, hist);
  k_pcg_gather<<<(nB + 1 + PB - 1) / PB, PB, 0, st>>>(d, P, 1, x0_mode, dz, hist ? hist + nR + 1 : nullptr);
  if (nR > 0) k_pcg_factor_red<<<(nR + PB - 1) / PB, PB, 0, st>>>(P);
  if (nB > 0) k_pcg_factor_black<<<(nB + PB - 1) / PB, PB, 0, st>>>(P, negpiv);
  if (nR > 0) k_pcg_resid0<<<(nR + PB - 1) / PB, PB, 0, st>>>(P, 0);
  if (nB > 0) k_pcg_resid0<<<(nB + PB - 1) / PB, PB, 0, st>>>(P, 1);
  k_pcg_bnorm<<<(nR + nB + PB - 1) / PB, PB, 0, st>>>(P);
}

void pcg_iteration(const PcgDev& P, int par, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  const int gB = std::max((nB + PB * NPT - 1) / (PB * NPT), 1), gR = std::max((nR + PB * NPT - 1) / (PB * NPT), 1);
  k_pcg_black_solve<double><<<gB, PB, 0, st>>>(P, par);
  k_pcg_red_solve<double><<<gR, PB, 0, st>>>(P, par, gB);
  if (P.diag_stored) k_pcg_apply<double, true><<<gR + gB, PB, 0, st>>>(P, par, gR);
  else k_pcg_apply<double, false><<<gR + gB, PB, 0, st>>>(P, par, gR);
}

void pcg_iteration_f(const PcgDevF& F, int par, cudaStream_t st) {
  const int nR = F.R.n, nB = F.B.n;
  const int gB = std::max((nB + PB * NPT - 1) / (PB * NPT), 1), gR = std::max((nR + PB * NPT - 1) / (PB * NPT), 1);
  k_pcg_black_solve<float><<<gB, PB, 0, st>>>(F, par);
  k_pcg_red_solve<float><<<gR, PB, 0, st>>>(F, par, gB);
  k_pcg_apply<float, false><<<gR + gB, PB, 0, st>>>(F, par, gR);
}

__global__ void k_pcg_init(PcgScal* sc, PcgScal init) { *sc = init; }

// Per-solve statistics into device memory (iterations, NSPCG-style ier, stopping-test value), the
// same mapping the host applies after a synchronous solve.
__global__ void k_pcg_stats(const PcgScal* sc, int ier0, int* iters_ier, double* relres, int slot) {
  const PcgScal& S = *sc;
  int ier = ier0;
  if (S.negpiv & 2) ier = -12;
  else if (S.ier != 0) ier = S.ier;
  else if ((S.negpiv & 1) && ier == 0) ier = 5;
  iters_ier[2 * slot] = S.in;
  iters_ier[2 * slot + 1] = ier;
  relres[slot] = S.stptst;
}

void pcg_init_scalars(PcgScal* sc, const PcgScal& init, cudaStream_t st) { k_pcg_init<<<1, 1, 0, st>>>(sc, init); }

void pcg_record_stats(const PcgScal* sc, int ier0, int* iters_ier, double* relres, int slot, cudaStream_t st) {
  k_pcg_stats<<<1, 1, 0, st>>>(sc, ier0, iters_ier, relres, slot);
}

void pcg_finish(const Dev& d, const PcgDev& P, double* hist, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  if (nR > 0) k_pcg_scatter<<<(nR + PB - 1) / PB, PB, 0, st>>>(d, P, 0, hist);
  if (nB > 0) k_pcg_scatter<<<(nB + PB - 1) / PB, PB, 0, st>>>(d, P, 1, hist ? hist + nR + 1 : nullptr);
}

// ------------------------------------------------------------------ iterative refinement
// FP64 residual of the current FP64 iterate and ||r||^2 (into sc->stptst, fixed-order sum).
__global__ void k_ir_norm(PcgDev P) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nR = P.R.n, nB = P.B.n;
  double v = 0;
  if (i < nR) v = P.R.r[i] * P.R.r[i];
  else if (i < nR + nB) v = P.B.r[i - nR] * P.B.r[i - nR];
  const double bs = block_sum(v, sh);
  if (threadIdx.x == 0) P.part0[blockIdx.x] = bs;
  if (last_block(&P.sc->cnt[3])) {
    const double tot = reduce_partials(P.part0, gridDim.x, sh);
    if (threadIdx.x == 0) P.sc->stptst = tot;
  }
}

// Inner FP32 system for the correction e: A e = r with e0 = 0.  Coefficients and the FP64 MIC
// pivots are rounded to FP32; the inner stopping test (test 5 on the inner residual) uses
// bnorm = ||r||.
__global__ void k_ir_inner_setup(PcgDev P, PcgDevF F, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  const PcgColorT<float>& G = color ? F.B : F.R;
  if (i > C.n) return;
  G.sx[i] = (float)C.sx[i];
  G.sy[i] = (float)C.sy[i];
  G.dinv[i] = (float)C.dinv[i];
  G.r[i] = (float)C.r[i];
  G.u[i] = 0.f; G.z[i] = 0.f; G.p[i] = 0.f; G.p2[i] = 0.f; G.q[i] = 0.f;
}

// u += e in FP64 (the zeta update is kept in double precision).
__global__ void k_ir_correct(PcgDev P, PcgDevF F, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  const PcgColorT<float>& G = color ? F.B : F.R;
  if (i >= C.n) return;
  C.u[i] = C.u[i] + (double)G.u[i];
}

void ir_residual(const PcgDev& P, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  if (nR > 0) k_pcg_resid0<<<(nR + PB - 1) / PB, PB, 0, st>>>(P, 0);
  if (nB > 0) k_pcg_resid0<<<(nB + PB - 1) / PB, PB, 0, st>>>(P, 1);
  k_ir_norm<<<(nR + nB + PB - 1) / PB, PB, 0, st>>>(P);
}

void ir_inner_setup(const PcgDev& P, const PcgDevF& F, cudaStream_t st) {
  k_ir_inner_setup<<<(P.R.n + 1 + PB - 1) / PB, PB, 0, st>>>(P, F, 0);
  k_ir_inner_setup<<<(P.B.n + 1 + PB - 1) / PB, PB, 0, st>>>(P, F, 1);
}

void ir_correct(const PcgDev& P, const PcgDevF& F, cudaStream_t st) {
  if (P.R.n > 0) k_ir_correct<<<(P.R.n + PB - 1) / PB, PB, 0, st>>>(P, F, 0);
  if (P.B.n > 0) k_ir_correct<<<(P.B.n + PB - 1) / PB, PB, 0, st>>>(P, F, 1);
}

int pcg_max_blocks(int nR, int nB) {
  return (nR + PB - 1) / PB + (nB + PB - 1) / PB + 2;   // also covers the setup kernels' grids
}

}  // namespace si3d
