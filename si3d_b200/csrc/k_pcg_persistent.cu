// Whole CG solve in one cooperative launch.
//
// The arithmetic of an iteration is that of the three-kernel form in k_zeta.cu (black half of
// M^-1 fused with u += alpha p and r -= alpha q; red half; p = z + beta p and q = A p on both
// colours), node for node, but all iterations run inside one kernel whose blocks are co-resident
// (cudaLaunchCooperativeKernel guarantees it), separated by grid barriers.  That removes the
// launch gaps, the host round trips that poll for convergence and the single-block reduction
// tails.  After a barrier every block sums the block partials itself, in the same fixed order,
// so every block computes the same alpha, beta and stopping decision without another
// synchronisation; block 0 publishes the final scalars.
//
// Every barrier wait is bounded: after kSpinLimit polls a block records SI3D_ETIMEOUT as the
// solve's ier, raises the barrier's abort flag and returns; the other blocks see the flag at
// their next wait and return too, so the kernel always ends.
#include <algorithm>

#include "../../include/si3d_gpu.h"
#include "common.cuh"
#include "coop.cuh"
#include "kernels.h"

namespace si3d {

namespace {

using namespace coop;

constexpr int PQB = 1024;   // threads per block of the cooperative solve (one block per SM)

// ---- adaptive eigenvalue estimates for stopping test 2: chgcon (nspcg.f:16499-16620), eigvss
// (:17201-17240), zbrent (:32976-33160) and determ (:16926-16962), run by one thread after each new
// alpha.  tri holds the Lanczos tridiagonal column by column: tri[2 (c - 1)] = T(1, c), tri[2 (c - 1) + 1]
// = T(2, c).
__device__ double lz_determ(int n, const double* tri, double x) {
  auto T = [&](int r, int c) { return tri[(c - 1) * 2 + (r - 1)]; };
  const int nm1 = n - 1;
  double d2 = T(1, n) - x;
  double d1 = d2 * (T(1, nm1) - x) - T(2, n);
  if (n != 2) {
    for (int l = nm1; l >= 2; --l) {
      const double d3 = d2;
      d2 = d1;
      d1 = (T(1, l - 1) - x) * d2 - d3 * T(2, l);
    }
  }
  return d1;
}

// Brent's root search on the determinant, in zbrent's own step order.
__device__ void lz_zbrent(int n, const double* tri, double eps, int nsig, double& aa, double& bb, int maxfn, int& ier) {
  double a = aa, b = bb;
  const double t = pow(0.1, (double)nsig);
  int ic = 2;
  double fa = lz_determ(n, tri, a), fb = lz_determ(n, tri, b), fc = 0, c = 0, d = 0, e = 0, s = b;
  double p, q, r, rone, tol, rm, temp;
  if (fa * fb > 0.0) { ier = 4; aa = a; bb = b; return; }
  for (;;) {
    c = a; fc = fa; d = b - c; e = d;
    for (;;) {
      if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
      tol = t * fmax(fabs(b), 0.1);
      rm = (c - b) / 2.0;
      if (fabs(fb) <= eps || fabs(c - b) <= tol) { aa = c; bb = b; return; }
      if (ic >= maxfn) { ier = 3; aa = c; bb = b; return; }
      bool bisect = fabs(e) < tol || fabs(fa) <= fabs(fb);
      if (!bisect) {
        s = fb / fa;
        if (a == c) {
          p = (c - b) * s;
          q = 1.0 - s;
        } else {
          q = fa / fc;
          r = fb / fc;
          rone = r - 1.0;
          p = s * ((c - b) * q * (q - r) - (b - a) * rone);
          q = (q - 1.0) * rone * (s - 1.0);
        }
        if (p > 0.0) q = -q;
        if (p < 0.0) p = -p;
        s = e;
        e = d;
        if (p + p >= 3.0 * rm * q || p + p >= fabs(s * q)) bisect = true;
        else d = p / q;
      }
      if (bisect) { e = rm; d = e; }
      a = b;
      fa = fb;
      temp = d;
      if (fabs(temp) <= tol / 2.0) temp = copysign(tol / 2.0, rm);
      b = b + temp;
      s = b;
      fb = lz_determ(n, tri, s);
      ic = ic + 1;
      if (!(fb * fc <= 0.0)) break;   // root no longer bracketed by (b, c): restart from (a, b)
    }
  }
}

__device__ double lz_eigvss(const double* tri, int n, double start, double end, int icode, double zeta, int itmax,
                            int& ier) {
  const int itmp = (int)(-log10(fabs(zeta)));
  const int nsig = itmp > 4 ? itmp : 4;
  const int maxfn = itmax > 50 ? itmax : 50;
  double a = start, b = end;
  lz_zbrent(n, tri, 0.0, nsig, a, b, maxfn, ier);
  return icode == 1 ? fmax(a, b) : fmin(a, b);
}

// chgcon after iteration ip (alpha: this iteration's, alphao: the previous one's, beta: this
// iteration's).  Updates S->emin/emax, the adaptivity flags and the bounds; sets S->chg_ier to 3/4
// when the root search stops as zbrent's do.
__device__ __noinline__ void lz_chgcon(PcgScal* S, double* tri, int ip, double alpha, double beta, double alphao) {
  auto T = [&](int r, int c) -> double& { return tri[(c - 1) * 2 + (r - 1)]; };
  if (ip == 0) {
    const double end = 1.0 / alpha;
    T(1, 1) = end; T(2, 1) = 0.0;
    if (S->maxadp) S->emax = end;
    if (S->minadp) S->emin = end;
    return;
  }
  const double t1 = 1.0 / alpha + beta / alphao;
  const double t2 = beta / (alphao * alphao);
  const double tsqr = sqrt(t2);
  T(1, ip + 1) = t1; T(2, ip + 1) = t2;
  if (ip == 1) {
    S->tl1 = T(1, 1) + tsqr; S->tl2 = t1 + tsqr;
    S->bl1 = T(1, 1) - tsqr; S->bl2 = t1 - tsqr;
    const double t3 = T(1, 1) + t1;
    const double t4 = sqrt((t1 - T(1, 1)) * (t1 - T(1, 1)) + 4.0 * t2);
    if (S->maxadp) S->emax = (t3 + t4) / 2.0;
    if (S->minadp) S->emin = (t3 - t4) / 2.0;
    return;
  }
  int ier = S->chg_ier;
  if (S->maxadp) {
    S->tl1 = fmax(S->tl1, S->tl2 + tsqr);
    S->tl2 = t1 + tsqr;
    const double emaxo = S->emax;
    const double end = fmax(S->tl1, S->tl2);
    const double e1 = lz_eigvss(tri, ip + 1, emaxo, end, 2, S->zeta, S->itmax, ier);
    if (ier != 3 && ier != 4) {
      S->emax = e1;
      if (fabs(S->emax - emaxo) < S->emax * S->zeta) S->maxadp = 0;
    } else S->maxadp = 0;
  }
  if (S->minadp) {
    S->bl1 = fmin(S->bl1, S->bl2 - tsqr);
    S->bl2 = t1 - tsqr;
    const double start = fmax(0.0, fmin(S->bl1, S->bl2));
    const double emino = S->emin;
    const double e1 = lz_eigvss(tri, ip + 1, start, emino, 1, S->zeta, S->itmax, ier);
    if (ier != 3 && ier != 4) {
      S->emin = e1;
      if (fabs(S->emin - emino) < S->emin * S->zeta) S->minadp = 0;
    } else S->minadp = 0;
  }
  S->chg_ier = ier;
}

// TEST2: stopping test 2 with chgcon's adaptive emin (test 5 otherwise); a separate instantiation keeps
// the test-5 loop free of the eigenvalue code.  The loop of one system, run by the nb blocks that
// share the barrier record `bar`, this block being block `bid` of them.
template <typename T, bool TEST2, bool DIAG>
__device__ __forceinline__ void pcg_loop_body(const PcgDevT<T>& P, GridBar* bar, int bid, int nb) {
  __shared__ double sh[(PQB / 32) * 4 + 4];
  __shared__ BarSt s_flag;
  if (threadIdx.x == 0) s_flag.epoch = 0;
  const PcgColorT<T> &R = P.R, &B = P.B;
  PcgScal* SC = P.sc;
  const int stride = nb * PQB;
  const int g0 = bid * PQB + threadIdx.x;
  // partial sums: (r,r) in part0, (r,z) in part1, (u,u) in part2, (z,z) in part3, black blocks at
  // [0, nb) and red blocks at [nb, 2 nb); (p,q) at part0 + 2 nb.  The four arrays are equally
  // spaced (part_n apart in one allocation).
  double* const pq_part = P.part0 + 2 * nb;
  const int pstride = P.part_n;
  // private copies of the CG scalars, identical in every block
  double alpha = SC->alpha, beta = SC->beta, rzdot = SC->rzdot, dkm1 = SC->dkm1, udnm = SC->udnm;
  const double zeta = SC->zeta, srelpr = SC->srelpr, bnorm = SC->bnorm, emin = SC->emin;
  int in = SC->in, q1 = SC->q1, ier = 0, par = 0;
  const int itmax = SC->itmax, hist_cap = SC->hist_cap;
  double stptst = SC->stptst;
  const bool t2 = TEST2;
  bool run = SC->done == 0;
  while (run) {
    const T* __restrict__ Bp = par ? B.p2 : B.p;
    const T* __restrict__ Rp = par ? R.p2 : R.p;
    const T a = (T)alpha;
    // ---- black nodes: u += alpha p, r -= alpha q, black half of M^-1 (icfstp/icsp/icbsp)
    // (neighbour indices are loaded one node ahead and every store follows all of a node's loads,
    // so a node costs one memory round trip)
    double v[4] = {0, 0, 0, 0};
    int4 q4n = (g0 < B.n) ? B.nbr[g0] : make_int4(0, 0, 0, 0);
    for (int j = g0; j < B.n; j += stride) {
      const int4 q4 = q4n;
      if (j + stride < B.n) q4n = B.nbr[j + stride];
      const T uj = B.u[j] + a * Bp[j];
      const T rj = B.r[j] - a * B.q[j];
      const int ks[4] = {q4.x, q4.y, q4.z, q4.w};
      const T t[4] = {-R.sx[q4.x], -R.sy[q4.y], -B.sy[j], -B.sx[j]};
      T x = rj;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int k = ks[c];
        const T rk = R.r[k] - a * R.q[k];
        const T xfk = rk * R.dinv[k];
        x = x - t[c] * xfk;
      }
      const T dj = B.dinv[j];
      x = x * dj;
      x = x / dj;
      const T zj = x * dj;
      B.u[j] = uj;
      B.r[j] = rj;
      B.z[j] = zj;
      v[0] += (double)rj * (double)rj; v[1] += (double)rj * (double)zj;
      v[2] += (double)uj * (double)uj; v[3] += (double)zj * (double)zj;
    }
    if (t2) {
      bsum<4, PQB>(v, sh);
      if (threadIdx.x == 0)
        for (int i = 0; i < 4; ++i) P.part0[i * pstride + bid] = v[i];
    } else {
      double w2[2] = {v[0], v[1]};
      bsum<2, PQB>(w2, sh);
      if (threadIdx.x == 0) { P.part0[bid] = w2[0]; P.part0[pstride + bid] = w2[1]; }
    }
    if (!grid_barrier(bar, SC, &s_flag, nb)) return;
    // ---- red nodes: u/r updates, red half of M^-1
    v[0] = v[1] = v[2] = v[3] = 0;
    q4n = (g0 < R.n) ? R.nbr[g0] : make_int4(0, 0, 0, 0);
    for (int k = g0; k < R.n; k += stride) {
      const int4 q4 = q4n;
      if (k + stride < R.n) q4n = R.nbr[k + stride];
      const T uk = R.u[k] + a * Rp[k];
      const T rk = R.r[k] - a * R.q[k];
      const T dk = R.dinv[k];
      T x = rk * dk;
      x = x / dk;
      x = x - (-B.sx[q4.x]) * B.z[q4.x];
      x = x - (-B.sy[q4.y]) * B.z[q4.y];
      x = x - (-R.sy[k]) * B.z[q4.z];
      x = x - (-R.sx[k]) * B.z[q4.w];
      const T zk = x * dk;
      R.u[k] = uk;
      R.r[k] = rk;
      R.z[k] = zk;
      v[0] += (double)rk * (double)rk; v[1] += (double)rk * (double)zk;
      v[2] += (double)uk * (double)uk; v[3] += (double)zk * (double)zk;
    }
    if (t2) {
      bsum<4, PQB>(v, sh);
      if (threadIdx.x == 0)
        for (int i = 0; i < 4; ++i) P.part0[i * pstride + nb + bid] = v[i];
    } else {
      double w2[2] = {v[0], v[1]};
      bsum<2, PQB>(w2, sh);
      if (threadIdx.x == 0) { P.part0[nb + bid] = w2[0]; P.part0[pstride + nb + bid] = w2[1]; }
    }
    if (!grid_barrier(bar, SC, &s_flag, nb)) return;
    // ---- every block: (r,r), (r,z) [, (u,u), (z,z)], the stopping test (pstops) and beta
    double rrt, rzt, uut = 0, zzt = 0;
    if (t2) {
      double w4[4];
      all_partials<4, PQB>(P.part0, 2 * nb, pstride, w4, sh);
      rrt = w4[0]; rzt = w4[1]; uut = w4[2]; zzt = w4[3];
    } else {
      double w2[2];
      all_partials<2, PQB>(P.part0, 2 * nb, pstride, w2, sh);
      rrt = w2[0]; rzt = w2[1];
    }
    dkm1 = rzdot;
    rzdot = rzt;
    if (!(rzt > 0.0)) { ier = -7; break; }
    const double tiny = 500.0 * srelpr;
    bool halt;
    if (!TEST2) {
      const double tl = sqrt(rrt);
      stptst = tl / bnorm;
      halt = tl < bnorm * zeta;
    } else {
      if (in < 1) {
        q1 = 0;
        udnm = 1.0;
        stptst = sqrt(rzt);
        halt = stptst < tiny;
      } else {
        if (!q1 && !((in > 5) && (in % 5 != 0))) {
          const double uold = udnm;
          udnm = sqrt(uut);
          if (udnm < tiny) udnm = 1.0;
          if ((in > 5) && (fabs(udnm - uold) < udnm * zeta)) q1 = 1;
        }
        const double em = __ldcg(&SC->emin);   // chgcon's latest estimate (block 0, before the last barrier)
        const double eminl = em < tiny ? tiny : em;
        const double tl = sqrt(zzt), tr = udnm * eminl;
        stptst = tl / tr;
        halt = tl < tr * zeta;
      }
    }
    if (halt) break;
    if (!(in < itmax)) { ier = 1; break; }
    if (in != 0) beta = rzdot / dkm1;
    // ---- p = z + beta p and q = A p on both colours (the new p goes to the other buffer)
    const T bt = (T)beta;
    double pq[1] = {0};
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const PcgColorT<T>& C = side ? B : R;
      const PcgColorT<T>& O = side ? R : B;
      const T* __restrict__ Cp = par ? C.p2 : C.p;
      const T* __restrict__ Op = par ? O.p2 : O.p;
      T* __restrict__ Cn = par ? C.p : C.p2;
      int4 q4n3 = (g0 < C.n) ? C.nbr[g0] : make_int4(0, 0, 0, 0);
      for (int i = g0; i < C.n; i += stride) {
        const int4 q4 = q4n3;
        if (i + stride < C.n) q4n3 = C.nbr[i + stride];
        const T pi = C.z[i] + bt * Cp[i];
        const T pW = O.z[q4.x] + bt * Op[q4.x];
        const T pS = O.z[q4.y] + bt * Op[q4.y];
        const T pN = O.z[q4.z] + bt * Op[q4.z];
        const T pE = O.z[q4.w] + bt * Op[q4.w];
        const T sxW = O.sx[q4.x], syS = O.sy[q4.y];
        const T diag = DIAG ? C.diag[i] : (T)1 + C.sx[i] + sxW + C.sy[i] + syS;
        T y = diag * pi;
        y = y + (-sxW) * pW;
        y = y + (-syS) * pS;
        y = y + (-C.sy[i]) * pN;
        y = y + (-C.sx[i]) * pE;
        Cn[i] = pi;
        C.q[i] = y;
        pq[0] += (double)pi * (double)y;
      }
    }
    bsum<1, PQB>(pq, sh);
    if (threadIdx.x == 0) pq_part[bid] = pq[0];
    if (!grid_barrier(bar, SC, &s_flag, nb)) return;
    double pap[1];
    all_partials<1, PQB>(pq_part, nb, 0, pap, sh);
    const double alpha_prev = alpha;
    alpha = rzdot / pap[0];
    if (!(pap[0] > 0.0)) { ier = -6; break; }
    if (bid == 0 && threadIdx.x == 0 && in < hist_cap) { P.hist_alpha[in] = alpha; P.hist_beta[in] = beta; }
    if (TEST2 && bid == 0 && threadIdx.x == 0 && P.tri && (SC->maxadp || SC->minadp))
      lz_chgcon(SC, P.tri, in, alpha, beta, alpha_prev);
    in += 1;
    par ^= 1;
  }
  if (bid == 0 && threadIdx.x == 0) {
    SC->alpha = alpha; SC->beta = beta; SC->rzdot = rzdot; SC->dkm1 = dkm1; SC->udnm = udnm; SC->q1 = q1;
    SC->in = in; SC->stptst = stptst;
    if (ier) SC->ier = ier;
    else if (SC->chg_ier) SC->ier = SC->chg_ier;
    SC->done = 1;
  }
}

template <typename T, bool TEST2, bool DIAG>
__global__ void __launch_bounds__(PQB, 1) k_pcg_loop(PcgDevT<T> P, GridBar* bar) {
  pcg_loop_body<T, TEST2, DIAG>(P, bar, blockIdx.x, gridDim.x);
}

// The FP64 loops of an ensemble's basins in one cooperative launch: basin m's system is solved by
// blocks [first, first + nblk) of the grid with its own barrier record, so each basin iterates to
// its own convergence and the launch ends when the last one has (stopping test 5, no stored
// diagonal: the basins the ensemble form admits).
__global__ void __launch_bounds__(PQB, 1) k_pcg_loop_ens(const PcgEnsItem* __restrict__ items, int nitems) {
  __shared__ PcgEnsItem s_it;
  __shared__ int s_m;
  if (threadIdx.x == 0) {
    int m = -1;
    for (int i = 0; i < nitems && m < 0; ++i)
      if ((int)blockIdx.x >= items[i].first && (int)blockIdx.x < items[i].first + items[i].nblk) m = i;
    s_m = m;
    if (m >= 0) s_it = items[m];
  }
  __syncthreads();
  if (s_m < 0) return;
  pcg_loop_body<double, false, false>(s_it.P, s_it.bar, (int)blockIdx.x - s_it.first, s_it.nblk);
}

// Cooperative launch (all blocks co-resident) through cudaLaunchKernelEx, which stream capture
// records as a cooperative kernel node.
template <typename T>
int launch_loop(const PcgDevT<T>& P, GridBar* bar, int nblocks, bool test2, cudaStream_t st, const GridBar* init) {
  if (init) {
    if (cudaMemcpyAsync(bar, init, sizeof(GridBar), cudaMemcpyHostToDevice, st) != cudaSuccess) return -1;
  } else if (cudaMemsetAsync(bar, 0, sizeof(GridBar), st) != cudaSuccess) {
    return -1;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(PQB);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e;
  if (P.diag_stored) e = test2 ? cudaLaunchKernelEx(&cfg, k_pcg_loop<T, true, true>, P, bar)
                               : cudaLaunchKernelEx(&cfg, k_pcg_loop<T, false, true>, P, bar);
  else e = test2 ? cudaLaunchKernelEx(&cfg, k_pcg_loop<T, true, false>, P, bar)
                 : cudaLaunchKernelEx(&cfg, k_pcg_loop<T, false, false>, P, bar);
  return e == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------- natural-order MIC-CG
// One block runs the whole solve of the reference's own ordering (nspcg.f: icfp :20724-20850 with
// property A, icsp/icfstp/icbsp :21759-21805, :22875-22922, :22729-22777, mult1 :23919-23947, itcg
// :8967-9092, pstops :25956-26100), row by row in the operation order of those routines.  The
// sweeps' recurrences along l run level by level (a level's rows in parallel, a block barrier
// between levels); dot products are block sums in a fixed order.
constexpr int NQB = 1024;

__device__ __forceinline__ double nat_coef(const NatDev& N, int i, int code) {
  switch (code) {
    case 0: return N.cW[i];
    case 1: return N.cS[i];
    case 2: return N.cN[i];
    case 3: return N.cE[i];
    default: return 0.0;   // an absent neighbour: adjust made it the row itself with coefficient 0
  }
}
__device__ __forceinline__ int nat_col(const int4& nb, int i, int code) {
  switch (code) {
    case 0: return nb.x;
    case 1: return nb.y;
    case 2: return nb.z;
    case 3: return nb.w;
    default: return i;
  }
}

// (A x)_i in mult1's order: the diagonal, then the off-diagonal columns as move1 left them.
__device__ __forceinline__ double nat_row_apply(const NatDev& N, const double* x, int i) {
  const int4 nb = N.nbr[i];
  const int ord = N.order[i];
  double y = N.cd[i] * x[i];
#pragma unroll
  for (int sl = 0; sl < 4; ++sl) {
    const int c = (ord >> (3 * sl)) & 7;
    y = y + nat_coef(N, i, c) * x[nat_col(nb, i, c)];
  }
  return y;
}

// Lower neighbours of row i in ascending row order (the order in which their pushes reach row i
// in icfp and icfstp), with their codes; returns how many.
__device__ __forceinline__ int nat_lower(const NatDev& N, int i, int4 nb, int (&rows)[4], int (&codes)[4]) {
  const int cand[4] = {nb.x, nb.y, nb.z, nb.w};
  int m = 0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (cand[c] < i) {   // absent neighbours are n > i
      int j = m++;
      while (j > 0 && rows[j - 1] > cand[c]) { rows[j] = rows[j - 1]; codes[j] = codes[j - 1]; --j; }
      rows[j] = cand[c];
      codes[j] = c;
    }
  }
  return m;
}

template <bool TEST2>
__global__ void __launch_bounds__(NQB, 1) k_pcg_natural(NatDev N) {
  __shared__ double sh[(NQB / 32) * 3 + 3];
  PcgScal* SC = N.sc;
  const int n = N.n, tid = threadIdx.x;
  // ---- icfp: MIC pivots, property A, omega = 1 (a row's pivot after its lower neighbours')
  for (int L = 0; L < N.nlev; ++L) {
    for (int q = N.lvl_off[L] + tid; q < N.lvl_off[L + 1]; q += NQB) {
      const int i = N.lvl_row[q];
      int rows[4], codes[4];
      const int m = nat_lower(N, i, N.nbr[i], rows, codes);
      double dd = N.cd[i];
      for (int t = 0; t < m; ++t) {
        const int k = rows[t];
        const int ok = N.order[k];
        double wk = 0.0;   // row sum of k's upper columns (icfp's wksp)
        for (int sl = 0; sl < N.nt; ++sl) wk = wk + nat_coef(N, k, (ok >> (3 * sl)) & 7);
        const double c = nat_coef(N, i, codes[t]);   // = A(k, i) (the matrix is symmetric)
        const double term = c / N.piv[k];
        dd = dd - term * (1.0 * wk - (1.0 - 1.0) * c);
      }
      N.piv[i] = dd;
    }
    __syncthreads();
  }
  int zero = 0, neg = 0;
  for (int i = tid; i < n; i += NQB) {
    const double pv = N.piv[i];
    if (pv == 0.0) zero = 1;
    const double di = 1.0 / pv;
    N.dinv[i] = di;
    if (di < 0.0) neg = 1;
  }
  zero = __syncthreads_or(zero);
  neg = __syncthreads_or(neg);
  if (zero) {
    if (tid == 0) { SC->negpiv = 2; SC->in = 0; SC->done = 1; }
    return;
  }
  // ---- cgw: r = b - A u, ||b|| (nmcalc)
  {
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = tid; i < n; i += NQB) {
      N.r[i] = N.b[i] - nat_row_apply(N, N.u, i);
      v[0] += N.b[i] * N.b[i];
    }
    bsum<3, NQB>(v, sh);
    if (tid == 0) SC->bnorm = fmax(sqrt(v[0]), SC->srelpr);
  }
  __syncthreads();
  const double zeta = SC->zeta, srelpr = SC->srelpr, bnorm = SC->bnorm, tiny = 500.0 * srelpr;
  const int itmax = SC->itmax, hist_cap = SC->hist_cap;
  double alpha = 0.0, beta = 0.0, alphao = 0.0, rzdot = 0.0, dkm1 = 0.0, udnm = 1.0, stptst = 0.0;
  bool q1 = false;
  int in = 0, ier = 0;
  bool first = true;
  for (;;) {
    if (!first)
      for (int i = tid; i < n; i += NQB) N.r[i] = N.r[i] - alpha * N.q[i];
    first = false;
    __syncthreads();
    // ---- z = M^-1 r (icsp): forward sweep level by level, z /= d, backward sweep in reverse
    for (int L = 0; L < N.nlev; ++L) {
      for (int q = N.lvl_off[L] + tid; q < N.lvl_off[L + 1]; q += NQB) {
        const int i = N.lvl_row[q];
        int rows[4], codes[4];
        const int m = nat_lower(N, i, N.nbr[i], rows, codes);
        double t = N.r[i];
        for (int j = 0; j < m; ++j) t = t - nat_coef(N, i, codes[j]) * N.z[rows[j]];
        N.z[i] = t * N.dinv[i];
      }
      __syncthreads();
    }
    for (int i = tid; i < n; i += NQB) N.z[i] = N.z[i] / N.dinv[i];
    __syncthreads();
    for (int L = N.nlev - 1; L >= 0; --L) {
      for (int q = N.lvl_off[L] + tid; q < N.lvl_off[L + 1]; q += NQB) {
        const int i = N.lvl_row[q];
        const int4 nb = N.nbr[i];
        const int ord = N.order[i];
        double sum = N.z[i];
        for (int sl = 0; sl < N.nt; ++sl) {
          const int c = (ord >> (3 * sl)) & 7;
          sum = sum - nat_coef(N, i, c) * N.z[nat_col(nb, i, c)];
        }
        N.z[i] = sum * N.dinv[i];
      }
      __syncthreads();
    }
    // ---- (r, z); pstops
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = tid; i < n; i += NQB) {
      const double ri = N.r[i], zi = N.z[i];
      v[0] += ri * zi;
      v[1] += ri * ri;
      v[2] += zi * zi;
    }
    bsum<3, NQB>(v, sh);
    dkm1 = rzdot;
    rzdot = v[0];
    if (!(rzdot > 0.0)) { ier = -7; break; }
    bool halt = false;
    if (TEST2) {
      if (in < 1) {
        q1 = false;
        udnm = 1.0;
        stptst = sqrt(rzdot);
        if (stptst < tiny) halt = true;
      } else {
        if (!q1 && !((in > 5) && (in % 5 != 0))) {
          const double uold = udnm;
          double w[1] = {0.0};
          for (int i = tid; i < n; i += NQB) w[0] += N.u[i] * N.u[i];
          bsum<1, NQB>(w, sh);
          udnm = sqrt(w[0]);
          if (udnm < tiny) udnm = 1.0;
          if ((in > 5) && (fabs(udnm - uold) < udnm * zeta)) q1 = true;
        }
        double eminl = __ldcg(&SC->emin);   // chgcon's latest estimate (written by thread 0)
        if (eminl < tiny) eminl = tiny;
        const double tl = sqrt(v[2]), tr = udnm * eminl;
        stptst = tl / tr;
        if (tl < tr * zeta) halt = true;
      }
    } else {
      const double tl = sqrt(v[1]);
      stptst = tl / bnorm;
      if (tl < bnorm * zeta) halt = true;
    }
    if (halt) break;
    if (!(in < itmax)) { ier = 1; break; }
    if (in != 0) beta = rzdot / dkm1;
    for (int i = tid; i < n; i += NQB) N.p[i] = N.z[i] + beta * N.p[i];
    __syncthreads();
    double w[1] = {0.0};
    for (int i = tid; i < n; i += NQB) {
      const double qi = nat_row_apply(N, N.p, i);
      N.q[i] = qi;
      w[0] += N.p[i] * qi;
    }
    bsum<1, NQB>(w, sh);
    alphao = alpha;
    alpha = rzdot / w[0];
    if (!(w[0] > 0.0)) { ier = -6; break; }
    if (tid == 0 && in < hist_cap) { N.hist_alpha[in] = alpha; N.hist_beta[in] = beta; }
    if (TEST2) {
      if (tid == 0 && (SC->maxadp || SC->minadp)) lz_chgcon(SC, N.tri, in, alpha, beta, alphao);
      __syncthreads();
    }
    for (int i = tid; i < n; i += NQB) N.u[i] = N.u[i] + alpha * N.p[i];
    ++in;
  }
  if (tid == 0) {
    SC->alpha = alpha; SC->beta = beta; SC->rzdot = rzdot; SC->udnm = udnm; SC->in = in; SC->stptst = stptst;
    if (ier) SC->ier = ier;
    else if (SC->chg_ier) SC->ier = SC->chg_ier;
    SC->negpiv = neg ? 1 : 0;
    SC->done = 1;
  }
}

// Rows of the natural system from matcon's sx, sy, qq, as SolverSparse assembles coeffA
// (si3d_procedures.f90:1950-1967), and the initial guess (x0 modes of the red-black gather).
__global__ void k_nat_gather(Dev d, NatDev N, int x0_mode, const double* __restrict__ dz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > N.n) return;
  if (i == N.n) {   // the zero slot of absent neighbours
    N.u[i] = N.r[i] = N.z[i] = N.p[i] = N.q[i] = N.b[i] = 0.0;
    N.cd[i] = N.cW[i] = N.cS[i] = N.cN[i] = N.cE[i] = 0.0;
    return;
  }
  const int l = i + 1, lm1 = d.g.lm1;
  const int lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l), lN = NB(d.g.lNC, l), lE = NB(d.g.lEC, l);
  const double sxi = d.s.sx[l - 1], syi = d.s.sy[l - 1];
  const double sxW = lW != lm1 ? d.s.sx[lW - 1] : 0.0, syS = lS != lm1 ? d.s.sy[lS - 1] : 0.0;
  N.cd[i] = d.s.rr[l - 1];   // 1 + sx + sx(W) + sy + sy(S), formed before open boundaries cut faces
  N.cW[i] = lW != lm1 ? -sxW : 0.0;
  N.cS[i] = lS != lm1 ? -syS : 0.0;
  N.cN[i] = lN != lm1 ? -syi : 0.0;
  N.cE[i] = lE != lm1 ? -sxi : 0.0;
  N.b[i] = d.s.qq[l - 1];
  double x0;
  switch (x0_mode) {
    case 1: x0 = 0.0; break;
    case 3: x0 = d.s.s[l - 1]; break;
    default: x0 = d.s.sp[l - 1]; if (x0_mode == 2 && dz) x0 = x0 + dz[l - 1];
  }
  N.u[i] = x0;
  N.z[i] = 0.0; N.p[i] = 0.0; N.q[i] = 0.0;
}

__global__ void k_nat_scatter(Dev d, NatDev N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N.n) return;
  d.s.s[i] = N.u[i];
}

}  // namespace

int pcg_loop_blocks(int device, int nR, int nB, int max_per_sm, bool fp32) {
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int occ2 = 0;
  if (fp32) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_loop<float, false, false>, PQB, 0);
    occ2 = occ;
  } else {
    int occ3 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_loop<double, false, false>, PQB, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_pcg_loop<double, true, true>, PQB, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k_pcg_loop<double, true, false>, PQB, 0);
    occ2 = std::min(occ2, occ3);
  }
  occ = std::min(occ, occ2);
  int per_sm = occ;
  if (max_per_sm > 0) per_sm = std::min(per_sm, max_per_sm);
  const int need = (std::max(nR, nB) + PQB - 1) / PQB;
  return std::max(1, std::min(sms * std::max(per_sm, 1), need));
}

int pcg_loop(const PcgDev& P, GridBar* bar, int nblocks, bool test2, cudaStream_t st, const GridBar* init) {
  return launch_loop<double>(P, bar, nblocks, test2, st, init);
}

int pcg_loop_ens_blocks(int device) {
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_loop_ens, PQB, 0);
  return sms * std::max(occ, 0);
}

int pcg_loop_ens(const PcgEnsItem* items, int nitems, int nblocks, GridBar* bars, cudaStream_t st) {
  if (cudaMemsetAsync(bars, 0, sizeof(GridBar) * (size_t)nitems, st) != cudaSuccess) return -1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(PQB);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_pcg_loop_ens, items, nitems) == cudaSuccess ? 0 : -1;
}

int pcg_loop_f(const PcgDevF& F, GridBar* bar, int nblocks, cudaStream_t st, const GridBar* init) {
  return launch_loop<float>(F, bar, nblocks, false, st, init);
}

}  // namespace si3d

namespace si3d {

void nat_setup(const Dev& d, const NatDev& N, int x0_mode, const double* dz, cudaStream_t st) {
  k_nat_gather<<<(N.n + 1 + 255) / 256, 256, 0, st>>>(d, N, x0_mode, dz);
}

int nat_solve(const NatDev& N, bool test2, cudaStream_t st) {
  if (test2) k_pcg_natural<true><<<1, NQB, 0, st>>>(N);
  else k_pcg_natural<false><<<1, NQB, 0, st>>>(N);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

void nat_finish(const Dev& d, const NatDev& N, cudaStream_t st) {
  k_nat_scatter<<<(N.n + 255) / 256, 256, 0, st>>>(d, N);
}

}  // namespace si3d
