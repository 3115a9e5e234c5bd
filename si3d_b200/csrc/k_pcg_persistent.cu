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
// the test-5 loop free of the eigenvalue code.
template <typename T, bool TEST2>
__global__ void __launch_bounds__(PQB, 1) k_pcg_loop(PcgDevT<T> P, GridBar* bar) {
  __shared__ double sh[(PQB / 32) * 4 + 4];
  __shared__ BarSt s_flag;
  if (threadIdx.x == 0) s_flag.epoch = 0;
  const PcgColorT<T> &R = P.R, &B = P.B;
  PcgScal* SC = P.sc;
  const int nb = gridDim.x;
  const int stride = nb * PQB;
  const int g0 = blockIdx.x * PQB + threadIdx.x;
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
        for (int i = 0; i < 4; ++i) P.part0[i * pstride + blockIdx.x] = v[i];
    } else {
      double w2[2] = {v[0], v[1]};
      bsum<2, PQB>(w2, sh);
      if (threadIdx.x == 0) { P.part0[blockIdx.x] = w2[0]; P.part0[pstride + blockIdx.x] = w2[1]; }
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
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
        for (int i = 0; i < 4; ++i) P.part0[i * pstride + nb + blockIdx.x] = v[i];
    } else {
      double w2[2] = {v[0], v[1]};
      bsum<2, PQB>(w2, sh);
      if (threadIdx.x == 0) { P.part0[nb + blockIdx.x] = w2[0]; P.part0[pstride + nb + blockIdx.x] = w2[1]; }
    }
    if (!grid_barrier(bar, SC, &s_flag)) return;
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
        const T diag = (T)1 + C.sx[i] + sxW + C.sy[i] + syS;
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
    if (threadIdx.x == 0) pq_part[blockIdx.x] = pq[0];
    if (!grid_barrier(bar, SC, &s_flag)) return;
    double pap[1];
    all_partials<1, PQB>(pq_part, nb, 0, pap, sh);
    const double alpha_prev = alpha;
    alpha = rzdot / pap[0];
    if (!(pap[0] > 0.0)) { ier = -6; break; }
    if (blockIdx.x == 0 && threadIdx.x == 0 && in < hist_cap) { P.hist_alpha[in] = alpha; P.hist_beta[in] = beta; }
    if (TEST2 && blockIdx.x == 0 && threadIdx.x == 0 && P.tri && (SC->maxadp || SC->minadp))
      lz_chgcon(SC, P.tri, in, alpha, beta, alpha_prev);
    in += 1;
    par ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SC->alpha = alpha; SC->beta = beta; SC->rzdot = rzdot; SC->dkm1 = dkm1; SC->udnm = udnm; SC->q1 = q1;
    SC->in = in; SC->stptst = stptst;
    if (ier) SC->ier = ier;
    else if (SC->chg_ier) SC->ier = SC->chg_ier;
    SC->done = 1;
  }
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
  const cudaError_t e = test2 ? cudaLaunchKernelEx(&cfg, k_pcg_loop<T, true>, P, bar)
                              : cudaLaunchKernelEx(&cfg, k_pcg_loop<T, false>, P, bar);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace

int pcg_loop_blocks(int device, int nR, int nB, int max_per_sm, bool fp32) {
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int occ2 = 0;
  if (fp32) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_loop<float, false>, PQB, 0);
    occ2 = occ;
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_loop<double, false>, PQB, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_pcg_loop<double, true>, PQB, 0);
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

int pcg_loop_f(const PcgDevF& F, GridBar* bar, int nblocks, cudaStream_t st, const GridBar* init) {
  return launch_loop<float>(F, bar, nblocks, false, st, init);
}

}  // namespace si3d
