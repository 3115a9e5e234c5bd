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
#include "common.cuh"
#include "kernels.h"

namespace si3d {

// ------------------------------------------------------------------ matcon
__global__ void k_matcon(Dev d) {
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
  double sum = 0;
  for (int k = d.g.k1; k <= kms; ++k)
    sum += (d.f.uhpp[IX(d, k, l)] - d.f.uhpp[IX(d, k, lW)]) / d.p.dx +
           (d.f.vhpp[IX(d, k, l)] - d.f.vhpp[IX(d, k, lS)]) / d.p.dy;
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
__global__ void k_pcg_gather(Dev d, PcgDev P, int color, int x0_mode, const double* __restrict__ dz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i > C.n) return;
  if (i == C.n) {  // the permanent zero slot
    C.sx[i] = 0.0; C.sy[i] = 0.0; C.u[i] = 0.0; C.r[i] = 0.0; C.z[i] = 0.0; C.p[i] = 0.0; C.q[i] = 0.0;
    C.rhs[i] = 0.0; C.dinv[i] = 0.0;
    return;
  }
  const int l = C.l[i];
  C.sx[i] = d.s.sx[l - 1];
  C.sy[i] = d.s.sy[l - 1];
  C.rhs[i] = d.s.qq[l - 1];
  double x0 = (x0_mode == 1) ? 0.0 : d.s.sp[l - 1];
  if (x0_mode == 2 && dz) x0 = x0 + dz[l - 1];
  C.u[i] = x0;
  C.z[i] = 0.0; C.p[i] = 0.0; C.q[i] = 0.0;
}

// Red pivots are the diagonal itself (no lower neighbours in red-black order).
__global__ void k_pcg_factor_red(PcgDev P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  if (i >= R.n) return;
  const int4 nb = R.nbr[i];
  const double diag = 1 + R.sx[i] + B.sx[nb.x] + R.sy[i] + B.sy[nb.y];
  R.dinv[i] = 1.0 / diag;
  // row sum of the upper triangle T (icfp wksp, nspcg.f:20786-20789), columns W, S, N, E
  const double tW = -B.sx[nb.x], tS = -B.sy[nb.y], tN = -R.sy[i], tE = -R.sx[i];
  R.diag[i] = diag;
  R.rs[i] = (((0.0 + tW) + tS) + tN) + tE;
}

// Black pivots: d(j) -= t(k,j)/d(k) * (omega*rowsum_T(k) - (omega-1)*t(k,j)) for every red
// neighbour k in increasing l order (W, S, N, E), omega = 1 (icfp, nspcg.f:20797-20806).
__global__ void k_pcg_factor_black(PcgDev P, int* __restrict__ negpiv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  if (j >= B.n) return;
  const int4 nb = B.nbr[j];
  double dj = 1 + B.sx[j] + R.sx[nb.x] + B.sy[j] + R.sy[nb.y];
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
  const double diag = 1 + C.sx[i] + O.sx[nb.x] + C.sy[i] + O.sy[nb.y];
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

// Black half of z = M^-1 r, fused with u += alpha p and r -= alpha q.
__global__ void __launch_bounds__(PB) k_pcg_black_solve(PcgDev P) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  const double alpha = P.sc->alpha;
  double rr = 0, rz = 0, uu = 0, zz = 0;
  if (j < B.n) {
    const int4 nb = B.nbr[j];
    const double uj = B.u[j] + alpha * B.p[j];
    const double rj = B.r[j] - alpha * B.q[j];
    B.u[j] = uj;
    B.r[j] = rj;
    // icfstp: the red rows scatter into this black row in l order W, S, N, E
    const int ks[4] = {nb.x, nb.y, nb.z, nb.w};
    const double t[4] = {-R.sx[nb.x], -R.sy[nb.y], -B.sy[j], -B.sx[j]};
    double x = rj;
    for (int c = 0; c < 4; ++c) {
      const int k = ks[c];
      const double rk = R.r[k] - alpha * R.q[k];
      const double xfk = rk * R.dinv[k];
      x = x - t[c] * xfk;
    }
    const double dj = B.dinv[j];
    x = x * dj;          // icfstp: x(i) = x(i)*d(i)
    x = x / dj;          // icsp:   x(i) = x(i)/d(i)
    const double zj = x * dj;  // icbsp on a row with no upper entries
    B.z[j] = zj;
    rr = rj * rj; rz = rj * zj; uu = uj * uj; zz = zj * zj;
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
__global__ void __launch_bounds__(PB) k_pcg_red_solve(PcgDev P, int nblk_black) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  const double alpha = P.sc->alpha;
  double rr = 0, rz = 0, uu = 0, zz = 0;
  if (k < R.n) {
    const int4 nb = R.nbr[k];
    const double uk = R.u[k] + alpha * R.p[k];
    const double rk = R.r[k] - alpha * R.q[k];
    R.u[k] = uk;
    R.r[k] = rk;
    const double dk = R.dinv[k];
    double x = rk * dk;   // icfstp
    x = x / dk;           // icsp
    // icbsp: sum = x - t(k,W) z_W - t(k,S) z_S - t(k,N) z_N - t(k,E) z_E
    x = x - (-B.sx[nb.x]) * B.z[nb.x];
    x = x - (-B.sy[nb.y]) * B.z[nb.y];
    x = x - (-R.sy[k]) * B.z[nb.z];
    x = x - (-R.sx[k]) * B.z[nb.w];
    const double zk = x * dk;
    R.z[k] = zk;
    rr = rk * rk; rz = rk * zk; uu = uk * uk; zz = zk * zk;
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

// p = z + beta p and q = A p on the black nodes (red neighbours' new p formed on the fly).
__global__ void __launch_bounds__(PB) k_pcg_black_apply(PcgDev P) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  const double beta = P.sc->beta;
  double pq = 0;
  if (j < B.n) {
    const int4 nb = B.nbr[j];
    const double pj = B.z[j] + beta * B.p[j];
    const double pW = R.z[nb.x] + beta * R.p[nb.x];
    const double pS = R.z[nb.y] + beta * R.p[nb.y];
    const double pN = R.z[nb.z] + beta * R.p[nb.z];
    const double pE = R.z[nb.w] + beta * R.p[nb.w];
    const double sxW = R.sx[nb.x], syS = R.sy[nb.y];
    const double diag = 1 + B.sx[j] + sxW + B.sy[j] + syS;
    double y = diag * pj;
    y = y + (-sxW) * pW;
    y = y + (-syS) * pS;
    y = y + (-B.sy[j]) * pN;
    y = y + (-B.sx[j]) * pE;
    B.p[j] = pj;
    B.q[j] = y;
    pq = pj * y;
  }
  const double s = block_sum(pq, sh);
  if (threadIdx.x == 0) P.part0[blockIdx.x] = s;
}

// p = z + beta p and q = A p on the red nodes, then (p,q), alpha and the iteration count.
__global__ void __launch_bounds__(PB) k_pcg_red_apply(PcgDev P, int nblk_black) {
  __shared__ double sh[32];
  if (P.sc->done) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor &R = P.R, &B = P.B;
  const double beta = P.sc->beta;
  double pq = 0;
  if (k < R.n) {
    const int4 nb = R.nbr[k];
    const double pk = R.z[k] + beta * R.p[k];
    const double sxW = B.sx[nb.x], syS = B.sy[nb.y];
    const double diag = 1 + R.sx[k] + sxW + R.sy[k] + syS;
    double y = diag * pk;
    y = y + (-sxW) * B.p[nb.x];
    y = y + (-syS) * B.p[nb.y];
    y = y + (-R.sy[k]) * B.p[nb.z];
    y = y + (-R.sx[k]) * B.p[nb.w];
    R.p[k] = pk;
    R.q[k] = y;
    pq = pk * y;
  }
  const double s = block_sum(pq, sh);
  if (threadIdx.x == 0) P.part0[nblk_black + blockIdx.x] = s;
  if (!last_block(&P.sc->cnt[1])) return;
  const double pap = reduce_partials(P.part0, nblk_black + gridDim.x, sh);
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
__global__ void k_pcg_scatter(Dev d, PcgDev P, int color) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const PcgColor& C = color ? P.B : P.R;
  if (i >= C.n) return;
  d.s.s[C.l[i] - 1] = C.u[i];
}

void pcg_setup(const Dev& d, const PcgDev& P, int x0_mode, const double* dz, int* negpiv, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  k_pcg_gather<<<(nR + 1 + PB - 1) / PB, PB, 0, st>>>(d, P, 0, x0_mode, dz);
  k_pcg_gather<<<(nB + 1 + PB - 1) / PB, PB, 0, st>>>(d, P, 1, x0_mode, dz);
  if (nR > 0) k_pcg_factor_red<<<(nR + PB - 1) / PB, PB, 0, st>>>(P);
  if (nB > 0) k_pcg_factor_black<<<(nB + PB - 1) / PB, PB, 0, st>>>(P, negpiv);
  if (nR > 0) k_pcg_resid0<<<(nR + PB - 1) / PB, PB, 0, st>>>(P, 0);
  if (nB > 0) k_pcg_resid0<<<(nB + PB - 1) / PB, PB, 0, st>>>(P, 1);
  k_pcg_bnorm<<<(nR + nB + PB - 1) / PB, PB, 0, st>>>(P);
}

void pcg_iteration(const PcgDev& P, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  const int gB = (nB + PB - 1) / PB, gR = (nR + PB - 1) / PB;
  const int gBb = gB > 0 ? gB : 1, gRr = gR > 0 ? gR : 1;
  k_pcg_black_solve<<<gBb, PB, 0, st>>>(P);
  k_pcg_red_solve<<<gRr, PB, 0, st>>>(P, gBb);
  k_pcg_black_apply<<<gBb, PB, 0, st>>>(P);
  k_pcg_red_apply<<<gRr, PB, 0, st>>>(P, gBb);
}

void pcg_finish(const Dev& d, const PcgDev& P, cudaStream_t st) {
  const int nR = P.R.n, nB = P.B.n;
  if (nR > 0) k_pcg_scatter<<<(nR + PB - 1) / PB, PB, 0, st>>>(d, P, 0);
  if (nB > 0) k_pcg_scatter<<<(nB + PB - 1) / PB, PB, 0, st>>>(d, P, 1);
}

int pcg_max_blocks(int nR, int nB) {
  return (nR + PB - 1) / PB + (nB + PB - 1) / PB + 2;
}

}  // namespace si3d
