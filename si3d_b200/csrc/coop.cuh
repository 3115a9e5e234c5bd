// Helpers of the cooperative (grid-barrier) kernels: block sums in a fixed order, every-block
// reduction of block partials, and a counting grid barrier with a bounded wait.
//
// Every barrier wait is bounded: after kSpinLimit polls (or the barrier record's own limit) a block
// records SI3D_ETIMEOUT as the solve's ier, raises the barrier's abort flag and returns false; the
// other blocks see the flag at their next wait and return too, so a kernel built on it always ends.
#pragma once
#include "../../include/si3d_gpu.h"
#include "kernels.h"

namespace si3d {
namespace coop {

constexpr int QB = 256;                       // threads per block
constexpr long long kSpinLimit = 1LL << 23;   // polls (an L2 round trip each) before a wait gives up: > 2 s

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Block-wide sums of NV values at once (fixed order) over blocks of BS threads; the totals are
// returned in v[] in every thread.  sh holds (BS / 32) * NV + NV doubles.
template <int NV, int BS = QB>
__device__ __forceinline__ void bsum(double (&v)[NV], double* sh) {
  constexpr int NW = BS / 32;
#pragma unroll
  for (int i = 0; i < NV; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) sh[i * NW + w] = v[i];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0;
#pragma unroll
    for (int q = 0; q < NW; ++q) t += sh[threadIdx.x * NW + q];
    sh[NW * NV + threadIdx.x] = t;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = sh[NW * NV + i];
  __syncthreads();
}

// Totals of NV partial arrays (n entries each, arrays `stride` apart), in every thread.
template <int NV, int BS = QB>
__device__ __forceinline__ void all_partials(const double* part, int n, int stride, double (&v)[NV], double* sh) {
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = 0;
  for (int j = threadIdx.x; j < n; j += BS) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] += __ldcg(part + i * stride + j);
  }
  bsum<NV, BS>(v, sh);
}

// Per-block state of the grid barrier, in shared memory: the outcome of the last wait, the
// number of barriers this block has passed, and, read at the first barrier of the launch, the
// arrivals a barrier waits for and the poll limit.  Zero `epoch` (thread 0) before the first
// barrier.
struct BarSt {
  int ok;
  unsigned int epoch;
  unsigned int expect;
  long long limit;
};

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid barrier on a monotonic arrival counter: barrier e (1, 2, ...) of the launch is passed once
// the counter reaches e * (nblocks + absent), nblocks being the blocks that share this barrier
// record (the whole grid, or one basin's share of an ensemble launch).  An arrival is one release-add (no round trip, no
// reset; the release orders the block's writes, which __syncthreads ordered before thread 0's
// arrival, ahead of it); the wait polls with acquire loads, which order the block's later reads
// after the other blocks' arrivals.  `absent` and `limit` (zero in every solve; a test sets them
// to make the wait run out) are read once, at the first barrier, so a barrier costs one release
// and the polls.  Bounded: returns false (in every thread of the block) once this block gave up
// or any block has.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, PcgScal* sc, BarSt* st, unsigned int nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (st->epoch == 0) {
      st->expect = nblocks + __ldcg(&bar->absent);
      const unsigned long long lim = __ldcg(&bar->limit);
      st->limit = lim ? (long long)lim : kSpinLimit;
    }
    int ok = 1;
    const unsigned long long target = (unsigned long long)(++st->epoch) * st->expect;
    const long long limit = st->limit;
    red_release_add(&bar->count, 1ull);
    long long spins = 0;
    while (ld_acquire64(&bar->count) < target) {
      if (++spins > limit || ((spins & 15) == 0 && ld_acquire(&bar->abort) != 0u)) { ok = 0; break; }
    }
    if (!ok && atomicExch(&bar->abort, 1u) == 0u) {
      sc->ier = SI3D_ETIMEOUT;
      sc->done = 1;
      __threadfence();
    }
    st->ok = ok;
  }
  __syncthreads();
  return st->ok != 0;
}

__device__ __forceinline__ bool grid_barrier(GridBar* bar, PcgScal* sc, BarSt* st) {
  return grid_barrier(bar, sc, st, gridDim.x);
}

}  // namespace coop
}  // namespace si3d
