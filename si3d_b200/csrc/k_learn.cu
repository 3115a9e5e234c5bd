// Learned initial guess for the zeta solve: network kernels (inference and training) and the
// solver-side feature / scatter / record kernels.  Network shape and parameter layout are fixed by
// include/si3d_learn.h.
//
// Channels-last images with a one-pixel halo.  The four 32 -> 32 forward convolutions run on the
// fifth-generation tensor cores (k_conv32_tc: TMA halo loads, tcgen05.mma into TMEM, a pipeline of
// producer, MMA and epilogue warps; see there).  The data gradient for training is an implicit GEMM
// on 8 x 16 pixel tiles with mma.sync m16n8k16 (M = 16 pixels of a tile row, N = 8 channels, K = 16
// channels of one tap; 9 taps x 2 channel halves = 18 K-steps) with tap-flipped, channel-transposed
// weights.  BF16 operands, FP32 accumulation.  The 4 -> 32 stem, the 32 -> 1 head and the weight
// gradients are small and run on the FP32 cores, accumulating in a fixed order.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/si3d_gpu.h"
#include "../../include/si3d_learn.h"
#include "common.cuh"
#include "learn.h"

namespace si3d {
namespace learn {

namespace {

using bf16 = __nv_bfloat16;

constexpr int C = SI3D_NET_C;
constexpr int TH = 8, TW = 16, TP = TH * TW;   // pixel tile
constexpr int HT = TH + 2, WT = TW + 2;        // tile with halo
constexpr int XS = 40;                         // shared-memory pixel stride of 32-channel tiles (bf16)
constexpr int OFF_STEM_B = 9 * 4 * C;
constexpr int OFF_BLK = OFF_STEM_B + C;
constexpr int BLK_SZ = 9 * C * C + C;
constexpr int OFF_HEAD_W = OFF_BLK + SI3D_NET_BLOCKS * BLK_SZ;
constexpr int OFF_HEAD_B = OFF_HEAD_W + 9 * C;
static_assert(OFF_HEAD_B + 1 == SI3D_NET_NPARAM, "parameter layout");
constexpr int WG_BLOCKS = 296;                 // weight-gradient partial sums (2 per SM)

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

struct TileIdx {
  int b, i0, j0;
};
__device__ __forceinline__ TileIdx tile_of(int t, int H, int W) {
  const int nj = (W + TW - 1) / TW, ni = (H + TH - 1) / TH;
  TileIdx r;
  r.b = t / (ni * nj);
  const int rem = t % (ni * nj);
  r.i0 = (rem / nj) * TH;
  r.j0 = (rem % nj) * TW;
  return r;
}

// ------------------------------------------------------------------ weights
// Block weights to the tensor-core layout [tap][n][k] (bf16): forward n = cout, k = cin;
// data gradient n = cin, k = cout with the tap mirrored.  Stem/head weights rounded to bf16 values.
__global__ void k_prep(const float* __restrict__ prm, bf16* __restrict__ wfwd, bf16* __restrict__ wbwd,
                       float* __restrict__ stem, float* __restrict__ head) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = SI3D_NET_BLOCKS * 9 * C * C;
  if (tid < nb) {
    const int blk = tid / (9 * C * C), r = tid % (9 * C * C);
    const int t = r / (C * C), n = (r / C) % C, k = r % C;
    const float* W = prm + OFF_BLK + blk * BLK_SZ;
    wfwd[tid] = __float2bfloat16_rn(W[(t * C + k) * C + n]);          // W[t][cin=k][cout=n]
    wbwd[tid] = __float2bfloat16_rn(W[((8 - t) * C + n) * C + k]);    // W[8-t][cin=n][cout=k]
  }
  if (tid < 9 * 4 * C) stem[tid] = bfr(prm[tid]);
  if (tid < C) stem[9 * 4 * C + tid] = prm[OFF_STEM_B + tid];
  if (tid < 9 * C) head[tid] = bfr(prm[OFF_HEAD_W + tid]);
  if (tid == 0) head[9 * C] = prm[OFF_HEAD_B];
}

// ------------------------------------------------------------------ stem: 4 -> 32, FP32 cores
// A block takes 8 rows x 32 pixels; thread (ti, tj) computes pixels tj and tj + 16 of row ti, so each
// weight it reads from shared memory serves two pixels, and a pixel's four input channels are one
// 16-byte read.  Per output channel the products are accumulated in the order tap, input channel,
// with the inputs rounded to BF16 first.
constexpr int ST_W = 2 * TW;                   // pixels per row of a stem tile
constexpr int ST_WT = ST_W + 2;                // with halo
__global__ void __launch_bounds__(TP) k_stem(const float* __restrict__ feat, const float* __restrict__ w, int H, int W,
                                             bf16* __restrict__ X, float* __restrict__ Y) {
  __shared__ __align__(16) float sF[HT * ST_WT * 4];
  __shared__ __align__(16) float sW[9 * 4 * C + C];
  const int b = blockIdx.z, i0 = blockIdx.y * TH, j0 = blockIdx.x * ST_W;
  for (int r = threadIdx.x; r < 9 * 4 * C + C; r += TP) sW[r] = w[r];
  for (int r = threadIdx.x; r < HT * ST_WT; r += TP) {
    const int gi = i0 + r / ST_WT - 1, gj = j0 + r % ST_WT - 1;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gi >= 0 && gi < H && gj >= 0 && gj < W) v = *reinterpret_cast<const float4*>(feat + (((size_t)b * H + gi) * W + gj) * 4);
    *reinterpret_cast<float4*>(&sF[r * 4]) = make_float4(bfr(v.x), bfr(v.y), bfr(v.z), bfr(v.w));
  }
  __syncthreads();
  const int ti = threadIdx.x / TW, tj = threadIdx.x % TW;
  float acc[2][C];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int co = 0; co < C; ++co) acc[h][co] = 0.f;
  for (int t = 0; t < 9; ++t) {
    const int pi = ti + t / 3, pj = tj + t % 3;   // halo coordinates of the tap's input
    const float4 va = *reinterpret_cast<const float4*>(&sF[(pi * ST_WT + pj) * 4]);
    const float4 vb = *reinterpret_cast<const float4*>(&sF[(pi * ST_WT + pj + TW) * 4]);
    const float xa[4] = {va.x, va.y, va.z, va.w}, xb[4] = {vb.x, vb.y, vb.z, vb.w};
#pragma unroll
    for (int ci = 0; ci < 4; ++ci) {
      const float4* w4 = reinterpret_cast<const float4*>(&sW[(t * 4 + ci) * C]);
#pragma unroll
      for (int q = 0; q < C / 4; ++q) {
        const float4 wq = w4[q];
        acc[0][4 * q + 0] = __fmaf_rn(xa[ci], wq.x, acc[0][4 * q + 0]);
        acc[0][4 * q + 1] = __fmaf_rn(xa[ci], wq.y, acc[0][4 * q + 1]);
        acc[0][4 * q + 2] = __fmaf_rn(xa[ci], wq.z, acc[0][4 * q + 2]);
        acc[0][4 * q + 3] = __fmaf_rn(xa[ci], wq.w, acc[0][4 * q + 3]);
        acc[1][4 * q + 0] = __fmaf_rn(xb[ci], wq.x, acc[1][4 * q + 0]);
        acc[1][4 * q + 1] = __fmaf_rn(xb[ci], wq.y, acc[1][4 * q + 1]);
        acc[1][4 * q + 2] = __fmaf_rn(xb[ci], wq.z, acc[1][4 * q + 2]);
        acc[1][4 * q + 3] = __fmaf_rn(xb[ci], wq.w, acc[1][4 * q + 3]);
      }
    }
  }
  const int gi = i0 + ti;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int gj = j0 + tj + h * TW;
    if (gi >= H || gj >= W) continue;
    const size_t p = ((size_t)b * H + gi) * W + gj;
    // the pixel's 32 channels as four 16-byte stores
#pragma unroll
    for (int c4 = 0; c4 < C / 8; ++c4) {
      uint4 o;
      uint32_t* o32 = reinterpret_cast<uint32_t*>(&o);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int co = c4 * 8 + 2 * e;
        const float y0 = acc[h][co] + sW[9 * 4 * C + co], y1 = acc[h][co + 1] + sW[9 * 4 * C + co + 1];
        if (Y) *reinterpret_cast<float2*>(Y + p * C + co) = make_float2(y0, y1);
        const __nv_bfloat162 ob = __floats2bfloat162_rn(fmaxf(y0, 0.f), fmaxf(y1, 0.f));
        o32[e] = *reinterpret_cast<const uint32_t*>(&ob);
      }
      *reinterpret_cast<uint4*>(X + p * C + c4 * 8) = o;
    }
  }
}

// ------------------------------------------------------------------ 32 -> 32 conv on the tensor cores
__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

enum { CONV_FWD = 0, CONV_BWD = 1 };

// out[p][n] = sum_{tap, k} in[p + off(tap)][k] * Wk[tap][n][k].
// CONV_FWD: y = out + bias; X_out = bf16(X_in + ReLU(y)); Y (optional) = y.
// CONV_BWD: G_out = G_in + out.
// Persistent blocks: the weights go to shared memory once per block, which then loops over 8 x 16
// pixel tiles (tile = blockIdx.x, blockIdx.x + gridDim.x, ...).
template <int MODE>
__global__ void __launch_bounds__(128) k_conv32(const bf16* __restrict__ Xin, const bf16* __restrict__ Wk,
                                                const float* __restrict__ bias, int B, int H, int W,
                                                bf16* __restrict__ Xout, float* __restrict__ Y,
                                                const float* __restrict__ Gin, float* __restrict__ Gout) {
  __shared__ __align__(16) bf16 sX[HT * WT * XS];
  __shared__ __align__(16) bf16 sW[9 * C * XS];
  for (int r = threadIdx.x; r < 9 * C * 4; r += 128) {
    const int row = r >> 2, part = r & 3;
    *reinterpret_cast<uint4*>(&sW[row * XS + part * 8]) = *reinterpret_cast<const uint4*>(&Wk[row * C + part * 8]);
  }
  const int ntj = (W + TW - 1) / TW, nti = (H + TH - 1) / TH, ntiles = B * nti * ntj;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int b = tile / (nti * ntj), rem = tile - b * (nti * ntj);
    const int i0 = (rem / ntj) * TH, j0 = (rem % ntj) * TW;
    __syncthreads();   // the previous tile's readers of sX are done
    for (int r = threadIdx.x; r < HT * WT * 4; r += 128) {
      const int pix = r >> 2, part = r & 3;
      const int gi = i0 + pix / WT - 1, gj = j0 + pix % WT - 1;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gi >= 0 && gi < H && gj >= 0 && gj < W)
        v = *reinterpret_cast<const uint4*>(&Xin[(((size_t)b * H + gi) * W + gj) * C + part * 8]);
      *reinterpret_cast<uint4*>(&sX[pix * XS + part * 8]) = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[r][nt][e] = 0.f;
#pragma unroll 1
    for (int t = 0; t < 9; ++t) {
      const int di = t / 3 - 1, dj = t % 3 - 1;
#pragma unroll
      for (int cb = 0; cb < 2; ++cb) {
        uint32_t bq[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const bf16* wp = &sW[(t * C + nt * 8 + g) * XS + cb * 16 + q * 2];
          bq[nt][0] = *reinterpret_cast<const uint32_t*>(wp);
          bq[nt][1] = *reinterpret_cast<const uint32_t*>(wp + 8);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int ty = warp * 2 + r;
          const bf16* xp = &sX[((ty + 1 + di) * WT + (g + 1 + dj)) * XS + cb * 16 + q * 2];
          const uint32_t a0 = *reinterpret_cast<const uint32_t*>(xp);
          const uint32_t a1 = *reinterpret_cast<const uint32_t*>(xp + 8 * XS);
          const uint32_t a2 = *reinterpret_cast<const uint32_t*>(xp + 8);
          const uint32_t a3 = *reinterpret_cast<const uint32_t*>(xp + 8 * XS + 8);
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[r][nt], a0, a1, a2, a3, bq[nt][0], bq[nt][1]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int ty = warp * 2 + r, gi = i0 + ty;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int tj = g + 8 * half, gj = j0 + tj;
        if (gi >= H || gj >= W) continue;
        const size_t p = ((size_t)b * H + gi) * W + gj;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int co = nt * 8 + 2 * q;
          const float v0 = acc[r][nt][2 * half], v1 = acc[r][nt][2 * half + 1];
          if (MODE == CONV_FWD) {
            const float y0 = v0 + bias[co], y1 = v1 + bias[co + 1];
            const bf16* xc = &sX[((ty + 1) * WT + tj + 1) * XS + co];
            const float x0 = __bfloat162float(xc[0]), x1 = __bfloat162float(xc[1]);
            if (Y) *reinterpret_cast<float2*>(Y + p * C + co) = make_float2(y0, y1);
            *reinterpret_cast<__nv_bfloat162*>(Xout + p * C + co) =
                __floats2bfloat162_rn(x0 + fmaxf(y0, 0.f), x1 + fmaxf(y1, 0.f));
          } else {
            const float2 gi2 = *reinterpret_cast<const float2*>(Gin + p * C + co);
            *reinterpret_cast<float2*>(Gout + p * C + co) = make_float2(gi2.x + v0, gi2.y + v1);
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------ 32 -> 32 conv, tcgen05 (forward)
// The convolution on the fifth-generation tensor cores, as a pipeline in one persistent block per
// SM that walks tiles of TC_R output rows x 128 pixels (tile blockIdx.x, + gridDim.x, ...):
//   warp 0 (one lane)   loads each tile's halo (TC_R + 2 rows x 130 pixels x 32 bf16 channels) with
//                       four TMA copies, one per 8-channel chunk, into a ring of TC_NS stages,
//                       zero-filled outside the image;
//   warp 1 (one lane)   issues per output row 9 taps x 2 K-halves = 18 tcgen05.mma (M = 128
//                       pixels, N = 32, K = 16, BF16 in, FP32 accumulate) into that row's 32 columns
//                       of one of two TMEM accumulators, then commits to the accumulator's "full"
//                       barrier and to the stage's "empty" barrier;
//   warps 2-5           read the accumulator (each warp its 32 TMEM lanes, i.e. pixels), add bias,
//                       ReLU and the residual (from the same stage), store, and release the
//                       accumulator and the stage.
// So tile i + 1 loads and tile i multiplies while tile i - 1 is written.  The stage holds
// [chunk][row][pixel][8 channels]: the A operand of tap (di, dj) for output row r is a K-major
// no-swizzle matrix starting at row r + 1 + di, pixel 1 + dj (core matrices of 8 pixels x 16 bytes,
// 128 bytes between pixel groups, one chunk between K halves) - no im2col.  Weights sit as
// sB[tap][chunk][cout][8 cin].  Every mbarrier wait is bounded; a role whose wait gives up raises a
// flag the others see, and the epilogue then writes NaN into the tiles it has not written, which
// the solve rejects.
constexpr int TC_R = 4;                        // output rows per tile
constexpr int TC_W = 128;                      // pixels per row (the MMA's M)
constexpr int TC_WT = TC_W + 2;                // with halo
constexpr int TC_CHUNK_TX = (TC_R + 2) * TC_WT * 16;   // bytes one chunk's TMA copy writes (12,480)
constexpr int TC_CHUNK = (TC_CHUNK_TX + 127) / 128 * 128;   // chunk stride, 128-byte aligned (12,544)
constexpr int TC_ROWB = TC_WT * 16;            // bytes of one halo row of a chunk
constexpr int TC_STAGE = 4 * TC_CHUNK;         // one halo tile
constexpr int TC_NS = 3;                       // halo tiles in flight
constexpr int TC_BBYTES = 9 * 4 * C * 16;      // 18,432
constexpr int TC_OSTRIDE = 80;                 // bytes per pixel of an epilogue warp's staging rows (64 + 16)
constexpr int TC_OBYTES = 4 * 32 * TC_OSTRIDE; // four epilogue warps x 32 pixels
constexpr int TC_SMEM = TC_NS * TC_STAGE + TC_BBYTES + TC_OBYTES + 1024;   // + alignment of the dynamic base
constexpr int TC_ACC = TC_R * C;               // TMEM columns of one accumulator (128)
constexpr int TC_COLS = 2 * TC_ACC;            // two accumulators
constexpr int TC_THREADS = 192;
constexpr long long TC_WAIT_LIMIT = 1LL << 24; // mbarrier polls before giving up
static_assert(TC_COLS == 256, "TMEM allocation");
static_assert(TC_STAGE % 1024 == 0 || TC_CHUNK % 128 == 0, "TMA destinations 128-byte aligned");

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major, N = 32, M = 128.
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(C >> 3) << 17) | ((uint32_t)(TC_W >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start address, the byte offsets between core
// matrices along K (leading) and along M/N (stride), descriptor version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Bounded wait for the completion of phase `parity` of an mbarrier; gives up (raising *fail) after
// TC_WAIT_LIMIT polls, or at once when another role has raised *fail.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, volatile int* fail, bool heed = true) {
  for (long long it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile("{\n.reg .pred q;\nmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\nselp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    if (ok) return true;
    if (heed && (it & 63) == 0 && *fail) return false;
  }
  *fail = 1;
  return false;
}

__device__ __forceinline__ void tc_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(mbar) : "memory");
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_conv32_tc(const __grid_constant__ CUtensorMap xmap,
                                                             const bf16* __restrict__ Wk,
                                                             const float* __restrict__ bias, int B, int H, int W,
                                                             bf16* __restrict__ Xout, float* __restrict__ Y) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) unsigned long long s_bar[2 * TC_NS + 4];   // full[NS], empty[NS], tfull[2], tempty[2]
  __shared__ float s_bias[C];
  __shared__ volatile int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rawBase = (uint32_t)__cvta_generic_to_shared(smem_raw);
  const uint32_t aBase = (rawBase + 1023u) & ~1023u;              // TC_NS stages of TC_STAGE bytes
  const uint32_t bBase = aBase + TC_NS * TC_STAGE;
  unsigned char* const sA = smem_raw + (aBase - rawBase);
  unsigned char* const sB = smem_raw + (bBase - rawBase);
  const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&s_bar[0]);
  auto full = [&](int st) { return bar0 + 8u * (uint32_t)st; };
  auto empty = [&](int st) { return bar0 + 8u * (uint32_t)(TC_NS + st); };
  auto tfull = [&](int a) { return bar0 + 8u * (uint32_t)(2 * TC_NS + a); };
  auto tempty = [&](int a) { return bar0 + 8u * (uint32_t)(2 * TC_NS + 2 + a); };
  // weights -> sB[tap][chunk][cout][8], bias; barriers; TMEM (warp 1)
  for (int r = tid; r < 9 * C * 4; r += TC_THREADS) {
    const int t = r / (C * 4), n = (r / 4) % C, kc = r % 4;
    *reinterpret_cast<uint4*>(sB + (((t * 4 + kc) * C + n) * 16)) =
        *reinterpret_cast<const uint4*>(&Wk[(t * C + n) * C + kc * 8]);
  }
  for (int r = tid; r < C; r += TC_THREADS) s_bias[r] = bias[r];
  if (tid == 0) {
    s_fail = 0;
    for (int st = 0; st < TC_NS; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(full(st)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 5;\n" :: "r"(empty(st)) : "memory");   // commit + 4 warps
    }
    for (int a = 0; a < 2; ++a) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(tfull(a)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" :: "r"(tempty(a)) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("prefetch.tensormap [%0];\n" :: "l"(reinterpret_cast<uint64_t>(&xmap)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 :: "r"((uint32_t)__cvta_generic_to_shared(&s_tmem)), "r"((uint32_t)TC_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // the weights (generic-proxy writes) become visible to the tensor core's reads
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int ntj = (W + TC_W - 1) / TC_W, nti = (H + TC_R - 1) / TC_R, ntiles = B * nti * ntj;
  auto tile_origin = [&](int t, int& b, int& i0, int& j0) {
    b = t / (nti * ntj);
    const int rem = t - b * (nti * ntj);
    i0 = (rem / ntj) * TC_R;
    j0 = (rem % ntj) * TC_W;
  };
  if (warp == 0) {
    // ---------------------------------------------------------------- producer
    if (lane == 0) {
      int issued = 0;
      for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
        const int st = i % TC_NS;
        if (i >= TC_NS && !tc_wait(empty(st), (uint32_t)((i / TC_NS - 1) & 1), &s_fail)) break;
        issued = i + 1;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                     :: "r"(full(st)), "r"((uint32_t)(4 * TC_CHUNK_TX)) : "memory");
        int b, i0, j0;
        tile_origin(t, b, i0, j0);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t dst = aBase + (uint32_t)(st * TC_STAGE + c * TC_CHUNK);
          asm volatile(
              "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
              :: "r"(dst), "l"(reinterpret_cast<uint64_t>(&xmap)), "r"(c * 8), "r"(j0 - 1), "r"(i0 - 1), "r"(b),
                 "r"(full(st)) : "memory");
        }
      }
      // after a failure, the copies still in flight land before the block leaves
      if (s_fail)
        for (int i = (issued > TC_NS ? issued - TC_NS : 0); i < issued; ++i)
          tc_wait(full(i % TC_NS), (uint32_t)((i / TC_NS) & 1), &s_fail, false);
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA issue
    if (lane == 0) {
      int issued = 0;
      for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
        const int st = i % TC_NS, a = i & 1;
        if (!tc_wait(full(st), (uint32_t)((i / TC_NS) & 1), &s_fail)) break;
        if (i >= 2 && !tc_wait(tempty(a), (uint32_t)((i / 2 - 1) & 1), &s_fail)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        // descriptors of the stage's first A matrix and of the first B matrix; the other 71 differ only
        // in their start address (the low 14 bits, address / 16), by compile-time offsets, so the
        // fully unrolled issue is an add and an MMA each
        const uint64_t ad0 = tc_desc(aBase + (uint32_t)(st * TC_STAGE), TC_CHUNK, 128);
        const uint64_t bd0 = tc_desc(bBase, C * 16, 128);
        const uint32_t d0 = tmem + (uint32_t)(a * TC_ACC);
#pragma unroll
        for (int r = 0; r < TC_R; ++r) {
#pragma unroll
          for (int tap = 0; tap < 9; ++tap) {
            const int di = tap / 3 - 1, dj = tap % 3 - 1;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const uint64_t ad = ad0 + (uint64_t)((2 * h * TC_CHUNK + (r + 1 + di) * TC_ROWB + (1 + dj) * 16) >> 4);
              const uint64_t bd = bd0 + (uint64_t)((((tap * 4 + 2 * h) * C) * 16) >> 4);
              const uint32_t acc = (tap > 0 || h > 0) ? 1u : 0u;   // the row's first product starts it
              asm volatile(
                  "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                  :: "r"(d0 + (uint32_t)(r * C)), "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc) : "memory");
            }
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                     :: "r"(tfull(a)) : "memory");
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                     :: "r"(empty(st)) : "memory");
        ++issued;
      }
      // the last multiplications have finished before the accumulators are freed
      if (issued > 0) tc_wait(tfull((issued - 1) & 1), (uint32_t)(((issued - 1) / 2) & 1), &s_fail);
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 2-5)
    const int q = warp & 3;              // TMEM lanes 32 q .. 32 q + 31 = pixels of this warp
    const int px = q * 32 + lane;
    // staging rows of this warp's output: the stores to global memory go out as contiguous runs
    unsigned char* const sO = sB + TC_BBYTES + (warp - 2) * 32 * TC_OSTRIDE;
    bool ok = true;
    for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
      const int st = i % TC_NS, a = i & 1;
      int b, i0, j0;
      tile_origin(t, b, i0, j0);
      // one lane of the warp waits (the others would only compete with the tensor core for shared
      // memory) for the accumulator and for the stage's halo tile, which is read below for the
      // residual (its barrier is complete already: the stage cannot be refilled before this warp
      // releases it); __syncwarp orders the other lanes' reads after the wait
      if (lane == 0 && ok) {
        ok = tc_wait(tfull(a), (uint32_t)((i / 2) & 1), &s_fail);
        if (ok) ok = tc_wait(full(st), (uint32_t)((i / TC_NS) & 1), &s_fail);
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;   // the TMEM reads below are warp-collective
      __syncwarp();
      if (ok) asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int gj = j0 + px;
      for (int r = 0; r < TC_R; ++r) {
        uint32_t v[C];
        if (ok) {
          const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * TC_ACC + r * C);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
              "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
              : "r"(taddr) : "memory");
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        } else {
#pragma unroll
          for (int k = 0; k < C; ++k) v[k] = 0u;
        }
        const int gi = i0 + r;
        if (gi >= H) continue;   // warp-uniform: the whole row is outside the image
        const bool inw = gj < W;
        const size_t p = ((size_t)b * H + gi) * W + gj;
        const unsigned char* xc = sA + st * TC_STAGE + (r + 1) * TC_ROWB + (px + 1) * 16;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint4 xin = ok ? *reinterpret_cast<const uint4*>(xc + c * TC_CHUNK) : make_uint4(0u, 0u, 0u, 0u);
          const __nv_bfloat162* x2 = reinterpret_cast<const __nv_bfloat162*>(&xin);
          uint4 o;
          uint32_t* o32 = reinterpret_cast<uint32_t*>(&o);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int co = c * 8 + 2 * e;
            float y0 = __uint_as_float(v[co]) + s_bias[co], y1 = __uint_as_float(v[co + 1]) + s_bias[co + 1];
            if (!ok) { y0 = __int_as_float(0x7fc00000); y1 = y0; }
            if (Y && inw) *reinterpret_cast<float2*>(Y + p * C + co) = make_float2(y0, y1);
            const float2 xf = __bfloat1622float2(x2[e]);
            const __nv_bfloat162 ob = __floats2bfloat162_rn(xf.x + fmaxf(y0, 0.f), xf.y + fmaxf(y1, 0.f));
            o32[e] = *reinterpret_cast<const uint32_t*>(&ob);
          }
          *reinterpret_cast<uint4*>(sO + lane * TC_OSTRIDE + c * 16) = o;
        }
        // the warp's 32 pixels are 2 KB in a row of the output: written as four runs of 512 bytes,
        // 16 bytes a lane (run k, lane l: pixel 8 k + l / 4, channels 8 (l % 4) ...)
        __syncwarp();
        const size_t p0 = ((size_t)b * H + gi) * W + (j0 + q * 32);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int byte = k * 512 + lane * 16, pl = byte >> 6, cc = (byte >> 4) & 3;
          if (j0 + q * 32 + pl < W)
            *reinterpret_cast<uint4*>(&Xout[(p0 + pl) * C + cc * 8]) =
                *reinterpret_cast<const uint4*>(sO + pl * TC_OSTRIDE + cc * 16);
        }
        __syncwarp();
      }
      // this warp is done with the accumulator and the stage
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (ok && lane == 0) {
        tc_arrive(tempty(a));
        tc_arrive(empty(st));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"((uint32_t)TC_COLS)
                 : "memory");
  }
}

// ------------------------------------------------------------------ head: 32 -> 1, FP32 cores
__global__ void __launch_bounds__(TP) k_head(const bf16* __restrict__ X, const float* __restrict__ w, int H, int W,
                                             float* __restrict__ out) {
  __shared__ __align__(16) bf16 sX[HT * WT * XS];
  __shared__ __align__(16) float sW[9 * C + 1];
  const int b = blockIdx.z, i0 = blockIdx.y * TH, j0 = blockIdx.x * TW;
  for (int r = threadIdx.x; r < 9 * C + 1; r += TP) sW[r] = w[r];
  for (int r = threadIdx.x; r < HT * WT * 4; r += TP) {
    const int pix = r >> 2, part = r & 3;
    const int gi = i0 + pix / WT - 1, gj = j0 + pix % WT - 1;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gi >= 0 && gi < H && gj >= 0 && gj < W)
      v = *reinterpret_cast<const uint4*>(&X[(((size_t)b * H + gi) * W + gj) * C + part * 8]);
    *reinterpret_cast<uint4*>(&sX[pix * XS + part * 8]) = v;
  }
  __syncthreads();
  const int ti = threadIdx.x / TW, tj = threadIdx.x % TW;
  const int gi = i0 + ti, gj = j0 + tj;
  if (gi >= H || gj >= W) return;
  float acc = 0.f;
  for (int t = 0; t < 9; ++t) {
    const uint4* xp = reinterpret_cast<const uint4*>(&sX[((ti + t / 3) * WT + tj + t % 3) * XS]);
    const float4* w4 = reinterpret_cast<const float4*>(&sW[t * C]);
#pragma unroll
    for (int q = 0; q < C / 8; ++q) {
      const uint4 xv = xp[q];
      const __nv_bfloat162* x2 = reinterpret_cast<const __nv_bfloat162*>(&xv);
      const float4 wa = w4[2 * q], wb = w4[2 * q + 1];
      const float2 f0 = __bfloat1622float2(x2[0]), f1 = __bfloat1622float2(x2[1]);
      const float2 f2 = __bfloat1622float2(x2[2]), f3 = __bfloat1622float2(x2[3]);
      acc = __fmaf_rn(f0.x, wa.x, acc); acc = __fmaf_rn(f0.y, wa.y, acc);
      acc = __fmaf_rn(f1.x, wa.z, acc); acc = __fmaf_rn(f1.y, wa.w, acc);
      acc = __fmaf_rn(f2.x, wb.x, acc); acc = __fmaf_rn(f2.y, wb.y, acc);
      acc = __fmaf_rn(f3.x, wb.z, acc); acc = __fmaf_rn(f3.y, wb.w, acc);
    }
  }
  out[((size_t)b * H + gi) * W + gj] = acc + sW[9 * C];
}

// ------------------------------------------------------------------ backward pieces
// G4[p][ci] = sum_tap gout[p - off(tap)] * wh[tap][ci]
__global__ void __launch_bounds__(TP) k_head_bwd(const float* __restrict__ gout, const float* __restrict__ w, int H,
                                                 int W, float* __restrict__ G) {
  __shared__ float sG[HT * WT];
  __shared__ float sW[9 * C];
  const int b = blockIdx.z, i0 = blockIdx.y * TH, j0 = blockIdx.x * TW;
  for (int r = threadIdx.x; r < 9 * C; r += TP) sW[r] = w[r];
  for (int r = threadIdx.x; r < HT * WT; r += TP) {
    const int gi = i0 + r / WT - 1, gj = j0 + r % WT - 1;
    sG[r] = (gi >= 0 && gi < H && gj >= 0 && gj < W) ? gout[((size_t)b * H + gi) * W + gj] : 0.f;
  }
  __syncthreads();
  const int ti = threadIdx.x / TW, tj = threadIdx.x % TW;
  const int gi = i0 + ti, gj = j0 + tj;
  if (gi >= H || gj >= W) return;
  const size_t p = ((size_t)b * H + gi) * W + gj;
  for (int ci = 0; ci < C; ++ci) {
    float acc = 0.f;
    for (int t = 0; t < 9; ++t) {
      const int tm = 8 - t;   // gout at p + off(8 - t) = p - off(t)
      acc = acc + sG[(ti + 1 + tm / 3 - 1) * WT + tj + 1 + tm % 3 - 1] * sW[t * C + ci];
    }
    G[p * C + ci] = acc;
  }
}

// DY = G * (Y > 0) in FP32 and a BF16 copy for the tensor-core data gradient.
__global__ void k_relu_bwd(const float* __restrict__ G, const float* __restrict__ Y, float* __restrict__ DY,
                           bf16* __restrict__ DYb, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = Y[i] > 0.f ? G[i] : 0.f;
  DY[i] = v;
  if (DYb) DYb[i] = __float2bfloat16_rn(v);
}

template <typename XT>
__device__ __forceinline__ float ld_as_float(const XT* p);
template <>
__device__ __forceinline__ float ld_as_float<float>(const float* p) { return bfr(*p); }
template <>
__device__ __forceinline__ float ld_as_float<bf16>(const bf16* p) { return __bfloat162float(*p); }

// Weight gradient partials: part[blk][(tap * CIN + ci) * COUT + co] = sum over the block's tiles of
// X[p + off(tap)][ci] * DY[p][co], and part[blk][9 * CIN * COUT + co] = sum DY[p][co].  Thread
// (rg, co) owns output channel co and the (tap, ci) rows rg, rg + NRG, ...; pixels are the outer loop,
// so each step reads one DY value and broadcasts X across the warp.
template <int CIN, int COUT, typename XT>
__global__ void __launch_bounds__(256) k_wgrad(const XT* __restrict__ X, const float* __restrict__ DY, int B, int H,
                                               int W, float* __restrict__ part) {
  constexpr int R = 9 * CIN;
  constexpr int NRG = 256 / COUT;
  constexpr int PER = (R + NRG - 1) / NRG;
  constexpr int NOUT = R * COUT + COUT;
  __shared__ float sX[HT * WT * CIN];
  __shared__ float sD[TP * COUT];
  const int co = threadIdx.x % COUT, rg = threadIdx.x / COUT;
  float acc[PER];
  float accb = 0.f;
#pragma unroll
  for (int m = 0; m < PER; ++m) acc[m] = 0.f;
  const int ntiles = B * ((H + TH - 1) / TH) * ((W + TW - 1) / TW);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const TileIdx T = tile_of(tile, H, W);
    __syncthreads();
    for (int r = threadIdx.x; r < HT * WT * CIN; r += 256) {
      const int pix = r / CIN, ci = r % CIN;
      const int gi = T.i0 + pix / WT - 1, gj = T.j0 + pix % WT - 1;
      sX[r] = (gi >= 0 && gi < H && gj >= 0 && gj < W) ? ld_as_float<XT>(X + (((size_t)T.b * H + gi) * W + gj) * CIN + ci)
                                                       : 0.f;
    }
    for (int r = threadIdx.x; r < TP * COUT; r += 256) {
      const int pix = r / COUT, c = r % COUT;
      const int gi = T.i0 + pix / TW, gj = T.j0 + pix % TW;
      sD[r] = (gi < H && gj < W) ? DY[(((size_t)T.b * H + gi) * W + gj) * COUT + c] : 0.f;
    }
    __syncthreads();
#pragma unroll 1
    for (int pix = 0; pix < TP; ++pix) {
      const float dv = sD[pix * COUT + co];
      const int base = ((pix / TW) * WT + pix % TW) * CIN;
      if (rg == 0) accb = accb + dv;
#pragma unroll
      for (int m = 0; m < PER; ++m) {
        const int r = rg + NRG * m;
        if (r < R) {
          const int t = r / CIN, ci = r % CIN;
          acc[m] = acc[m] + sX[base + ((t / 3) * WT + t % 3) * CIN + ci] * dv;
        }
      }
    }
  }
  float* o = part + (size_t)blockIdx.x * NOUT;
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int r = rg + NRG * m;
    if (r < R) o[r * COUT + co] = acc[m];
  }
  if (rg == 0) o[R * COUT + co] = accb;
}

// grad[off + o] = sum_blk part[blk][o] (fixed order); the weight part [9][CIN][COUT] first, then
// the COUT bias entries.
__global__ void k_wgrad_reduce(const float* __restrict__ part, int nblk, int nout, float* __restrict__ grad) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nout) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s = s + part[(size_t)b * nout + o];
  grad[o] = s;
}

// ------------------------------------------------------------------ loss and optimiser
__global__ void k_loss_part(const float* __restrict__ out, const float* __restrict__ t, const float* __restrict__ mask,
                            int n, float* __restrict__ part) {
  __shared__ float s1[256], s2[256];
  float a = 0.f, m = 0.f;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    if (mask[i] > 0.f) {
      const float d = out[i] - t[i];
      a = a + d * d;
      m = m + 1.f;
    }
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) { s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = s1[0]; part[2 * blockIdx.x + 1] = s2[0]; }
}

__global__ void k_loss_final(const float* __restrict__ part, int nblk, float* __restrict__ loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float a = 0.f, m = 0.f;
  for (int b = 0; b < nblk; ++b) { a = a + part[2 * b]; m = m + part[2 * b + 1]; }
  loss[0] = m > 0.f ? a / m : 0.f;
  loss[1] = m;
}

__global__ void k_loss_grad(const float* __restrict__ out, const float* __restrict__ t, const float* __restrict__ mask,
                            int n, const float* __restrict__ loss, float* __restrict__ gout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float m = loss[1];
  gout[i] = (mask[i] > 0.f && m > 0.f) ? 2.f * (out[i] - t[i]) / m : 0.f;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ------------------------------------------------------------------ solver-side kernels
// r0 = qq - A sp for every wet column (SolverSparse's matrix: diagonal rr, off-diagonals -sx_W,
// -sy_S, -sy, -sx) and block partial sums of r0^2.
__global__ void k_feat_resid(Dev d, double* __restrict__ r0, double* __restrict__ part) {
  __shared__ double sh[256];
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  double v = 0.0;
  if (l <= d.g.lm) {
    const int lE = NB(d.g.lEC, l), lW = NB(d.g.lWC, l), lN = NB(d.g.lNC, l), lS = NB(d.g.lSC, l);
    const double* sp = d.s.sp;
    const double ax = d.s.rr[l - 1] * sp[l - 1] - d.s.sx[lW - 1] * sp[lW - 1] - d.s.sy[lS - 1] * sp[lS - 1] -
                      d.s.sy[l - 1] * sp[lN - 1] - d.s.sx[l - 1] * sp[lE - 1];
    const double r = d.s.qq[l - 1] - ax;
    r0[l - 1] = r;
    v = r * r;
  }
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// One block of 256 threads: strided partial sums, then a tree in shared memory (fixed order).
__global__ void k_feat_sigma(const double* __restrict__ part, int nblk, int lm, double* __restrict__ sigma) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += 256) s += part[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sigma[0] = lm > 0 ? sqrt(sh[0] / lm) : 0.0;
}

__global__ void k_feat_write(Dev d, const int* __restrict__ pix, const double* __restrict__ r0,
                             const double* __restrict__ sigma, float* __restrict__ feat) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const double s = sigma[0];
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  float4 f;
  f.x = (float)(r0[l - 1] * inv);
  f.y = (float)((d.s.sp[l - 1] - d.s.spp[l - 1]) * inv);
  f.z = (float)(d.g.hhs[l - 1] / 30.0);
  f.w = 1.f;
  *reinterpret_cast<float4*>(feat + (size_t)pix[l - 1] * 4) = f;
}

__global__ void k_feat_scatter(int lm, const int* __restrict__ pix, const float* __restrict__ out,
                               const double* __restrict__ sigma, double* __restrict__ dz) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > lm) return;
  const double s = sigma[0];
  dz[l - 1] = s > 0.0 ? s * (double)out[pix[l - 1]] : 0.0;
}

__global__ void k_record(Dev d, const int* __restrict__ pix, const float* __restrict__ feat,
                         const double* __restrict__ sigma, float* __restrict__ rec) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const size_t p = (size_t)pix[l - 1];
  const float4 f = *reinterpret_cast<const float4*>(feat + p * 4);
  const double s = sigma[0];
  float* o = rec + p * 5;
  o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
  o[4] = s > 0.0 ? (float)((d.s.s[l - 1] - d.s.sp[l - 1]) / s) : 0.f;
}

dim3 tiles(int B, int H, int W) { return dim3((W + TW - 1) / TW, (H + TH - 1) / TH, B); }

}  // namespace

// ---------------------------------------------------------------------------- host side
size_t Workspace::bytes(int B, int H, int W, bool training) {
  const size_t P = (size_t)B * H * W;
  size_t s = 0;
  auto add = [&](size_t n) { s += (n + 255) / 256 * 256; };
  add(2 * SI3D_NET_BLOCKS * 9 * C * C * sizeof(bf16));   // wfwd, wbwd
  add((9 * 4 * C + C) * sizeof(float));
  add((9 * C + 1) * sizeof(float));
  const int nx = training ? SI3D_NET_BLOCKS + 1 : 2;
  for (int i = 0; i < nx; ++i) add(P * C * sizeof(bf16));
  if (training) {
    for (int i = 0; i < SI3D_NET_BLOCKS + 1; ++i) add(P * C * sizeof(float));   // y0..y4
    for (int i = 0; i < 3; ++i) add(P * C * sizeof(float));                     // G, G', DY
    add(P * C * sizeof(bf16));                                                   // DYb
    add((size_t)WG_BLOCKS * (9 * C * C + C) * sizeof(float));                    // weight-gradient partials
  }
  return s;
}

bool Workspace::carve(void* base, size_t avail, int B, int H, int W, bool training) {
  if (!base || avail < bytes(B, H, W, training)) return false;
  const size_t P = (size_t)B * H * W;
  char* q = static_cast<char*>(base);
  auto take = [&](size_t n) { void* r = q; q += (n + 255) / 256 * 256; return r; };
  wfwd = static_cast<bf16*>(take(SI3D_NET_BLOCKS * 9 * C * C * sizeof(bf16) * 2));
  wbwd = wfwd + SI3D_NET_BLOCKS * 9 * C * C;
  stem = static_cast<float*>(take((9 * 4 * C + C) * sizeof(float)));
  head = static_cast<float*>(take((9 * C + 1) * sizeof(float)));
  const int nx = training ? SI3D_NET_BLOCKS + 1 : 2;
  for (int i = 0; i < SI3D_NET_BLOCKS + 1; ++i) x[i] = nullptr;
  for (int i = 0; i < nx; ++i) x[i] = static_cast<bf16*>(take(P * C * sizeof(bf16)));
  for (int i = 0; i < SI3D_NET_BLOCKS + 1; ++i) y[i] = nullptr;
  G0 = G1 = DY = nullptr;
  DYb = nullptr;
  part = nullptr;
  if (training) {
    for (int i = 0; i < SI3D_NET_BLOCKS + 1; ++i) y[i] = static_cast<float*>(take(P * C * sizeof(float)));
    G0 = static_cast<float*>(take(P * C * sizeof(float)));
    G1 = static_cast<float*>(take(P * C * sizeof(float)));
    DY = static_cast<float*>(take(P * C * sizeof(float)));
    DYb = static_cast<bf16*>(take(P * C * sizeof(bf16)));
    part = static_cast<float*>(take((size_t)WG_BLOCKS * (9 * C * C + C) * sizeof(float)));
  }
  this->training = training;
  return true;
}

void prepare(const Workspace& ws, const float* params, cudaStream_t st) {
  const int n = SI3D_NET_BLOCKS * 9 * C * C;
  k_prep<<<(n + 255) / 256, 256, 0, st>>>(params, ws.wfwd, ws.wbwd, ws.stem, ws.head);
}

// Persistent grid of the convolution: every resident block of the device, at most one per tile.
template <int MODE>
int conv_blocks(int B, int H, int W) {
  int dev = 0, sms = 1, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv32<MODE>, 128, 0);
  const long long ntiles = (long long)B * ((H + TH - 1) / TH) * ((W + TW - 1) / TW);
  return (int)std::max(1LL, std::min(ntiles, (long long)sms * std::max(occ, 1)));
}

// Persistent grid of the tcgen05 convolution: one block per SM (its shared memory takes most of
// one), enabled once per device.
int conv_tc_blocks(int B, int H, int W) {
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  static bool attr_set[64] = {false};
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    cudaFuncSetAttribute(k_conv32_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    attr_set[dev] = true;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long ntiles = (long long)B * ((H + TC_R - 1) / TC_R) * ((W + TC_W - 1) / TC_W);
  return (int)std::max(1LL, std::min(ntiles, (long long)sms));
}

// cuTensorMapEncodeTiled from the driver, looked up once.
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// TMA map of a channels-last activation image [B][H][W][C] (bf16): boxes of 8 channels (16 bytes,
// the innermost extent) x 130 pixels x (TC_R + 2) rows of one image; coordinates outside the image
// read as zero.
bool activation_map(CUtensorMap* m, const bf16* x, int B, int H, int W) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_tiled();
  if (!enc || (reinterpret_cast<uintptr_t>(x) & 15u) != 0) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[3] = {(cuuint64_t)C * sizeof(bf16), (cuuint64_t)W * C * sizeof(bf16),
                                 (cuuint64_t)H * W * C * sizeof(bf16)};
  const cuuint32_t box[4] = {8, (cuuint32_t)TC_WT, (cuuint32_t)(TC_R + 2), 1};
  const cuuint32_t elem[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(x), dims, strides, box, elem,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int forward(const Workspace& ws, const float* params, const float* feat, int B, int H, int W, float* out,
            cudaStream_t st) {
  const float* bias0 = params + OFF_BLK + 9 * C * C;
  const dim3 grid = tiles(B, H, W);
  CUtensorMap maps[SI3D_NET_BLOCKS];
  for (int k = 0; k < SI3D_NET_BLOCKS; ++k)
    if (!activation_map(&maps[k], ws.training ? ws.x[k] : ws.x[k & 1], B, H, W)) return SI3D_ECUDA;
  k_stem<<<dim3((W + ST_W - 1) / ST_W, (H + TH - 1) / TH, B), TP, 0, st>>>(feat, ws.stem, H, W, ws.x[0],
                                                                         ws.training ? ws.y[0] : nullptr);
  const int nb = conv_tc_blocks(B, H, W);
  for (int k = 0; k < SI3D_NET_BLOCKS; ++k) {
    bf16* xout = ws.training ? ws.x[k + 1] : ws.x[(k + 1) & 1];
    k_conv32_tc<<<nb, TC_THREADS, TC_SMEM, st>>>(maps[k], ws.wfwd + (size_t)k * 9 * C * C,
                                                  bias0 + (size_t)k * BLK_SZ, B, H, W, xout,
                                                  ws.training ? ws.y[k + 1] : nullptr);
  }
  const bf16* xl = ws.training ? ws.x[SI3D_NET_BLOCKS] : ws.x[SI3D_NET_BLOCKS & 1];
  k_head<<<grid, TP, 0, st>>>(xl, ws.head, H, W, out);
  return 0;
}

void backward(const Workspace& ws, const float* feat, const float* gout, int B, int H, int W, float* grad,
              cudaStream_t st) {
  const dim3 grid = tiles(B, H, W);
  const size_t n = (size_t)B * H * W * C;
  const int eb = (int)((n + 255) / 256);
  // head
  k_wgrad<C, 1, bf16><<<WG_BLOCKS, 256, 0, st>>>(ws.x[SI3D_NET_BLOCKS], gout, B, H, W, ws.part);
  k_wgrad_reduce<<<(9 * C + 1 + 255) / 256, 256, 0, st>>>(ws.part, WG_BLOCKS, 9 * C + 1, grad + OFF_HEAD_W);
  k_head_bwd<<<grid, TP, 0, st>>>(gout, ws.head, H, W, ws.G0);
  float* G = ws.G0;
  float* Gn = ws.G1;
  for (int k = SI3D_NET_BLOCKS - 1; k >= 0; --k) {
    k_relu_bwd<<<eb, 256, 0, st>>>(G, ws.y[k + 1], ws.DY, ws.DYb, n);
    k_wgrad<C, C, bf16><<<WG_BLOCKS, 256, 0, st>>>(ws.x[k], ws.DY, B, H, W, ws.part);
    k_wgrad_reduce<<<(BLK_SZ + 255) / 256, 256, 0, st>>>(ws.part, WG_BLOCKS, BLK_SZ, grad + OFF_BLK + k * BLK_SZ);
    k_conv32<CONV_BWD><<<conv_blocks<CONV_BWD>(B, H, W), 128, 0, st>>>(ws.DYb, ws.wbwd + (size_t)k * 9 * C * C, nullptr,
                                                                       B, H, W, nullptr, nullptr, G, Gn);
    std::swap(G, Gn);
  }
  k_relu_bwd<<<eb, 256, 0, st>>>(G, ws.y[0], ws.DY, nullptr, n);
  k_wgrad<4, C, float><<<WG_BLOCKS, 256, 0, st>>>(feat, ws.DY, B, H, W, ws.part);
  k_wgrad_reduce<<<(9 * 4 * C + C + 255) / 256, 256, 0, st>>>(ws.part, WG_BLOCKS, 9 * 4 * C + C, grad);
}

void features(const Dev& d, const int* pix, double* r0, double* part, double* sigma, float* feat, cudaStream_t st) {
  const int nb = (d.g.lm + 255) / 256;
  k_feat_resid<<<nb, 256, 0, st>>>(d, r0, part);
  k_feat_sigma<<<1, 256, 0, st>>>(part, nb, d.g.lm, sigma);
  k_feat_write<<<nb, 256, 0, st>>>(d, pix, r0, sigma, feat);
}

void scatter(int lm, const int* pix, const float* out, const double* sigma, double* dz, cudaStream_t st) {
  k_feat_scatter<<<(lm + 255) / 256, 256, 0, st>>>(lm, pix, out, sigma, dz);
}

void record(const Dev& d, const int* pix, const float* feat, const double* sigma, float* rec, cudaStream_t st) {
  k_record<<<(d.g.lm + 255) / 256, 256, 0, st>>>(d, pix, feat, sigma, rec);
}

int feature_partials(int lm) { return (lm + 255) / 256; }

}  // namespace learn
}  // namespace si3d

// ---------------------------------------------------------------------------- C ABI (training)
using si3d::learn::Workspace;

extern "C" {

size_t si3d_net_workspace_bytes(int B, int H, int W) {
  if (B < 1 || H < 1 || W < 1) return 0;
  return Workspace::bytes(B, H, W, true);
}

int si3d_net_forward(const float* params, const float* feat, int B, int H, int W, float* out, void* ws_ptr,
                     size_t ws_bytes) {
  if (!params || !feat || !out || B < 1 || H < 1 || W < 1) return SI3D_EDIMS;
  Workspace ws;
  if (!ws.carve(ws_ptr, ws_bytes, B, H, W, true)) return SI3D_EDIMS;
  si3d::learn::prepare(ws, params, 0);
  if (int rc = si3d::learn::forward(ws, params, feat, B, H, W, out, 0)) return rc;
  return cudaGetLastError() == cudaSuccess ? SI3D_OK : SI3D_ECUDA;
}

int si3d_net_loss(const float* out, const float* target, const float* mask, int n, float* gout, float* loss_dev) {
  if (!out || !target || !mask || !gout || !loss_dev || n < 1) return SI3D_EDIMS;
  constexpr int NB = 148;
  float* part = loss_dev + 2;   // the caller's loss buffer holds 2 + 2 * 148 floats
  si3d::learn::k_loss_part<<<NB, 256>>>(out, target, mask, n, part);
  si3d::learn::k_loss_final<<<1, 32>>>(part, NB, loss_dev);
  si3d::learn::k_loss_grad<<<(n + 255) / 256, 256>>>(out, target, mask, n, loss_dev, gout);
  return cudaGetLastError() == cudaSuccess ? SI3D_OK : SI3D_ECUDA;
}

int si3d_net_backward(const float* params, const float* feat, const float* gout, int B, int H, int W, float* grad,
                      void* ws_ptr, size_t ws_bytes) {
  if (!params || !feat || !gout || !grad || B < 1 || H < 1 || W < 1) return SI3D_EDIMS;
  Workspace ws;
  if (!ws.carve(ws_ptr, ws_bytes, B, H, W, true)) return SI3D_EDIMS;
  si3d::learn::backward(ws, feat, gout, B, H, W, grad, 0);
  return cudaGetLastError() == cudaSuccess ? SI3D_OK : SI3D_ECUDA;
}

int si3d_net_adam(float* params, const float* grad, float* m, float* v, int n, float lr, float beta1, float beta2,
                  float eps, int t) {
  if (!params || !grad || !m || !v || n < 1 || t < 1) return SI3D_EDIMS;
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  si3d::learn::k_adam<<<(n + 255) / 256, 256>>>(params, grad, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? SI3D_OK : SI3D_ECUDA;
}

int si3d_net_sync(void) { return cudaDeviceSynchronize() == cudaSuccess ? SI3D_OK : SI3D_ECUDA; }

}  // extern "C"
