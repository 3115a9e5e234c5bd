// Internal interface of the learned initial guess (k_learn.cu) for the solver orchestration.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/si3d_learn.h"
#include "common.cuh"

namespace si3d {
namespace learn {

// Device buffers of one network evaluation (carved from one allocation).  Inference keeps two
// ping-pong activation images; training keeps every layer's input and pre-activation for the
// backward pass.
struct Workspace {
  __nv_bfloat16 *wfwd = nullptr, *wbwd = nullptr;   // tensor-core weights [block][tap][n][k]
  float *stem = nullptr, *head = nullptr;           // bf16-rounded stem/head weights + biases
  __nv_bfloat16* x[SI3D_NET_BLOCKS + 1] = {};        // activations (layer inputs), channels-last
  float* y[SI3D_NET_BLOCKS + 1] = {};                // pre-activations (training)
  float *G0 = nullptr, *G1 = nullptr, *DY = nullptr;
  __nv_bfloat16* DYb = nullptr;
  float* part = nullptr;                            // weight-gradient partial sums
  bool training = false;
  static size_t bytes(int B, int H, int W, bool training);
  bool carve(void* base, size_t avail, int B, int H, int W, bool training);
};

void prepare(const Workspace& ws, const float* params, cudaStream_t st);
// 0, or SI3D_ECUDA when the activations' TMA maps cannot be made (nothing is launched then)
int forward(const Workspace& ws, const float* params, const float* feat, int B, int H, int W, float* out,
            cudaStream_t st);
void backward(const Workspace& ws, const float* feat, const float* gout, int B, int H, int W, float* grad,
              cudaStream_t st);

// Solver side: features of the current zeta system into feat[pix(l)] (r0, sigma on the device),
// prediction scatter dz(l) = sigma * out[pix(l)], and the training record of one solve.
int feature_partials(int lm);
void features(const Dev& d, const int* pix, double* r0, double* part, double* sigma, float* feat, cudaStream_t st);
void scatter(int lm, const int* pix, const float* out, const double* sigma, double* dz, cudaStream_t st);
void record(const Dev& d, const int* pix, const float* feat, const double* sigma, float* rec, cudaStream_t st);

}  // namespace learn
}  // namespace si3d
