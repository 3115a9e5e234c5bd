// Allocation-free variant of the batched two-right-hand-side tridiagonal solver.
//
// Some callers cannot call cudaMalloc: a model coupled into a framework that owns the device
// allocator and its memory budget, or a time loop that must not allocate once it is running.  This
// entry point takes the caller's device buffers for inputs and outputs, and the Thomas sweep's
// scratch (the forward-sweep ratios c1) comes from a fixed array compiled into the library, so
// the call allocates nothing.
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds its
// 8 MiB until the process exits.  Host code cannot use the name of the array as a device address,
// so every call looks the address up with cudaGetSymbolAddress in the context that is current at
// that moment (a cached address could belong to another context of the same device, or to a module
// image that a device reset has since replaced); the lookup is cheap next to the synchronisation
// that ends the call.  Every call shares the one array: the forward sweep writes each scratch
// element before the backward sweep reads it, so nothing has to be cleared between calls, but two
// calls whose kernels overlap on the same GPU race on it.
#include <cuda_runtime.h>

#include "../../include/si3d_gpu.h"
#include "kernels.h"

namespace {

static __device__ __align__(256) double g_trid_scratch[SI3D_NOALLOC_MAX_ELEMS];

}  // namespace

extern "C" int si3d_gpu_column_tridiag_noalloc(int n, int nsys, const double* a, const double* b, const double* c,
                                               const double* g, const double* r, double* ag, double* ar,
                                               void* stream) {
  if (n < 1 || nsys < 1 || !a || !b || !c || !g || !r || !ag || !ar) return SI3D_EDIMS;
  if ((long long)n * (long long)nsys > (long long)SI3D_NOALLOC_MAX_ELEMS) return SI3D_ECAPACITY;
  // An error left pending by the caller's earlier work is reported, not cleared, and nothing is
  // launched on top of it.
  if (cudaPeekAtLastError() != cudaSuccess) return SI3D_ECUDA;
  void* scratch = nullptr;
  if (cudaGetSymbolAddress(&scratch, g_trid_scratch) != cudaSuccess || !scratch) return SI3D_ECUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  si3d::launch_column_tridiag(n, nsys, a, b, c, g, r, ag, ar, static_cast<double*>(scratch), st);
  if (cudaPeekAtLastError() != cudaSuccess) return SI3D_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SI3D_ECUDA;
  return 0;
}
