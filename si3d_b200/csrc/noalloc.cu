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
// so the first call on each device looks the address up with cudaGetSymbolAddress while that
// device is current and caches it; make that first call before any stream capture.  Every call
// shares the one array: the forward sweep writes each scratch element before the backward sweep
// reads it, so nothing has to be cleared between calls, but two calls whose kernels overlap on
// the same GPU race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/si3d_gpu.h"
#include "kernels.h"

namespace {

static __device__ __align__(256) double g_trid_scratch[SI3D_NOALLOC_MAX_ELEMS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SI3D_ENODEV;
  if (dev < 0 || dev >= kMaxDevices) return SI3D_ENODEV;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_trid_scratch) != cudaSuccess || !p) return SI3D_ECUDA;
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace

extern "C" int si3d_gpu_column_tridiag_noalloc(int n, int nsys, const double* a, const double* b, const double* c,
                                               const double* g, const double* r, double* ag, double* ar,
                                               void* stream) {
  if (n < 1 || nsys < 1 || !a || !b || !c || !g || !r || !ag || !ar) return SI3D_EDIMS;
  if ((long long)n * (long long)nsys > (long long)SI3D_NOALLOC_MAX_ELEMS) return SI3D_ECAPACITY;
  double* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  si3d::launch_column_tridiag(n, nsys, a, b, c, g, r, ag, ar, scratch, st);
  if (cudaGetLastError() != cudaSuccess) return SI3D_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SI3D_ECUDA;
  return 0;
}
