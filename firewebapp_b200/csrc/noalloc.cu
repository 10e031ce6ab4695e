// EDC entry point for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc themselves or let a
// plugin call it: a framework whose own allocator owns all device memory (a
// fixed arena sized at start-up, or a caching allocator that must see every
// byte), or a time-step loop that cannot take the device-wide
// synchronisation a cudaMalloc/cudaFree can cause.  fs_edc needs a scratch
// buffer from its caller; this variant needs none.
//
// fs_edc_noalloc runs the same three EDC kernels as fs_edc, with the flag
// scan's scratch in a file-scope device array instead of a caller buffer.
// The array's address is looked up once per device, with that device
// current, at the first call on it.  Every call shares the array: agg and
// carry are fully rewritten by each call before they are read, so nothing
// has to start at zero, and calls whose kernels overlap on the GPU race on
// it.
#include <mutex>
#include "common.cuh"
#include "kernels.h"

#define NOALLOC_MAX_DEVICES 64
#define EDC_NOALLOC_SCRATCH_BYTES (2 * (FS_EDC_NOALLOC_MAX_CELLS / 1024) + 16)

static __device__ __align__(256) unsigned char g_edc_scratch[EDC_NOALLOC_SCRATCH_BYTES];

static std::mutex g_scratch_mu;
static void* g_scratch_ptr[NOALLOC_MAX_DEVICES];

// Address of the scratch array on the current device (looked up once per device).
static int edc_static_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fs_set_error("fs_edc_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
    return FS_ECUDA;
  }
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
    fs_set_error("fs_edc_noalloc: device %d outside the supported 0..%d", dev,
                 NOALLOC_MAX_DEVICES - 1);
    return FS_EARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_edc_scratch);
    if (e != cudaSuccess || !p) {
      fs_set_error("fs_edc_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                   cudaGetErrorString(e));
      return FS_ECUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return FS_OK;
}

extern "C" int fs_edc_noalloc(int64_t n, const double* rho, double* T_g, double* Y_F,
                              double* Y_O2, const double* k, const double* eps,
                              const double* Y_H2O, double* omega, double chi_rad, double cp_g,
                              double dt, int n_substeps, double s_stoich, double hoc_J,
                              int extinction, void* stream) {
  if (n < 0 || n > (int64_t)FS_EDC_NOALLOC_MAX_CELLS) {
    fs_set_error("fs_edc_noalloc: n = %lld cells is outside 0..%lld (the static scratch limit)",
                 (long long)n, (long long)FS_EDC_NOALLOC_MAX_CELLS);
    return FS_EARG;
  }
  if (n == 0) return FS_OK;
  void* scratch = nullptr;
  int rc = edc_static_scratch(&scratch);
  if (rc != FS_OK) return rc;
  rc = launch_edc(n, rho, T_g, Y_F, Y_O2, k, eps, Y_H2O, omega, chi_rad, cp_g, dt, n_substeps,
                  s_stoich, hoc_J, extinction, scratch, (cudaStream_t)stream);
  if (rc != FS_OK) fs_set_error("fs_edc_noalloc: launch failed (status %d)", rc);
  return rc;
}
