// Shared device helpers for the Tier-3 step kernels (sm_100a, FP64).
//
// Layout: every 3D field is a C-contiguous float64 array (Nz, Ny, Nx),
// cell (k, j, i) at flat index (k*Ny + j)*Nx + i, exactly the numpy layout
// the reference kernels mutate in place (spread_3d.py:88-155).
//
// Arithmetic is transcribed operation by operation from the reference
// expressions; the library is built with FMA contraction, so a multiply-add
// rounds once where numba rounds twice, and libm transcendental functions
// (exp/pow/tanh) are within a few ulp of glibc: results agree with the
// reference to round-off.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/firestep.h"

// Division by a run-time invariant divisor d >= 1 as a multiply-high, an
// add and two shifts (Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, unsigned case with
// l = ceil(log2 d)): exact for every 32-bit dividend.  Replaces the 64-bit
// divisions a flat cell index would otherwise need to recover (i, j, k).
struct FastDiv {
  uint32_t d, m, s1, s2;
};
inline FastDiv fastdiv_make(uint32_t d) {
  FastDiv f;
  f.d = d;
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < (unsigned long long)d) ++l;
  f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  f.s1 = l < 1 ? l : 1;
  f.s2 = l > 1 ? l - 1 : 0;
  return f;
}
__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(f.m, n);
#else
  const uint32_t t = (uint32_t)(((unsigned long long)f.m * n) >> 32);
#endif
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

// Grid geometry as the kernels see it.  dz/da/db are device arrays of length nz
// (dz_arr, d_face_above, d_face_below of Grid3D, spread_3d.py:180-188);
// fnx/fny divide by nx and ny (grids hold fewer than 2^31 cells).
struct GridDev {
  int nx, ny, nz;
  double dx, dy;
  const double* dz;
  const double* da;
  const double* db;
  FastDiv fnx, fny;
};

// Set-up work (copies of host arrays, clearing of new buffers) runs on a
// private non-blocking stream that is synchronised before the set-up returns:
// it neither waits for nor disturbs other threads' streams, one of which may
// be capturing a CUDA graph (a cudaDeviceSynchronize or a legacy default
// stream operation would then fail or break that capture).
struct SetupStream {
  cudaStream_t s = nullptr;
  SetupStream() {
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
  }
  ~SetupStream() {
    if (s) cudaStreamDestroy(s);
  }
  SetupStream(const SetupStream&) = delete;
  SetupStream& operator=(const SetupStream&) = delete;
  bool sync() const { return s && cudaStreamSynchronize(s) == cudaSuccess; }
};

// (i, j, k) of flat cell index c = (k*ny + j)*nx + i
__device__ __forceinline__ void split_cell(uint32_t c, const FastDiv& fnx, const FastDiv& fny,
                                           int& i, int& j, int& k) {
  const uint32_t r = fdiv(c, fnx);
  i = (int)(c - r * fnx.d);
  const uint32_t kk = fdiv(r, fny);
  j = (int)(r - kk * fny.d);
  k = (int)kk;
}

__host__ __device__ inline int64_t cidx(const GridDev& g, int k, int j, int i) {
  return ((int64_t)k * g.ny + j) * (int64_t)g.nx + i;
}

__device__ __forceinline__ int wrapj(int j, int ny) {
  int r = j % ny;
  return r < 0 ? r + ny : r;
}

// minmod limiter (muscl_3d.py:37-44), as selects (no divergent branches):
// 0 when a*b <= 0, else the argument of smaller magnitude
__device__ __forceinline__ double minmod(double a, double b) {
  const double lo = a < b ? a : b, hi = a > b ? a : b;
  const double m = a > 0.0 ? lo : hi;
  return (a * b <= 0.0) ? 0.0 : m;
}

// upwind-biased MUSCL face value at i+1/2 from cells i-1..i+2 (muscl_3d.py:47-64):
// uf >= 0: pi + 0.5 minmod(pi - pim1, pip1 - pi); else pip1 - 0.5 minmod(pip1 - pi,
// pip2 - pip1).  Both sides are formed by selects; x + (-0.5 s) equals x - 0.5 s
// exactly, so the values are the branchy form's bit for bit.
__device__ __forceinline__ double muscl_face(double pim1, double pi, double pip1,
                                             double pip2, double uf) {
  const bool up = uf >= 0.0;
  const double a = up ? pi - pim1 : pip1 - pi;
  const double b = up ? pip1 - pi : pip2 - pip1;
  const double base = up ? pi : pip1;
  const double half = up ? 0.5 : -0.5;
  return base + half * minmod(a, b);
}

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Launch geometry helpers: one thread per cell, x fastest.
struct Launch3 {
  dim3 grid, block;
};
inline Launch3 launch_cells(const GridDev& g) {
  Launch3 L;
  int bx = g.nx >= 128 ? 128 : (g.nx >= 64 ? 64 : 32);
  int by = 256 / bx;
  L.block = dim3(bx, by, 1);
  L.grid = dim3((g.nx + bx - 1) / bx, (g.ny + by - 1) / by, g.nz);
  return L;
}

__host__ __device__ inline int64_t ncells(const GridDev& g) { return (int64_t)g.nx * g.ny * g.nz; }
__device__ __forceinline__ int64_t ncells_dev(const GridDev& g) { return (int64_t)g.nx * g.ny * g.nz; }

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// last CUDA error -> status
inline int cuda_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FS_OK : FS_ECUDA;
}

// Per-thread error text for fs_last_error().
void fs_set_error(const char* fmt, ...);

// Count of kernel launches issued by this library (fs_launch_count()).
void fs_count_launch();
// wait for a stream with a blocking-sync event (no host spinning)
int fs_stream_wait(cudaStream_t st);
