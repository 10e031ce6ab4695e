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

// minmod limiter (muscl_3d.py:37-44): 0 when a*b <= 0, else the argument of
// smaller magnitude.  When a*b > 0 both arguments are finite, non-zero and of
// one sign, so that argument is exactly copysign(min(|a|, |b|), a): one
// hardware minimum in place of compare-and-select chains.  Symmetric in a, b
// (the product and the chosen value do not depend on the order).
__device__ __forceinline__ double minmod(double a, double b) {
  const double m = copysign(fmin(fabs(a), fabs(b)), a);
  return (a * b <= 0.0) ? 0.0 : m;
}

// upwind-biased MUSCL face value at i+1/2 from cells i-1..i+2 (muscl_3d.py:47-64):
// uf >= 0: pi + 0.5 minmod(pi - pim1, pip1 - pi); else pip1 - 0.5 minmod(pip1 - pi,
// pip2 - pip1).  The difference pip1 - pi is common to both sides, so by the
// limiter's symmetry only its other argument is selected; x + (-0.5 s) equals
// x - 0.5 s exactly, so the values are the branchy form's bit for bit.
__device__ __forceinline__ double muscl_face(double pim1, double pi, double pip1,
                                             double pip2, double uf) {
  const bool up = uf >= 0.0;
  const double m = minmod(pip1 - pi, up ? pi - pim1 : pip2 - pip1);
  const double base = up ? pi : pip1;
  const double half = up ? 0.5 : -0.5;
  return base + half * m;
}

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Vertical solid conduction of one cell (solid_conduction_3d.py:56-127): the
// harmonic-mean face conductances to the bed cells above and below and the
// explicit update; cap = 1 clips the result to [lo, hi] (the T_s cap that
// follows the conduction, spread_3d.py:3193-3196).  T0 = Ts[c].
__device__ __forceinline__ double solid_cond_cell(const GridDev& g, const double* __restrict__ Ts,
                                                  const double* __restrict__ as, int k, int64_t c,
                                                  double T0, double k_solid, double inv_rho_cp,
                                                  double dt, int cap, double lo, double hi) {
  const int64_t sz = (int64_t)g.nx * g.ny;
  const double asc = as[c];
  if (asc <= 0.0) {
    double x = T0;
    if (cap) {
      if (x > hi) x = hi;
      if (x < lo) x = lo;
    }
    return x;
  }
  double fu = 0.0, fd = 0.0;
  if (k < g.nz - 1) {
    double aa = as[c + sz];
    if (aa > 0.0) {
      double ae = 2.0 * asc * aa / (asc + aa);
      fu = k_solid * ae * (Ts[c + sz] - T0) / g.da[k];
    }
  }
  if (k > 0) {
    double ab = as[c - sz];
    if (ab > 0.0) {
      double ae = 2.0 * asc * ab / (asc + ab);
      fd = k_solid * ae * (Ts[c - sz] - T0) / g.db[k];
    }
  }
  double src = (fu + fd) / g.dz[k];
  double dT = dt * src * inv_rho_cp / asc;
  double x = T0 + dT;
  if (cap) {
    if (x > hi) x = hi;
    if (x < lo) x = lo;
  }
  return x;
}

// EDC flag scan tiling: a block of EDC_TPB threads owns EDC_TILE consecutive
// cells, EDC_CPT per thread (thread t: cells EDC_CPT*t .. EDC_CPT*t + 3 of the
// tile), so a thread's loads are two 16-byte vectors per FP64 field and the
// tile's flat order is thread order, then the order within the thread.
#define EDC_TPB 256
#define EDC_CPT 4
#define EDC_TILE (EDC_TPB * EDC_CPT)

// Exclusive max-scan over the block's threads of `last` (every thread's
// largest code, -1 for none): the largest code of the threads before this
// one.  `sh` holds EDC_TPB / 32 ints; one barrier.
__device__ __forceinline__ int edc_block_exclusive_max(int last, int* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int v = last;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, y);
  }
  if (lane == 31) sh[wid] = v;
  int ex = __shfl_up_sync(0xffffffffu, v, 1);
  if (lane == 0) ex = -1;
  __syncthreads();
  for (int w = 0; w < wid; ++w) ex = max(ex, sh[w]);
  return ex;
}

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
