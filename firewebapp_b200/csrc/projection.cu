// Pressure projection (projection_3d.py ProjectionSolver3D, fft_pcg path).
//
// Operator (projection_3d.py:66-175 _fill_var_density_data with alpha_g = 1):
//   A p = div((1/rho_face) grad p) + 1e-6 p, rho floored at 0.01,
//   x: Neumann inlet / Dirichlet p=0 outlet face; y periodic;
//   z: Neumann wall / Dirichlet p=0 top face; non-uniform dz.
// Row k of A carries 1/dz_k, so S = -diag(dz) A is symmetric positive
// definite; S is stored as face conductances g (one per interior face) plus
// a per-cell term e (Dirichlet faces and the -dz_k 1e-6 shift):
//   (S x)_c = e_c x_c + sum_faces g_f (x_c - x_nb).
// The reference solves A p = rhs with BiCGSTAB + an FFT preconditioner
// (projection_3d.py:756-791); here S p = -dz rhs is solved with CG
// preconditioned by one geometric-multigrid V-cycle:
//   * coarse cells aggregate 2x2x2 fine cells (odd tails keep 1);
//   * coarse operator = 1/2 (P^T S P) with piecewise-constant P, which keeps
//     the face-conductance form (coarse face = sum of fine faces across it);
//   * nu pre- and nu post-sweeps of damped Jacobi (default nu = 4, omega = 0.9:
//     fewer CG iterations than 0.8 at the same cost per iteration, measured);
//   * the coarsest level (<= 64 cells) is solved with a dense inverse built
//     at each rebuild.
// The stopping test mirrors scipy's: ||b - A x||_2 < rtol ||b||_2 on the
// unsymmetrised system, warm-started from the previous solution.
#include <vector>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include "common.cuh"
#include "kernels.h"

#define PROJ_EPS 1.0e-6
#define MG_OMEGA 0.8          // damping of the coarsest level's smoothing-only solve
#define MG_OMEGA_DEFAULT 0.9  // damping of the V-cycle's smoothing sweeps
#define MG_NU_DEFAULT 4
#define MG_COARSE_MAX 48
// blocks of the reducing CG kernels (8 per SM of the 148: enough loads in
// flight to stream HBM); their partials are added in block order
#define RED_BLOCKS 1184
#define RED_THREADS 256
// Device scalar slots: 0 rz, 1 pq, 2 rz_new, 4 ||b_A||^2, 5 ||r_A||^2,
// 6 (rtol ||b_A||)^2, 7 converged flag, 8 iterations done.
#define SC_DONE 7
#define SC_IT 8
// Kernels of a PCG iteration return at once when the solve has converged,
// so iterations queued past convergence change nothing.
#define PCG_SKIP(done) \
  if ((done) && *(done) != 0.0) return;

// a level's extents with the divisions that recover (i, j, k) from a flat index
struct Dims {
  int nx, ny, nz;
  FastDiv fnx, fny;
};
inline Dims dims_make(int nx, int ny, int nz) {
  Dims D;
  D.nx = nx; D.ny = ny; D.nz = nz;
  D.fnx = fastdiv_make((uint32_t)nx);
  D.fny = fastdiv_make((uint32_t)ny);
  return D;
}

template <typename T>
struct MGLevelT {
  int nx, ny, nz;
  Dims dims;
  int64_t n;
  T *gx, *gy, *gz, *e, *dinv;  // conductances, per-cell term, 1/diag
  T *x, *b, *t, *s;            // correction, rhs, temps
};
using MGLevel = MGLevelT<double>;

struct ProjCtx {
  GridDev g;
  int nlev;
  MGLevel lev[16];
  double* Ainv;       // dense inverse at the coarsest level
  double* pc_r;       // PCG residual (level 0)
  double* pc_z;
  double* pc_p;
  double* pc_q;
  double* rhs;        // b_S
  double* partial;    // block partial sums [RED_BLOCKS * 4]
  double* scal;       // device scalars
  double* h_scal;     // pinned host mirror
  double* p_prev;     // warm start / solution (owned)
  double* ir;         // 1/max(rho, 0.01)
  int have_prev;
  int last_iters;     // CG iterations of the previous solve (batch size hint)
  cudaStream_t cs;    // private stream for graph capture
  cudaGraphExec_t iter_exec;  // one captured PCG iteration (0 until captured)
  int iter_kernels;   // kernels in that graph
  int graph_failed;
  int nu;             // Jacobi sweeps before and after the coarse correction
  int nu0;            // the same on the finest level (0: nu)
  double omega;       // Jacobi damping
  int tail_on;        // coarse levels in one launch (k_mg_vcycle_tail)
  // mixed-precision form: the V-cycle in FP32 (levels, coarse inverse, the
  // residual it smooths and the correction it returns); CG stays FP64
  int fp32;
  MGLevelT<float> lev32[16];
  float* Ainv32;
  float *r32, *z32;
  // host-side statistics of the last solve (ms): total, fetch waits (sum, max),
  // graph-launch calls (sum, max), fetches, iteration launches, iterations
  double stats[8];
  // learned form: flexible CG preconditioned by a U-Net (unet.cu), falling
  // back to V-cycle PCG from the current iterate when it stalls
  void* net;
  int max_learned;    // learned iterations before the fallback
  double stall;       // fallback when the residual norm shrinks by less than
                      // this factor per iteration (over the last 3)
  double* log_r0;     // optional copies of the starting residual / iterate
  double* log_x0;
  // last solve: learned iterations, V-cycle iterations, fell back (0/1);
  // then the number of fallbacks since creation
  double fcg[4];
};

// ---------------------------------------------------------------------------
__global__ void k_proj_level0(GridDev g, const double* __restrict__ rho, double* ir, double* gx,
                              double* gy, double* gz, double* e, double dx2, double dy2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  int64_t c = cidx(g, k, j, i);
  auto IR = [&](int64_t q) {
    double r = rho[q];
    double m = (r >= 0.01 || r != r) ? r : 0.01;
    return 1.0 / m;
  };
  double irc = IR(c);
  ir[c] = irc;
  const double dzk = g.dz[k];
  const double idz = 1.0 / dzk;
  double ee = -dzk * PROJ_EPS;
  // x faces
  if (i < nx - 1) {
    gx[c] = dzk * ((0.5 * (irc + IR(c + 1))) / dx2);
  } else {
    gx[c] = 0.0;
    ee += dzk * ((2.0 * irc) / dx2);
  }
  // y faces (periodic); Ny == 1 has no y coupling (projection_3d.py:128)
  if (ny > 1) {
    int jp = j + 1 < ny ? j + 1 : 0;
    gy[c] = dzk * ((0.5 * (irc + IR(c - (int64_t)j * sy + (int64_t)jp * sy))) / dy2);
  } else {
    gy[c] = 0.0;
  }
  // z faces
  if (k < nz - 1) {
    gz[c] = dzk * (((0.5 * (irc + IR(c + sz))) * idz) / g.da[k]);
  } else {
    gz[c] = 0.0;
    ee += dzk * (((2.0 * irc) * idz) * idz);
  }
  e[c] = ee;
}

// diagonal of a face-conductance operator -> 1/diag
template <typename T>
__global__ void k_mg_diag(Dims D, const T* __restrict__ gx,
                          const T* __restrict__ gy, const T* __restrict__ gz,
                          const T* __restrict__ e, T* dinv) {
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  int64_t n = (int64_t)nx * ny * nz;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  int i, j, k;
  split_cell((uint32_t)c, D.fnx, D.fny, i, j, k);
  int64_t sy = nx, sz = (int64_t)nx * ny;
  T d = e[c] + gx[c] + gy[c] + gz[c];
  if (i > 0) d += gx[c - 1];
  if (ny > 1) {
    int jm = j > 0 ? j - 1 : ny - 1;
    d += gy[c - (int64_t)j * sy + (int64_t)jm * sy];
  }
  if (k > 0) d += gz[c - sz];
  dinv[c] = T(1) / d;
}

// (S x)_c for a face-conductance operator
template <typename T>
__device__ __forceinline__ T mg_apply(int nx, int ny, int nz, const T* __restrict__ gx,
                                           const T* __restrict__ gy,
                                           const T* __restrict__ gz,
                                           const T* __restrict__ e,
                                           const T* __restrict__ x, int64_t c, int i, int j,
                                           int k) {
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const T xc = x[c];
  T y = e[c] * xc;
  if (i < nx - 1) y += gx[c] * (xc - x[c + 1]);
  if (i > 0) y += gx[c - 1] * (xc - x[c - 1]);
  if (ny > 1) {
    int jp = j + 1 < ny ? j + 1 : 0;
    int jm = j > 0 ? j - 1 : ny - 1;
    int64_t cp = c - (int64_t)j * sy + (int64_t)jp * sy;
    int64_t cm = c - (int64_t)j * sy + (int64_t)jm * sy;
    y += gy[c] * (xc - x[cp]);
    y += gy[cm] * (xc - x[cm]);
  }
  if (k < nz - 1) y += gz[c] * (xc - x[c + sz]);
  if (k > 0) y += gz[c - sz] * (xc - x[c - sz]);
  return y;
}

// Galerkin aggregation of level f into level c (coarse = scale * P^T S_f P)
template <typename T>
__global__ void k_mg_coarsen(int fx, int fy, int fz, const T* __restrict__ gxf,
                             const T* __restrict__ gyf, const T* __restrict__ gzf,
                             const T* __restrict__ ef, Dims DC, T* gxc,
                             T* gyc, T* gzc, T* ec, double scale_) {
  const int cx = DC.nx, cy = DC.ny, cz = DC.nz;
  int64_t n = (int64_t)cx * cy * cz;
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  int I, J, K;
  split_cell((uint32_t)q, DC.fnx, DC.fny, I, J, K);
  const int64_t fsy = fx, fsz = (int64_t)fx * fy;
  int i0 = 2 * I, i1 = min(2 * I + 1, fx - 1);
  int j0 = 2 * J, j1 = min(2 * J + 1, fy - 1);
  int k0 = 2 * K, k1 = min(2 * K + 1, fz - 1);
  T se = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  for (int k = k0; k <= k1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) se += ef[(int64_t)k * fsz + (int64_t)j * fsy + i];
  if (I < cx - 1) {
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j) sx += gxf[(int64_t)k * fsz + (int64_t)j * fsy + i1];
  }
  if (cy > 1) {
    for (int k = k0; k <= k1; ++k)
      for (int i = i0; i <= i1; ++i) sy += gyf[(int64_t)k * fsz + (int64_t)j1 * fsy + i];
  }
  if (K < cz - 1) {
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) sz += gzf[(int64_t)k1 * fsz + (int64_t)j * fsy + i];
  }
  const T scale = (T)scale_;
  gxc[q] = scale * sx;
  gyc[q] = scale * sy;
  gzc[q] = scale * sz;
  ec[q] = scale * se;
}

// Dense inverse of the coarsest operator (Gauss-Jordan in shared memory, n <= 64).
template <typename T>
__global__ void k_mg_coarse_inverse(int nx, int ny, int nz, const T* __restrict__ gx,
                                    const T* __restrict__ gy, const T* __restrict__ gz,
                                    const T* __restrict__ e, T* Ainv) {
  __shared__ T M[MG_COARSE_MAX][2 * MG_COARSE_MAX + 1];
  const int n = nx * ny * nz;
  const int t = threadIdx.x;
  for (int r = t; r < n; r += blockDim.x) {
    for (int q = 0; q < 2 * n; ++q) M[r][q] = 0.0;
  }
  __syncthreads();
  if (t == 0) {
    const int sy = nx, sz = nx * ny;
    for (int c = 0; c < n; ++c) {
      int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
      M[c][c] += e[c];
      if (i < nx - 1) { M[c][c] += gx[c]; M[c][c + 1] -= gx[c]; }
      if (i > 0) { M[c][c] += gx[c - 1]; M[c][c - 1] -= gx[c - 1]; }
      if (ny > 1) {
        int jp = j + 1 < ny ? j + 1 : 0, jm = j > 0 ? j - 1 : ny - 1;
        int cp = c - j * sy + jp * sy, cm = c - j * sy + jm * sy;
        M[c][c] += gy[c]; M[c][cp] -= gy[c];
        M[c][c] += gy[cm]; M[c][cm] -= gy[cm];
      }
      if (k < nz - 1) { M[c][c] += gz[c]; M[c][c + sz] -= gz[c]; }
      if (k > 0) { M[c][c] += gz[c - sz]; M[c][c - sz] -= gz[c - sz]; }
      M[c][n + c] = 1.0;
    }
  }
  __syncthreads();
  for (int piv = 0; piv < n; ++piv) {
    T d = M[piv][piv];
    __syncthreads();
    for (int q = t; q < 2 * n; q += blockDim.x) M[piv][q] /= d;
    __syncthreads();
    for (int r = t; r < n; r += blockDim.x) {
      if (r == piv) continue;
      T f = M[r][piv];
      if (f != 0.0)
        for (int q = 0; q < 2 * n; ++q) M[r][q] -= f * M[piv][q];
    }
    __syncthreads();
  }
  for (int r = t; r < n; r += blockDim.x)
    for (int q = 0; q < n; ++q) Ainv[r * n + q] = M[r][n + q];
}

template <typename T>
__global__ void k_mg_coarse_solve(int n, const T* __restrict__ Ainv,
                                  const T* __restrict__ b, T* x, const double* done) {
  PCG_SKIP(done);
  int r = threadIdx.x;
  if (r >= n) return;
  T s = 0.0;
  for (int q = 0; q < n; ++q) s += Ainv[r * n + q] * b[q];
  x[r] = s;
}

// damped Jacobi sweep: xo = x + w (b - S x) / d ; x == null means x = 0
template <typename T>
__global__ void k_mg_jacobi(Dims D, const T* __restrict__ gx,
                            const T* __restrict__ gy, const T* __restrict__ gz,
                            const T* __restrict__ e, const T* __restrict__ dinv,
                            const T* __restrict__ b, const T* __restrict__ x, T* xo,
                            double w_, const double* done) {
  PCG_SKIP(done);
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const T w = (T)w_;
  int64_t n = (int64_t)nx * ny * nz;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (!x) {
    xo[c] = w * b[c] * dinv[c];
    return;
  }
  int i, j, k;
  split_cell((uint32_t)c, D.fnx, D.fny, i, j, k);
  T r = b[c] - mg_apply(nx, ny, nz, gx, gy, gz, e, x, c, i, j, k);
  xo[c] = x[c] + w * r * dinv[c];
}

// coarse rhs = sum over children of the fine residual (b - S x)
template <typename T>
__global__ void k_mg_restrict_residual(Dims DF, const T* __restrict__ gx,
                                       const T* __restrict__ gy,
                                       const T* __restrict__ gz,
                                       const T* __restrict__ e, const T* __restrict__ b,
                                       const T* __restrict__ x, Dims DC,
                                       T* bc, const double* done) {
  PCG_SKIP(done);
  const int fx = DF.nx, fy = DF.ny, fz = DF.nz;
  const int cx = DC.nx, cy = DC.ny, cz = DC.nz;
  int64_t n = (int64_t)cx * cy * cz;
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  int I, J, K;
  split_cell((uint32_t)q, DC.fnx, DC.fny, I, J, K);
  const int64_t fsy = fx, fsz = (int64_t)fx * fy;
  T s = 0.0;
  for (int k = 2 * K; k <= min(2 * K + 1, fz - 1); ++k)
    for (int j = 2 * J; j <= min(2 * J + 1, fy - 1); ++j)
      for (int i = 2 * I; i <= min(2 * I + 1, fx - 1); ++i) {
        int64_t c = (int64_t)k * fsz + (int64_t)j * fsy + i;
        s += b[c] - mg_apply(fx, fy, fz, gx, gy, gz, e, x, c, i, j, k);
      }
  bc[q] = s;
}

// x_f += P x_c (piecewise constant)
template <typename T>
__global__ void k_mg_prolong(Dims DF, T* x, int cx, int cy,
                             const T* __restrict__ xc, const double* done) {
  PCG_SKIP(done);
  int64_t n = (int64_t)DF.nx * DF.ny * DF.nz;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  int i, j, k;
  split_cell((uint32_t)c, DF.fnx, DF.fny, i, j, k);
  x[c] += xc[((int64_t)(k >> 1) * cy + (j >> 1)) * cx + (i >> 1)];
}

// ---------------------------------------------------------------------------
// deterministic FP64 dot products: fixed block count, fixed reduction tree
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NV>
__device__ __forceinline__ void block_sums_store(double (&v)[NV], double* partial) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = warp_sum(v[q]);
    if (lane == 0) sh[q][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = lane < (blockDim.x >> 5) ? sh[q][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) partial[q * RED_BLOCKS + blockIdx.x] = s;
    }
  }
}

__global__ void k_finish_sums(const double* __restrict__ partial, int nv, double* out,
                              const double* done) {
  PCG_SKIP(done);
  int q = threadIdx.x >> 5;
  int lane = threadIdx.x & 31;
  if (q >= nv) return;
  double s = 0.0;
  for (int b = lane; b < RED_BLOCKS; b += 32) s += partial[q * RED_BLOCKS + b];
  s = warp_sum(s);
  if (lane == 0) out[q] = s;
}

// rhs: b_S = -dz_k (div - target)/dt, plus ||(div - target)/dt||^2
__global__ void k_proj_rhs(GridDev g, const double* __restrict__ u, const double* __restrict__ v,
                           const double* __restrict__ w, const double* __restrict__ u_in,
                           const double* __restrict__ target, double dt, double* bS,
                           double* partial) {
  const int64_t n = ncells_dev(g);
  const int nx = g.nx, ny = g.ny;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)RED_BLOCKS * blockDim.x) {
    int i, j, k;
    split_cell((uint32_t)c, g.fnx, g.fny, i, j, k);
    double div;
    if (i > 0) div = (u[c] - u[c - 1]) / g.dx;
    else div = (u[c] - u_in[(int64_t)k * ny + j]) / g.dx;
    if (ny > 1) {
      int jm = j > 0 ? j - 1 : ny - 1;
      div += (v[c] - v[c - (int64_t)j * sy + (int64_t)jm * sy]) / g.dy;
    }
    if (k > 0) div += (w[c] - w[c - sz]) / g.dz[k];
    else div += (w[c] - 0.0) / g.dz[0];
    if (target) div = div - target[c];
    double rA = div / dt;
    bS[c] = -g.dz[k] * rA;
    acc[0] += rA * rA;
  }
  block_sums_store<1>(acc, partial);
}

// q = S p and partial of p.q
__global__ void k_pcg_matvec(Dims D, const double* __restrict__ gx,
                             const double* __restrict__ gy, const double* __restrict__ gz,
                             const double* __restrict__ e, const double* __restrict__ p, double* q,
                             double* partial, const double* done) {
  PCG_SKIP(done);
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const int64_t n = (int64_t)nx * ny * nz;
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)RED_BLOCKS * blockDim.x) {
    int i, j, k;
    split_cell((uint32_t)c, D.fnx, D.fny, i, j, k);
    double y = mg_apply(nx, ny, nz, gx, gy, gz, e, p, c, i, j, k);
    q[c] = y;
    acc[0] += p[c] * y;
  }
  block_sums_store<1>(acc, partial);
}

// r = b - S x, partial of ||r_A||^2 with r_A = -r / dz_k
__global__ void k_pcg_residual(GridDev g, const double* __restrict__ gx,
                               const double* __restrict__ gy, const double* __restrict__ gz,
                               const double* __restrict__ e, const double* __restrict__ b,
                               const double* __restrict__ x, double* r, double* partial) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t n = (int64_t)nx * ny * nz;
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)RED_BLOCKS * blockDim.x) {
    int i, j, k;
    split_cell((uint32_t)c, g.fnx, g.fny, i, j, k);
    double rr = b[c] - mg_apply(nx, ny, nz, gx, gy, gz, e, x, c, i, j, k);
    r[c] = rr;
    double ra = rr / g.dz[k];
    acc[0] += ra * ra;
  }
  block_sums_store<1>(acc, partial);
}

// x += alpha p ; r -= alpha q ; partial ||r_A||^2   (alpha = rz / pq from device scalars)
__global__ void k_pcg_update(GridDev g, const double* __restrict__ scal, double* x, double* r,
                             const double* __restrict__ p, const double* __restrict__ q,
                             double* partial) {
  PCG_SKIP(scal + SC_DONE);
  const int64_t n = ncells_dev(g);
  const double alpha = scal[0] / scal[1];
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)RED_BLOCKS * blockDim.x) {
    x[c] += alpha * p[c];
    double rr = r[c] - alpha * q[c];
    r[c] = rr;
    double ra = rr / g.dz[(int)fdiv(fdiv((uint32_t)c, g.fnx), g.fny)];
    acc[0] += ra * ra;
  }
  block_sums_store<1>(acc, partial);
}

// partial of r.z
__global__ void k_dot(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                      double* partial, const double* done) {
  PCG_SKIP(done);
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)RED_BLOCKS * blockDim.x)
    acc[0] += a[c] * b[c];
  block_sums_store<1>(acc, partial);
}

// p = z + beta p, beta = rz_new / rz_old ; first iteration p = z
__global__ void k_pcg_dir(int64_t n, const double* __restrict__ scal, const double* __restrict__ z,
                          double* p) {
  PCG_SKIP(scal + SC_DONE);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (scal[SC_IT] == 0.0) { p[c] = z[c]; return; }
  double beta = scal[2] / scal[0];
  p[c] = z[c] + beta * p[c];
}

__global__ void k_set_scal(double* scal, int dst, int src) {
  PCG_SKIP(scal + SC_DONE);
  scal[dst] = scal[src];
}

// end of an iteration: count it and test ||r_A|| < rtol ||b_A||
__global__ void k_pcg_check(double* scal) {
  if (scal[SC_DONE] != 0.0) return;
  scal[SC_IT] += 1.0;
  if (scal[5] < scal[6]) scal[SC_DONE] = 1.0;
}

// start of a solve: tolerance, initial test, iteration count; b == 0 -> x = 0
__global__ void k_pcg_init(double* scal, double rtol2) {
  scal[6] = rtol2 * scal[4];
  scal[SC_IT] = 0.0;
  scal[SC_DONE] = (scal[5] < scal[6] || scal[4] == 0.0) ? 1.0 : 0.0;
}

__global__ void k_zero_if_zero_rhs(int64_t n, const double* __restrict__ scal, double* x) {
  if (scal[4] != 0.0) return;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) x[c] = 0.0;
}

// Flexible CG (truncated to one previous direction): p = z - (z.q_prev / p.q_prev) p,
// first iteration p = z.  Slots: 10 z.q_prev, 11 p.q of the previous iteration.
__global__ void k_fcg_dir(int64_t n, const double* __restrict__ scal, const double* __restrict__ z,
                          double* p) {
  PCG_SKIP(scal + SC_DONE);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (scal[SC_IT] == 0.0) { p[c] = z[c]; return; }
  const double beta = -scal[10] / scal[11];
  p[c] = z[c] + beta * p[c];
}

// alpha = p.r / p.q into slot 0 (read by k_pcg_update); a zero direction
// (p.q = 0, e.g. a network output of 0) gives alpha = 0, so the residual
// stalls and the solve falls back instead of dividing by zero
__global__ void k_fcg_alpha(double* scal) {
  if (scal[SC_DONE] != 0.0) return;
  const bool ok = scal[1] > 0.0;
  scal[0] = ok ? scal[12] : 0.0;
  if (!ok) scal[1] = 1.0;
}

// out = b - S x (level operator, any precision)
template <typename T>
__global__ void k_lp_residual(Dims D, const T* __restrict__ gx,
                              const T* __restrict__ gy, const T* __restrict__ gz,
                              const T* __restrict__ e, const T* __restrict__ b,
                              const T* __restrict__ x, T* out) {
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  int64_t n = (int64_t)nx * ny * nz;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  int i, j, k;
  split_cell((uint32_t)c, D.fnx, D.fny, i, j, k);
  out[c] = b[c] - mg_apply(nx, ny, nz, gx, gy, gz, e, x, c, i, j, k);
}

// e1 = float(e0) - t
__global__ void k_lp_err(int64_t n, const double* __restrict__ e0, const float* __restrict__ t,
                         float* e1) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) e1[c] = (float)e0[c] - t[c];
}

// restart as V-cycle PCG from the current iterate (the residual was just
// recomputed into slot 5)
__global__ void k_fcg_restart(double* scal) {
  scal[SC_IT] = 0.0;
  scal[SC_DONE] = (scal[5] < scal[6]) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// velocity correction (projection_3d.py:818-842)
// ---------------------------------------------------------------------------
__global__ void k_proj_correct(GridDev g, double* u, double* v, double* w,
                               const double* __restrict__ p, const double* __restrict__ ir,
                               double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  int64_t c = cidx(g, k, j, i);
  const double pc = p[c], irc = ir[c];
  if (nx > 2) {
    if (i < nx - 1) u[c] -= dt * (p[c + 1] - pc) / g.dx * (0.5 * (irc + ir[c + 1]));
    else u[c] += 2.0 * dt * pc / g.dx * irc;
  }
  if (ny > 1) {
    int jp = j + 1 < ny ? j + 1 : 0;
    int64_t cp = c - (int64_t)j * sy + (int64_t)jp * sy;
    v[c] -= dt * (p[cp] - pc) / g.dy * (0.5 * (irc + ir[cp]));
  }
  if (nz > 2) {
    if (k < nz - 1) w[c] -= dt * (p[c + sz] - pc) / g.da[k] * (0.5 * (irc + ir[c + sz]));
    else w[c] += 2.0 * dt * pc / g.dz[nz - 1] * irc;
  }
}

// max |div(u) - target| (projection_3d.py:847-892 plain branch)
__global__ void k_div_resid_max(GridDev g, const double* __restrict__ u,
                                const double* __restrict__ v, const double* __restrict__ w,
                                const double* __restrict__ u_in, const double* __restrict__ target,
                                double* div_out, unsigned long long* out_key) {
  const int64_t n = ncells_dev(g);
  const int nx = g.nx, ny = g.ny;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  double best = 0.0;
  bool nan = false;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    split_cell((uint32_t)c, g.fnx, g.fny, i, j, k);
    double div;
    if (i > 0) div = (u[c] - u[c - 1]) / g.dx;
    else div = (u[c] - u_in[(int64_t)k * ny + j]) / g.dx;
    if (ny > 1) {
      int jm = j > 0 ? j - 1 : ny - 1;
      div += (v[c] - v[c - (int64_t)j * sy + (int64_t)jm * sy]) / g.dy;
    }
    if (k > 0) div += (w[c] - w[c - sz]) / g.dz[k];
    else div += (w[c] - 0.0) / g.dz[0];
    if (div_out) div_out[c] = div;
    if (target) div = div - target[c];
    double a = fabs(div);
    if (a != a) nan = true;
    else if (a > best) best = a;
  }
  unsigned long long key = nan ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(best);
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_xor_sync(0xffffffffu, key, o);
    key = y > key ? y : key;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out_key, key);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static double* dalloc(int64_t n) {
  double* p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return nullptr;
  return p;
}

void* proj_create(const GridDev& g) {
  ProjCtx* P = new ProjCtx();
  P->g = g;
  int nx = g.nx, ny = g.ny, nz = g.nz;
  int L = 0;
  while (true) {
    MGLevel& lv = P->lev[L];
    lv.nx = nx; lv.ny = ny; lv.nz = nz; lv.n = (int64_t)nx * ny * nz;
    lv.dims = dims_make(nx, ny, nz);
    lv.gx = dalloc(lv.n); lv.gy = dalloc(lv.n); lv.gz = dalloc(lv.n); lv.e = dalloc(lv.n);
    lv.dinv = dalloc(lv.n); lv.x = dalloc(lv.n); lv.b = dalloc(lv.n); lv.t = dalloc(lv.n);
    lv.s = dalloc(lv.n);
    ++L;
    if (lv.n <= MG_COARSE_MAX || L >= 16) break;
    int cx = (nx + 1) / 2, cy = (ny + 1) / 2, cz = (nz + 1) / 2;
    if (cx == nx && cy == ny && cz == nz) break;
    nx = cx; ny = cy; nz = cz;
  }
  P->nlev = L;
  int64_t n0 = P->lev[0].n;
  int64_t nc = P->lev[L - 1].n;
  P->Ainv = dalloc(nc <= MG_COARSE_MAX ? nc * nc : 1);
  P->pc_r = dalloc(n0); P->pc_z = dalloc(n0); P->pc_p = dalloc(n0); P->pc_q = dalloc(n0);
  P->rhs = dalloc(n0);
  P->partial = dalloc(RED_BLOCKS * 4);
  P->scal = dalloc(16);
  cudaMallocHost(&P->h_scal, sizeof(double) * 16);
  P->p_prev = dalloc(n0);
  P->ir = dalloc(n0);
  {
    // cleared before any solve is queued, on a private stream
    SetupStream ss;
    cudaMemsetAsync(P->p_prev, 0, sizeof(double) * n0, ss.s);
    cudaMemsetAsync(P->scal, 0, sizeof(double) * 16, ss.s);
    ss.sync();
  }
  P->have_prev = 0;
  P->last_iters = 0;
  P->iter_exec = nullptr;
  P->iter_kernels = 0;
  P->graph_failed = 0;
  P->nu = MG_NU_DEFAULT;
  P->nu0 = 0;
  P->tail_on = 1;
  P->fp32 = 0;
  P->Ainv32 = nullptr; P->r32 = nullptr; P->z32 = nullptr;
  for (int l = 0; l < 16; ++l) P->lev32[l] = MGLevelT<float>{};
  for (int q = 0; q < 8; ++q) P->stats[q] = 0.0;
  P->omega = MG_OMEGA_DEFAULT;
  P->net = nullptr;
  P->max_learned = 30;
  P->stall = 0.9;
  P->log_r0 = nullptr;
  P->log_x0 = nullptr;
  for (int q = 0; q < 4; ++q) P->fcg[q] = 0.0;
  cudaStreamCreateWithFlags(&P->cs, cudaStreamNonBlocking);
  if (cudaGetLastError() != cudaSuccess || !P->p_prev) {
    proj_destroy(P);
    return nullptr;
  }
  return P;
}

void proj_destroy(void* h) {
  ProjCtx* P = (ProjCtx*)h;
  if (!P) return;
  for (int l = 0; l < P->nlev; ++l) {
    MGLevel& lv = P->lev[l];
    cudaFree(lv.gx); cudaFree(lv.gy); cudaFree(lv.gz); cudaFree(lv.e); cudaFree(lv.dinv);
    cudaFree(lv.x); cudaFree(lv.b); cudaFree(lv.t); cudaFree(lv.s);
  }
  for (int l = 0; l < P->nlev; ++l) {
    MGLevelT<float>& lv = P->lev32[l];
    cudaFree(lv.gx); cudaFree(lv.gy); cudaFree(lv.gz); cudaFree(lv.e); cudaFree(lv.dinv);
    cudaFree(lv.x); cudaFree(lv.b); cudaFree(lv.t); cudaFree(lv.s);
  }
  cudaFree(P->Ainv32); cudaFree(P->r32); cudaFree(P->z32);
  if (P->iter_exec) cudaGraphExecDestroy(P->iter_exec);
  if (P->cs) cudaStreamDestroy(P->cs);
  cudaFree(P->Ainv); cudaFree(P->pc_r); cudaFree(P->pc_z); cudaFree(P->pc_p); cudaFree(P->pc_q);
  cudaFree(P->rhs); cudaFree(P->partial); cudaFree(P->scal); cudaFreeHost(P->h_scal);
  cudaFree(P->p_prev); cudaFree(P->ir);
  delete P;
}

double* proj_pressure(void* h) { return ((ProjCtx*)h)->p_prev; }
const double* proj_inv_rho(void* h) { return ((ProjCtx*)h)->ir; }
int proj_nlevels(void* h) { return ((ProjCtx*)h)->nlev; }

__global__ void k_cvt_d2f(int64_t n, const double* __restrict__ a, float* b, const double* done) {
  PCG_SKIP(done);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) b[c] = (float)a[c];
}
__global__ void k_cvt_f2d(int64_t n, const float* __restrict__ a, double* b, const double* done) {
  PCG_SKIP(done);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < n) b[c] = (double)a[c];
}

template <typename T>
static void rebuild_levels(ProjCtx* P, MGLevelT<T>* lev, T* Ainv, cudaStream_t st) {
  for (int l = 0; l < P->nlev; ++l) {
    MGLevelT<T>& f = lev[l];
    if (l > 0) {
      MGLevelT<T>& pf = lev[l - 1];
      k_mg_coarsen<T><<<blocks_for(f.n, 128), 128, 0, st>>>(pf.nx, pf.ny, pf.nz, pf.gx, pf.gy,
                                                           pf.gz, pf.e, f.dims, f.gx,
                                                           f.gy, f.gz, f.e, 0.5);
      fs_count_launch();
    }
    k_mg_diag<T><<<blocks_for(f.n, 256), 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e,
                                                       f.dinv);
    fs_count_launch();
  }
  MGLevelT<T>& c = lev[P->nlev - 1];
  if (c.n <= MG_COARSE_MAX) {
    k_mg_coarse_inverse<T><<<1, 64, 0, st>>>(c.nx, c.ny, c.nz, c.gx, c.gy, c.gz, c.e, Ainv);
    fs_count_launch();
  }
}

int proj_rebuild(void* h, const double* rho, cudaStream_t st) {
  ProjCtx* P = (ProjCtx*)h;
  const GridDev& g = P->g;
  MGLevel& l0 = P->lev[0];
  Launch3 L = launch_cells(g);
  k_proj_level0<<<L.grid, L.block, 0, st>>>(g, rho, P->ir, l0.gx, l0.gy, l0.gz, l0.e,
                                            g.dx * g.dx, g.dy * g.dy); fs_count_launch();
  if (P->fp32) {
    // the FP64 level-0 operator stays the CG's; the preconditioner gets an FP32 copy
    MGLevelT<float>& f0 = P->lev32[0];
    const double* src[4] = {l0.gx, l0.gy, l0.gz, l0.e};
    float* dst[4] = {f0.gx, f0.gy, f0.gz, f0.e};
    for (int q = 0; q < 4; ++q) {
      k_cvt_d2f<<<blocks_for(l0.n, 256), 256, 0, st>>>(l0.n, src[q], dst[q], nullptr);
      fs_count_launch();
    }
    rebuild_levels<float>(P, P->lev32, P->Ainv32, st);
  } else {
    rebuild_levels<double>(P, P->lev, P->Ainv, st);
  }
  return cuda_status();
}

int proj_set_precision(void* h, int fp32) {
  ProjCtx* P = (ProjCtx*)h;
  fp32 = fp32 ? 1 : 0;
  if (fp32 == P->fp32) return FS_OK;
  if (fp32 && !P->lev32[0].gx) {
    for (int l = 0; l < P->nlev; ++l) {
      MGLevelT<float>& lv = P->lev32[l];
      const MGLevel& ld = P->lev[l];
      lv.nx = ld.nx; lv.ny = ld.ny; lv.nz = ld.nz; lv.n = ld.n; lv.dims = ld.dims;
      float** arrs[9] = {&lv.gx, &lv.gy, &lv.gz, &lv.e, &lv.dinv, &lv.x, &lv.b, &lv.t, &lv.s};
      for (float** a : arrs)
        if (cudaMalloc(a, sizeof(float) * (size_t)(lv.n > 0 ? lv.n : 1)) != cudaSuccess)
          return FS_ECUDA;
    }
    const int64_t nc = P->lev[P->nlev - 1].n;
    if (cudaMalloc(&P->Ainv32, sizeof(float) * (size_t)(nc <= MG_COARSE_MAX ? nc * nc : 1)) !=
            cudaSuccess ||
        cudaMalloc(&P->r32, sizeof(float) * P->lev[0].n) != cudaSuccess ||
        cudaMalloc(&P->z32, sizeof(float) * P->lev[0].n) != cudaSuccess)
      return FS_ECUDA;
  }
  P->fp32 = fp32;
  if (P->iter_exec) cudaGraphExecDestroy(P->iter_exec);  // the iteration graph changes
  P->iter_exec = nullptr;
  P->graph_failed = 0;
  return FS_OK;
}

// z = V-cycle(r) on level l (b = rhs, x = result); returns kernels launched
// ---------------------------------------------------------------------------
// The coarse end of the V-cycle in one launch: every level from the first one
// whose tail fits in shared memory (operator, right-hand sides and vectors of
// all coarser levels, plus the coarsest level's dense inverse) down to the
// coarsest and back, in one CTA, with a __syncthreads between the sweeps,
// instead of one launch per sweep (a few microseconds of launch and drain
// each for a few hundred cells).  The first tail level's right-hand side
// comes from global memory and its correction goes back there.  The order of
// operations and every per-cell expression are those of vcycle() with
// k_mg_jacobi, k_mg_restrict_residual, k_mg_coarse_solve and k_mg_prolong, so
// the correction is bit-identical.
#define MG_TAIL_SMEM (200 * 1024)
#define MG_TAIL_MAX 10
#define MG_TAIL_THREADS 512
template <typename T>
struct MGTail {
  MGLevelT<T> lev[MG_TAIL_MAX];  // the tail's levels (global arrays), finest first
  int nl, nu;
  double omega;
  const T* Ainv;
};

// elements of shared memory the tail of levels lev[0..nl-1] needs
template <typename T>
__host__ __device__ inline int64_t tail_smem_elems(const MGLevelT<T>* lev, int nl) {
  int64_t e = 0;
  for (int q = 0; q < nl; ++q) e += 9 * lev[q].n;
  const int64_t nc = lev[nl - 1].n;
  return e + (nc <= MG_COARSE_MAX ? nc * nc : 0);
}

template <typename T>
__device__ __forceinline__ T tail_apply(const MGLevelT<T>& f, const T* x, int64_t c, int i,
                                        int j, int k) {
  const int nx = f.nx, ny = f.ny, nz = f.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const T xc = x[c];
  T y = f.e[c] * xc;
  if (i < nx - 1) y += f.gx[c] * (xc - x[c + 1]);
  if (i > 0) y += f.gx[c - 1] * (xc - x[c - 1]);
  if (ny > 1) {
    int jp = j + 1 < ny ? j + 1 : 0;
    int jm = j > 0 ? j - 1 : ny - 1;
    int64_t cp = c - (int64_t)j * sy + (int64_t)jp * sy;
    int64_t cm = c - (int64_t)j * sy + (int64_t)jm * sy;
    y += f.gy[c] * (xc - x[cp]);
    y += f.gy[cm] * (xc - x[cm]);
  }
  if (k < nz - 1) y += f.gz[c] * (xc - x[c + sz]);
  if (k > 0) y += f.gz[c - sz] * (xc - x[c - sz]);
  return y;
}

template <typename T>
__device__ __forceinline__ void tail_jacobi(const MGLevelT<T>& f, const T* b, const T* x, T* xo,
                                            T w) {
  for (int64_t c = threadIdx.x; c < f.n; c += blockDim.x) {
    if (!x) {
      xo[c] = w * b[c] * f.dinv[c];
      continue;
    }
    int i, j, k;
    split_cell((uint32_t)c, f.dims.fnx, f.dims.fny, i, j, k);
    T r = b[c] - tail_apply(f, x, c, i, j, k);
    xo[c] = x[c] + w * r * f.dinv[c];
  }
}

template <typename T>
__global__ void __launch_bounds__(MG_TAIL_THREADS, 1)
    k_mg_vcycle_tail(MGTail<T> a, const double* done) {
  PCG_SKIP(done);
  extern __shared__ __align__(16) unsigned char tsh[];
  T* sp = (T*)tsh;
  // the levels in shared memory: operator copied in, vectors private
  MGLevelT<T> L[MG_TAIL_MAX];
  for (int q = 0; q < a.nl; ++q) {
    const MGLevelT<T>& g = a.lev[q];
    const int64_t n = g.n;
    MGLevelT<T>& f = L[q];
    f.nx = g.nx; f.ny = g.ny; f.nz = g.nz; f.n = n; f.dims = g.dims;
    f.gx = sp; f.gy = sp + n; f.gz = sp + 2 * n; f.e = sp + 3 * n; f.dinv = sp + 4 * n;
    f.b = sp + 5 * n; f.x = sp + 6 * n; f.t = sp + 7 * n; f.s = sp + 8 * n;
    sp += 9 * n;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) {
      f.gx[c] = g.gx[c]; f.gy[c] = g.gy[c]; f.gz[c] = g.gz[c]; f.e[c] = g.e[c];
      f.dinv[c] = g.dinv[c];
      if (q == 0) f.b[c] = g.b[c];
    }
  }
  const int64_t ncs = L[a.nl - 1].n;
  T* Ainv = sp;
  if (ncs <= MG_COARSE_MAX)
    for (int64_t c = threadIdx.x; c < ncs * ncs; c += blockDim.x) Ainv[c] = a.Ainv[c];
  __syncthreads();
  const T w = (T)a.omega;
  const int nu = a.nu;
  // down: pre-smoothing from x = 0 ending in t, residual restricted to the next level's b
  for (int l = 0; l + 1 < a.nl; ++l) {
    const MGLevelT<T>& f = L[l];
    const T* src = nullptr;
    for (int s = 0; s < nu; ++s) {
      T* dst = ((nu - 1 - s) % 2 == 0) ? f.t : f.s;
      tail_jacobi(f, f.b, src, dst, w);
      __syncthreads();
      src = dst;
    }
    const MGLevelT<T>& cl = L[l + 1];
    const int64_t fsy = f.nx, fsz = (int64_t)f.nx * f.ny;
    for (int64_t q = threadIdx.x; q < cl.n; q += blockDim.x) {
      int I, J, K;
      split_cell((uint32_t)q, cl.dims.fnx, cl.dims.fny, I, J, K);
      T sum = 0.0;
      for (int k = 2 * K; k <= min(2 * K + 1, f.nz - 1); ++k)
        for (int j = 2 * J; j <= min(2 * J + 1, f.ny - 1); ++j)
          for (int i = 2 * I; i <= min(2 * I + 1, f.nx - 1); ++i) {
            int64_t c = (int64_t)k * fsz + (int64_t)j * fsy + i;
            sum += f.b[c] - tail_apply(f, f.t, c, i, j, k);
          }
      cl.b[q] = sum;
    }
    __syncthreads();
  }
  // coarsest level: dense solve, or smoothing only when it is too large for it
  {
    const MGLevelT<T>& f = L[a.nl - 1];
    if (f.n <= MG_COARSE_MAX) {
      for (int r = threadIdx.x; r < (int)f.n; r += blockDim.x) {
        T sum = 0.0;
        for (int q = 0; q < (int)f.n; ++q) sum += Ainv[r * f.n + q] * f.b[q];
        f.x[r] = sum;
      }
      __syncthreads();
    } else {
      const T wc = (T)MG_OMEGA;
      tail_jacobi(f, f.b, (const T*)nullptr, f.x, wc);
      __syncthreads();
      for (int s = 0; s < 8; ++s) {
        const T* src = (s & 1) ? f.t : f.x;
        T* dst = (s & 1) ? f.x : f.t;
        tail_jacobi(f, f.b, src, dst, wc);
        __syncthreads();
      }
    }
  }
  // up: prolongation into t, post-smoothing from t ending in the level's x
  for (int l = a.nl - 2; l >= 0; --l) {
    const MGLevelT<T>& f = L[l];
    const MGLevelT<T>& cl = L[l + 1];
    for (int64_t c = threadIdx.x; c < f.n; c += blockDim.x) {
      int i, j, k;
      split_cell((uint32_t)c, f.dims.fnx, f.dims.fny, i, j, k);
      f.t[c] += cl.x[((int64_t)(k >> 1) * cl.ny + (j >> 1)) * cl.nx + (i >> 1)];
    }
    __syncthreads();
    const T* src = f.t;
    for (int s = 0; s < nu; ++s) {
      T* dst = (s == nu - 1) ? f.x : ((s % 2 == 0) ? f.s : f.t);
      tail_jacobi(f, f.b, src, dst, w);
      __syncthreads();
      src = dst;
    }
  }
  // the first tail level's correction back to global memory
  for (int64_t c = threadIdx.x; c < L[0].n; c += blockDim.x) a.lev[0].x[c] = L[0].x[c];
}

template <typename T>
static int vcycle(ProjCtx* P, MGLevelT<T>* lev, const T* Ainv, int l, const T* b, T* x,
                  const double* done, cudaStream_t st) {
  MGLevelT<T>& f = lev[l];
  int nk = 0;
  // the coarse end in one launch (its first level's b and x are the level's own)
  if (l > 0 && P->tail_on && P->nlev - l <= MG_TAIL_MAX && b == f.b && x == f.x &&
      tail_smem_elems(lev + l, P->nlev - l) * (int64_t)sizeof(T) <= MG_TAIL_SMEM) {
    MGTail<T> ta{};
    ta.nl = P->nlev - l;
    for (int q = 0; q < ta.nl; ++q) ta.lev[q] = lev[l + q];
    ta.nu = P->nu;
    ta.omega = P->omega;
    ta.Ainv = Ainv;
    const size_t smem = (size_t)tail_smem_elems(lev + l, ta.nl) * sizeof(T);
    cudaFuncSetAttribute(k_mg_vcycle_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         MG_TAIL_SMEM);
    k_mg_vcycle_tail<T><<<1, MG_TAIL_THREADS, smem, st>>>(ta, done);
    return 1;
  }
  if (l == P->nlev - 1) {
    if (f.n <= MG_COARSE_MAX) {
      k_mg_coarse_solve<T><<<1, 64, 0, st>>>((int)f.n, Ainv, b, x, done);
      ++nk;
    } else {
      // not coarsenable and too large for the dense solve: smoothing only
      k_mg_jacobi<T><<<blocks_for(f.n, 256), 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz,
                                                          f.e, f.dinv, b, nullptr, x, MG_OMEGA,
                                                          done);
      ++nk;
      for (int s = 0; s < 8; ++s) {
        const T* src = (s & 1) ? f.t : x;
        T* dst = (s & 1) ? x : f.t;
        k_mg_jacobi<T><<<blocks_for(f.n, 256), 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz,
                                                            f.e, f.dinv, b, src, dst, MG_OMEGA,
                                                            done);
        ++nk;
      }
    }
    return nk;
  }
  MGLevelT<T>& cl = lev[l + 1];
  unsigned nb = blocks_for(f.n, 256);
  const int nu = (l == 0 && P->nu0 > 0) ? P->nu0 : P->nu;
  const double om = P->omega;
  // pre-smoothing from x = 0, ending in t:  sweep i writes t when (nu-1-i) is even, else s
  const T* src = nullptr;
  for (int i = 0; i < nu; ++i) {
    T* dst = ((nu - 1 - i) % 2 == 0) ? f.t : f.s;
    k_mg_jacobi<T><<<nb, 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e, f.dinv, b, src,
                                       dst, om, done);
    src = dst;
    ++nk;
  }
  k_mg_restrict_residual<T><<<blocks_for(cl.n, 128), 128, 0, st>>>(
      f.dims, f.gx, f.gy, f.gz, f.e, b, f.t, cl.dims, cl.b, done);
  ++nk;
  nk += vcycle<T>(P, lev, Ainv, l + 1, cl.b, cl.x, done, st);
  k_mg_prolong<T><<<nb, 256, 0, st>>>(f.dims, f.t, cl.nx, cl.ny, cl.x, done);
  ++nk;
  // post-smoothing from t, ending in x:  s, t, s, ... then x
  src = f.t;
  for (int i = 0; i < nu; ++i) {
    T* dst = (i == nu - 1) ? x : ((i % 2 == 0) ? f.s : f.t);
    k_mg_jacobi<T><<<nb, 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e, f.dinv, b, src,
                                       dst, om, done);
    src = dst;
    ++nk;
  }
  return nk;
}


void proj_stats(void* h, double* out8) {
  ProjCtx* P = (ProjCtx*)h;
  for (int q = 0; q < 8; ++q) out8[q] = P->stats[q];
}

int proj_configure(void* h, int nu, double omega) {
  ProjCtx* P = (ProjCtx*)h;
  if (nu < 1 || nu > 16 || !(omega > 0.0 && omega < 2.0)) return FS_EARG;
  if (nu != P->nu || omega != P->omega) {
    P->nu = nu;
    P->omega = omega;
    if (P->iter_exec) cudaGraphExecDestroy(P->iter_exec);
    P->iter_exec = nullptr;
    P->graph_failed = 0;
  }
  return FS_OK;
}

int proj_set_fine_sweeps(void* h, int nu0) {
  ProjCtx* P = (ProjCtx*)h;
  if (nu0 < 0 || nu0 > 16) return FS_EARG;
  if (nu0 != P->nu0) {
    P->nu0 = nu0;
    if (P->iter_exec) cudaGraphExecDestroy(P->iter_exec);
    P->iter_exec = nullptr;
    P->graph_failed = 0;
  }
  return FS_OK;
}

int proj_set_coarse_tail(void* h, int on) {
  ProjCtx* P = (ProjCtx*)h;
  if ((on != 0) != (P->tail_on != 0)) {
    P->tail_on = on ? 1 : 0;
    if (P->iter_exec) cudaGraphExecDestroy(P->iter_exec);
    P->iter_exec = nullptr;
    P->graph_failed = 0;
  }
  return FS_OK;
}

// One preconditioned-CG iteration, every kernel a no-op once converged.
static int pcg_iteration(ProjCtx* P, double* x, cudaStream_t st) {
  MGLevel& l0 = P->lev[0];
  const int64_t n = l0.n;
  const double* done = P->scal + SC_DONE;
  int nk;
  if (P->fp32) {
    k_cvt_d2f<<<blocks_for(n, 256), 256, 0, st>>>(n, P->pc_r, P->r32, done);
    nk = vcycle<float>(P, P->lev32, P->Ainv32, 0, P->r32, P->z32, done, st);
    k_cvt_f2d<<<blocks_for(n, 256), 256, 0, st>>>(n, P->z32, P->pc_z, done);
    nk += 2;
  } else {
    nk = vcycle<double>(P, P->lev, P->Ainv, 0, P->pc_r, P->pc_z, done, st);
  }
  k_dot<<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, P->pc_r, P->pc_z, P->partial, done);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 2, done);  // rz_new
  k_pcg_dir<<<blocks_for(n, 256), 256, 0, st>>>(n, P->scal, P->pc_z, P->pc_p);
  k_set_scal<<<1, 1, 0, st>>>(P->scal, 0, 2);  // rz = rz_new
  k_pcg_matvec<<<RED_BLOCKS, RED_THREADS, 0, st>>>(l0.dims, l0.gx, l0.gy, l0.gz,
                                                   l0.e, P->pc_p, P->pc_q, P->partial, done);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 1, done);  // pq
  k_pcg_update<<<RED_BLOCKS, RED_THREADS, 0, st>>>(P->g, P->scal, x, P->pc_r, P->pc_p, P->pc_q,
                                                   P->partial);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 5, done);  // ||r_A||^2
  k_pcg_check<<<1, 1, 0, st>>>(P->scal);
  return nk + 10;
}

// Capture one iteration as a CUDA graph (on the context's private stream).
static void capture_iteration(ProjCtx* P) {
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(P->cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    P->graph_failed = 1;
    return;
  }
  int nk = pcg_iteration(P, P->p_prev, P->cs);
  if (cudaStreamEndCapture(P->cs, &graph) != cudaSuccess || !graph) {
    cudaGetLastError();
    P->graph_failed = 1;
    return;
  }
  if (cudaGraphInstantiate(&P->iter_exec, graph, 0) != cudaSuccess) {
    cudaGetLastError();
    P->iter_exec = nullptr;
    P->graph_failed = 1;
  }
  cudaGraphDestroy(graph);
  P->iter_kernels = nk;
}

static int launch_iterations(ProjCtx* P, int count, cudaStream_t st) {
  for (int q = 0; q < count; ++q) {
    if (P->iter_exec) {
      if (cudaGraphLaunch(P->iter_exec, st) != cudaSuccess) return FS_ECUDA;
      for (int k = 0; k < P->iter_kernels; ++k) fs_count_launch();
    } else {
      int nk = pcg_iteration(P, P->p_prev, st);
      for (int k = 0; k < nk; ++k) fs_count_launch();
    }
  }
  return FS_OK;
}

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

static int fetch(ProjCtx* P, int n, cudaStream_t st) {
  const auto t0 = Clock::now();
  cudaMemcpyAsync(P->h_scal, P->scal, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  const int rc = fs_stream_wait(st) != FS_OK ? FS_ECUDA : FS_OK;
  const double w = ms_since(t0);
  P->stats[1] += w;
  if (w > P->stats[2]) P->stats[2] = w;
  P->stats[5] += 1.0;
  return rc;
}

// Pre-smoothing of the learned preconditioner: nu damped-Jacobi sweeps on
// the FP32 level-0 operator from x = 0 for S t = r32, ending in f.t (the
// V-cycle's first half at level 0); then f.b = r32 - S t.
static void lp_presmooth(ProjCtx* P, cudaStream_t st) {
  MGLevelT<float>& f = P->lev32[0];
  const unsigned nb = blocks_for(f.n, 256);
  const float* src = nullptr;
  for (int i = 0; i < P->nu; ++i) {
    float* dst = ((P->nu - 1 - i) % 2 == 0) ? f.t : f.s;
    k_mg_jacobi<float><<<nb, 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e, f.dinv,
                                           P->r32, src, dst, P->omega, nullptr);
    src = dst;
    fs_count_launch();
  }
  k_lp_residual<float><<<nb, 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e, P->r32, f.t,
                                           f.b);
  fs_count_launch();
}

// The learned preconditioner z = M(r), a two-level cycle whose coarse
// correction is the network: pre-smoothing (lp_presmooth), s = t + N(r1)
// (the network's estimate of S^-1 r1, scaled back), then nu post-smoothing
// sweeps from s.  The sweeps remove the high-frequency part of the network's
// error, which the residual norm would otherwise be dominated by.
static int learned_precond(ProjCtx* P, cudaStream_t st) {
  MGLevelT<float>& f = P->lev32[0];
  const int64_t n = f.n;
  const unsigned nb = blocks_for(n, 256);
  k_cvt_d2f<<<nb, 256, 0, st>>>(n, P->pc_r, P->r32, nullptr);
  fs_count_launch();
  lp_presmooth(P, st);
  int rc = unet_correct(P->net, f.b, f.t, f.s, st);
  if (rc) return rc;
  const float* src = f.s;
  for (int i = 0; i < P->nu; ++i) {
    float* dst = (i == P->nu - 1) ? P->z32 : ((i % 2 == 0) ? f.t : f.x);
    k_mg_jacobi<float><<<nb, 256, 0, st>>>(f.dims, f.gx, f.gy, f.gz, f.e, f.dinv,
                                           P->r32, src, dst, P->omega, nullptr);
    src = dst;
    fs_count_launch();
  }
  k_cvt_f2d<<<nb, 256, 0, st>>>(n, P->z32, P->pc_z, nullptr);
  fs_count_launch();
  return cuda_status();
}

// Training pair for the network from a logged solve (r0, e0 with S e0 = r0):
// the residual after pre-smoothing and the error left, r1 = r0 - S t and
// e1 = e0 - t, in FP32 (the operator of the last rebuild).
int proj_smooth_pair(void* h, const double* r0, const double* e0, float* r1, float* e1,
                     cudaStream_t st) {
  ProjCtx* P = (ProjCtx*)h;
  if (!P->fp32) return FS_EARG;
  MGLevelT<float>& f = P->lev32[0];
  const int64_t n = f.n;
  const unsigned nb = blocks_for(n, 256);
  k_cvt_d2f<<<nb, 256, 0, st>>>(n, r0, P->r32, nullptr);
  fs_count_launch();
  lp_presmooth(P, st);
  cudaMemcpyAsync(r1, f.b, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
  k_lp_err<<<nb, 256, 0, st>>>(n, e0, f.t, e1);
  fs_count_launch();
  return cuda_status();
}

// One flexible-CG iteration with the learned preconditioner (kernels as in
// pcg_iteration; the host reads the scalars after every iteration).
static int fcg_iteration(ProjCtx* P, double* x, int it, cudaStream_t st) {
  MGLevel& l0 = P->lev[0];
  const int64_t n = l0.n;
  const double* done = P->scal + SC_DONE;
  int rc = learned_precond(P, st);
  if (rc) return rc;
  if (it > 0) {
    k_dot<<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, P->pc_z, P->pc_q, P->partial, done);
    k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 10, done);  // z.q_prev
    fs_count_launch(); fs_count_launch();
  }
  k_fcg_dir<<<blocks_for(n, 256), 256, 0, st>>>(n, P->scal, P->pc_z, P->pc_p);
  k_pcg_matvec<<<RED_BLOCKS, RED_THREADS, 0, st>>>(l0.dims, l0.gx, l0.gy, l0.gz,
                                                   l0.e, P->pc_p, P->pc_q, P->partial, done);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 1, done);  // p.q
  k_dot<<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, P->pc_p, P->pc_r, P->partial, done);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 12, done);  // p.r
  k_fcg_alpha<<<1, 1, 0, st>>>(P->scal);  // alpha = p.r / p.q
  k_pcg_update<<<RED_BLOCKS, RED_THREADS, 0, st>>>(P->g, P->scal, x, P->pc_r, P->pc_p, P->pc_q,
                                                   P->partial);
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 5, done);  // ||r_A||^2
  k_set_scal<<<1, 1, 0, st>>>(P->scal, 11, 1);
  k_pcg_check<<<1, 1, 0, st>>>(P->scal);
  for (int k = 0; k < 10; ++k) fs_count_launch();
  return cuda_status();
}

// Learned iterations until convergence, a stall or max_learned; on a stall
// the residual is recomputed and the scalars reset so that the V-cycle PCG
// loop continues from the current iterate.
static int fcg_solve(ProjCtx* P, double* x, int maxiter, int* learned, cudaStream_t st) {
  const GridDev& g = P->g;
  MGLevel& l0 = P->lev[0];
  std::vector<double> rn;
  int it = 0;
  while (true) {
    int stt = fetch(P, 9, st);
    if (stt) return stt;
    const double bn2 = P->h_scal[4], rn2 = P->h_scal[5];
    if (!(bn2 == bn2) || !(rn2 == rn2)) return FS_ENONFINITE;
    if (P->h_scal[SC_DONE] != 0.0) break;
    rn.push_back(rn2);
    bool fall = it >= P->max_learned || it >= maxiter;
    if (!fall && it >= 3) {
      const double f = std::pow(rn2 / rn[it - 3], 1.0 / 6.0);  // per-iteration norm factor
      fall = !(f < P->stall);
    }
    if (fall) {
      k_pcg_residual<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, l0.gx, l0.gy, l0.gz, l0.e, P->rhs, x,
                                                         P->pc_r, P->partial);
      k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 5, nullptr);
      k_fcg_restart<<<1, 1, 0, st>>>(P->scal);
      fs_count_launch(); fs_count_launch(); fs_count_launch();
      P->fcg[2] = 1.0;
      P->fcg[3] += 1.0;
      break;
    }
    stt = fcg_iteration(P, x, it, st);
    if (stt) return stt;
    ++it;
  }
  *learned = it;
  P->fcg[0] = it;
  return cuda_status();
}

int proj_set_learned(void* h, void* net, int max_learned, double stall) {
  ProjCtx* P = (ProjCtx*)h;
  if (max_learned < 0 || !(stall > 0.0 && stall <= 1.0)) return FS_EARG;
  // the learned cycle runs on the FP32 level-0 operator of the mixed form
  if (net && (!P->fp32 || unet_cells(net) != P->lev[0].n)) return FS_EARG;
  P->net = net;
  P->max_learned = max_learned;
  P->stall = stall;
  return FS_OK;
}

int proj_set_log(void* h, double* r0, double* x0) {
  ProjCtx* P = (ProjCtx*)h;
  if ((r0 == nullptr) != (x0 == nullptr)) return FS_EARG;
  P->log_r0 = r0;
  P->log_x0 = x0;
  return FS_OK;
}

void proj_fcg_stats(void* h, double* out4) {
  ProjCtx* P = (ProjCtx*)h;
  for (int q = 0; q < 4; ++q) out4[q] = P->fcg[q];
}

// Solve for the pressure and correct u, v, w in place.  The iterations run
// as graph launches in batches (sized from the previous solve's count); the
// host reads the converged flag once per batch.
int proj_project(void* h, double* u, double* v, double* w, const double* u_in,
                 const double* target, double dt, double rtol, int maxiter, int* iters,
                 cudaStream_t st) {
  ProjCtx* P = (ProjCtx*)h;
  const GridDev& g = P->g;
  MGLevel& l0 = P->lev[0];
  const int64_t n = l0.n;
  const auto t_start = Clock::now();
  for (int q = 0; q < 8; ++q) P->stats[q] = 0.0;
  *iters = 0;
  k_proj_rhs<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, u, v, w, u_in, target, dt, P->rhs,
                                                 P->partial); fs_count_launch();
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 4, nullptr); fs_count_launch();
  double* x = P->p_prev;
  k_pcg_residual<<<RED_BLOCKS, RED_THREADS, 0, st>>>(g, l0.gx, l0.gy, l0.gz, l0.e, P->rhs, x,
                                                     P->pc_r, P->partial); fs_count_launch();
  k_finish_sums<<<1, 32, 0, st>>>(P->partial, 1, P->scal + 5, nullptr); fs_count_launch();
  k_pcg_init<<<1, 1, 0, st>>>(P->scal, rtol * rtol); fs_count_launch();
  k_zero_if_zero_rhs<<<blocks_for(n, 256), 256, 0, st>>>(n, P->scal, x); fs_count_launch();
  if (P->log_r0) {
    cudaMemcpyAsync(P->log_r0, P->pc_r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(P->log_x0, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  }
  int learned = 0;
  P->fcg[0] = P->fcg[1] = P->fcg[2] = 0.0;
  if (P->net) {
    int stt = fcg_solve(P, x, maxiter, &learned, st);
    if (stt) return stt;
  }
  if (!P->iter_exec && !P->graph_failed) capture_iteration(P);
  int launched = learned;
  int batch = P->last_iters > 2 ? P->last_iters - 2 : 1;
  while (true) {
    int stt = fetch(P, 9, st);
    if (stt) return stt;
    const double bn2 = P->h_scal[4], rn2 = P->h_scal[5];
    if (!(bn2 == bn2) || !(rn2 == rn2)) return FS_ENONFINITE;
    if (P->h_scal[SC_DONE] != 0.0) break;
    if (launched >= maxiter) return FS_ENOCONV;
    if (batch > maxiter - launched) batch = maxiter - launched;
    const auto tl = Clock::now();
    stt = launch_iterations(P, batch, st);
    const double lw = ms_since(tl);
    P->stats[3] += lw;
    if (lw > P->stats[4]) P->stats[4] = lw;
    if (stt) return stt;
    launched += batch;
    P->stats[6] += batch;
    batch = 2;
  }
  if (P->net && P->fcg[2] != 0.0) P->fcg[1] = P->h_scal[SC_IT];
  *iters = P->fcg[2] != 0.0 ? learned + (int)P->h_scal[SC_IT] : (int)P->h_scal[SC_IT];
  P->last_iters = *iters;
  P->stats[7] = *iters;
  P->stats[0] = ms_since(t_start);
  P->have_prev = 1;
  Launch3 L = launch_cells(g);
  k_proj_correct<<<L.grid, L.block, 0, st>>>(g, u, v, w, x, P->ir, dt); fs_count_launch();
  return cuda_status();
}

int launch_div_resid_max(const GridDev& g, const double* u, const double* v, const double* w,
                         const double* u_in, const double* target, double* div_out,
                         unsigned long long* out_key, cudaStream_t st) {
  cudaMemsetAsync(out_key, 0, sizeof(unsigned long long), st);
  int64_t n = ncells(g);
  unsigned nb = blocks_for(n, 256);
  if (nb > 1184) nb = 1184;
  k_div_resid_max<<<nb, 256, 0, st>>>(g, u, v, w, u_in, target, div_out, out_key); fs_count_launch();
  return cuda_status();
}

// apply the symmetrised operator to x (test hook): y = S x  and A x = -y / dz
int proj_apply(void* h, const double* x, double* y, cudaStream_t st) {
  ProjCtx* P = (ProjCtx*)h;
  MGLevel& l0 = P->lev[0];
  k_pcg_matvec<<<RED_BLOCKS, RED_THREADS, 0, st>>>(l0.dims, l0.gx, l0.gy, l0.gz, l0.e,
                                                   x, y, P->partial, nullptr); fs_count_launch();
  return cuda_status();
}
