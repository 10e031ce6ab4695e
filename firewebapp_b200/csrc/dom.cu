// Discrete-ordinates radiation (dom_3d.py:286-473 DOMRadiationSolver.solve).
//
// Each source iteration sweeps every ordinate with step differencing
// (dom_3d.py:147-211).  Within one ordinate the upwind dependencies run along
// +-x, +-y, +-z, so all cells on a hyperplane i'+j'+k' = d (sweep-direction
// coordinates) are independent; one launch per hyperplane processes that
// plane for all ordinates of all octants at once.  The y-periodic inflow at
// the first row reads the intensity left by the previous sweep at the other
// end of the row, exactly as the reference's in-place sweep does (the source
// cell sits on a later hyperplane, so it is still the previous value).
// Intensities persist across calls (the reference keeps I_set).
#include <vector>
#include <cstring>
#include <utility>
#include "common.cuh"
#include "kernels.h"

#define PI_D 3.141592653589793
#define SIGMA_SB_D 5.67e-8

struct DomCtx {
  GridDev g;
  int M;
  double *ox, *oy, *oz, *w;  // device ordinates and weights
  std::vector<double> hox, hoy, hoz, hw;
  double* I;                  // M * N
  double *G, *Gp;             // current / previous G
  double *ks, *kg, *ksafe, *B;
  double *Ig_out, *Isoil, *qin;  // (Ny, Nx)
  unsigned long long* keys;      // reduction slots
  unsigned long long* h_keys;
  double eps_w, tol, relax, kgmax;
  int max_iter;
  int last_iters;
  // optional per-sweep timing (CUDA events on the launching stream)
  int timing;
  cudaEvent_t ev0[32], ev1[32];
  double sweep_ms;
  long long sweep_count;
};

__device__ __forceinline__ double clip01(double x) {
  if (x < 0.0) x = 0.0;
  if (x > 1.0) x = 1.0;
  return x;
}

__global__ void k_dom_setup(GridDev g, const double* __restrict__ Ts, const double* __restrict__ Tg,
                            const double* __restrict__ as, const double* __restrict__ om,
                            const double* __restrict__ YH, const double* __restrict__ rho,
                            const double* __restrict__ Mloc, double sigma, double Tamb4,
                            double kgmax, double* ks, double* kg, double* ksafe, double* B) {
  int64_t n = ncells_dev(g);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double ksol = sigma * as[c];
  if (Mloc) ksol = ksol * (1.0 + 5.0 * Mloc[c]);
  double of = clip01(om[c] / 1.0e-3);
  double tf = clip01((Tg[c] - 600.0) / 400.0);
  double mx = (of >= tf || of != of) ? of : tf;
  double kgas = kgmax * mx;
  if (YH && rho) kgas = kgas + 30.0 * rho[c] * YH[c];
  double kap = ksol + kgas;
  double ksf = (kap >= 1.0e-3 || kap != kap) ? kap : 1.0e-3;
  double T4;
  if (kap > 1.0e-9) {
    T4 = (ksol * pow(Ts[c], 4.0) + kgas * pow(Tg[c], 4.0)) / ksf;
  } else {
    T4 = Tamb4;
  }
  ks[c] = ksol;
  kg[c] = kgas;
  ksafe[c] = ksf;
  B[c] = SIGMA_SB_D * T4 / PI_D;
}

__global__ void k_dom_ground_init(int n2, const double* __restrict__ Tsoil, double eps_w,
                                  double I_amb, double* Isoil, double* Ig) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  double e = Tsoil ? eps_w * SIGMA_SB_D * pow(Tsoil[q], 4.0) / PI_D : eps_w * I_amb;
  Isoil[q] = e;
  Ig[q] = e;
}

struct SweepArgs {
  const double *ox, *oy, *oz;
  double* I;
  const double *ksafe, *B, *Ig;
  double I_amb, inv_dx, inv_dy;
  int M;
  int plane;
  int periodic;
};

__global__ void k_dom_plane(GridDev g, SweepArgs a) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t plane_cells = (int64_t)ny * nz;
  int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (tid >= plane_cells * a.M) return;
  const int n = (int)(tid / plane_cells);
  const int64_t rem = tid - (int64_t)n * plane_cells;
  const int kp = (int)(rem / ny);
  const int jp = (int)(rem - (int64_t)kp * ny);
  const int ip = a.plane - jp - kp;
  if (ip < 0 || ip >= nx) return;
  const double xi = a.ox[n], eta = a.oy[n], mu = a.oz[n];
  const int i = xi >= 0.0 ? ip : nx - 1 - ip;
  const int j = eta >= 0.0 ? jp : ny - 1 - jp;
  const int k = mu >= 0.0 ? kp : nz - 1 - kp;
  const int64_t N = ncells_dev(g);
  double* I = a.I + (int64_t)n * N;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int64_t c = cidx(g, k, j, i);
  double Ix, Iy, Iz;
  if (xi >= 0.0) Ix = i > 0 ? I[c - 1] : a.I_amb;
  else Ix = i < nx - 1 ? I[c + 1] : a.I_amb;
  if (eta >= 0.0) {
    if (j > 0) Iy = I[c - sy];
    else Iy = a.periodic ? I[c + (int64_t)(ny - 1) * sy] : a.I_amb;
  } else {
    if (j < ny - 1) Iy = I[c + sy];
    else Iy = a.periodic ? I[c - (int64_t)(ny - 1) * sy] : a.I_amb;
  }
  if (mu >= 0.0) {
    Iz = k > 0 ? I[c - sz] : (mu > 0.0 ? a.Ig[(int64_t)j * nx + i] : 0.0);
  } else {
    Iz = k < nz - 1 ? I[c + sz] : a.I_amb;
  }
  const double ix = fabs(xi) * a.inv_dx;
  const double iy = fabs(eta) * a.inv_dy;
  const double iz = fabs(mu) / g.dz[k];
  const double kap = a.ksafe[c];
  double num = kap * a.B[c] + ix * Ix + iy * Iy + iz * Iz;
  double den = kap + ix + iy + iz;
  I[c] = num / den;
}

// One thread block sweeps one ordinate over the whole grid in hyperplane order.
// In sweep coordinates (i',j',k') every upwind neighbour of a cell on plane d
// lies on plane d-1 in the same (k',j') pencil (x), the (k',j'-1) pencil (y)
// or the (k'-1,j') pencil (z), so the block keeps, for every pencil, its value
// on the previous plane in shared memory (double buffered: plane d writes the
// buffer plane d-2 used).  Only the y-periodic inflow of the first row reads
// global memory: the previous sweep's value at the far end of the row, which
// this sweep overwrites only on a later plane.
__global__ void __launch_bounds__(1024) k_dom_sweep_block(GridDev g, SweepArgs a) {
  extern __shared__ double sh[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int npen = ny * nz;
  double* bufA = sh;
  double* bufB = sh + npen;
  const int n = blockIdx.x;
  const double xi = a.ox[n], eta = a.oy[n], mu = a.oz[n];
  const bool fx = xi >= 0.0, fy = eta >= 0.0, fz = mu >= 0.0;
  const double ix = fabs(xi) * a.inv_dx;
  const double iy = fabs(eta) * a.inv_dy;
  const double amu = fabs(mu);
  const int64_t N = ncells_dev(g);
  double* I = a.I + (int64_t)n * N;
  const int64_t sy = nx;
  const int nplanes = nx + ny + nz - 2;
  for (int d = 0; d < nplanes; ++d) {
    double* cur = (d & 1) ? bufB : bufA;
    const double* prev = (d & 1) ? bufA : bufB;
    // pencils on this plane: k' in [kp0, kp1], j' such that 0 <= d-j'-k' < nx
    const int kp0 = max(0, d - (nx - 1) - (ny - 1));
    const int kp1 = min(nz - 1, d);
    for (int q = kp0 * ny + threadIdx.x; q <= kp1 * ny + ny - 1; q += blockDim.x) {
      const int kp = q / ny;
      const int jp = q - kp * ny;
      const int ip = d - jp - kp;
      if (ip < 0 || ip >= nx) continue;
      const int i = fx ? ip : nx - 1 - ip;
      const int j = fy ? jp : ny - 1 - jp;
      const int k = fz ? kp : nz - 1 - kp;
      const int64_t c = cidx(g, k, j, i);
      const double Ix = ip > 0 ? prev[q] : a.I_amb;
      double Iy;
      if (jp > 0) Iy = prev[q - 1];
      else Iy = a.periodic ? I[c + (fy ? (int64_t)(ny - 1) * sy : -(int64_t)(ny - 1) * sy)]
                           : a.I_amb;
      double Iz;
      if (kp > 0) Iz = prev[q - ny];
      else if (fz) Iz = mu > 0.0 ? a.Ig[(int64_t)j * nx + i] : 0.0;
      else Iz = a.I_amb;
      const double iz = amu / g.dz[k];
      const double kap = a.ksafe[c];
      const double num = kap * a.B[c] + ix * Ix + iy * Iy + iz * Iz;
      const double den = kap + ix + iy + iz;
      const double v = num / den;
      cur[q] = v;
      I[c] = v;
    }
    __syncthreads();
  }
}

// G = sum_n w_n I_n (ordinate order); also max G and max |G - G_prev|
__global__ void k_dom_G(int64_t N, int M, const double* __restrict__ w,
                        const double* __restrict__ I, double* G, const double* __restrict__ Gp,
                        unsigned long long* keys) {
  unsigned long long bg = 0, bd = 0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N;
       c += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int n = 0; n < M; ++n) s += w[n] * I[(int64_t)n * N + c];
    G[c] = s;
    double d = fabs(s - Gp[c]);
    // keys for non-negative doubles (NaN maps above +inf)
    unsigned long long ks = (s != s) ? 0x7ff8000000000000ull
                                     : (unsigned long long)__double_as_longlong(s > 0.0 ? s : 0.0);
    unsigned long long kd = (d != d) ? 0x7ff8000000000000ull
                                     : (unsigned long long)__double_as_longlong(d);
    bg = ks > bg ? ks : bg;
    bd = kd > bd ? kd : bd;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_xor_sync(0xffffffffu, bg, o);
    bg = y > bg ? y : bg;
    y = __shfl_xor_sync(0xffffffffu, bd, o);
    bd = y > bd ? y : bd;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(keys, bg);
    atomicMax(keys + 1, bd);
  }
}

// q_in at the ground, new ground intensity with under-relaxation
__global__ void k_dom_ground(int n2, int M, const double* __restrict__ oz,
                             const double* __restrict__ w, const double* __restrict__ I, int64_t N,
                             const double* __restrict__ Isoil, double refl, double relax,
                             double* Ig, double* qin) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  double s = 0.0;
  for (int n = 0; n < M; ++n) {
    double mu = oz[n];
    if (mu < 0.0) s += w[n] * fabs(mu) * I[(int64_t)n * N + q];
  }
  qin[q] = s;
  double Inew = Isoil[q] + refl * s;
  Ig[q] = relax * Inew + (1.0 - relax) * Ig[q];
}

__global__ void k_dom_finish(GridDev g, const double* __restrict__ ks, const double* __restrict__ kg,
                             const double* __restrict__ ksafe, const double* __restrict__ B,
                             const double* __restrict__ G, double* qs, double* qg) {
  int64_t n = ncells_dev(g);
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  int k = (int)(c / ((int64_t)g.nx * g.ny));
  double kap = ks[c] + kg[c];
  double net = kap * (G[c] - 4.0 * PI_D * B[c]);
  double nph = net * g.dz[k];
  double fs = kap > 1.0e-9 ? ks[c] / ksafe[c] : 0.0;
  double fg = kap > 1.0e-9 ? kg[c] / ksafe[c] : 0.0;
  qs[c] = nph * fs;
  qg[c] = nph * fg;
}

__global__ void k_scale2(int n2, const double* __restrict__ a, double s, double* out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n2) out[q] = s * a[q];
}

void* dom_create(const GridDev& g, int M, const double* ox, const double* oy, const double* oz,
                 const double* w, double kgmax) {
  DomCtx* D = new DomCtx();
  D->g = g;
  D->M = M;
  D->hox.assign(ox, ox + M); D->hoy.assign(oy, oy + M); D->hoz.assign(oz, oz + M);
  D->hw.assign(w, w + M);
  int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  cudaMalloc(&D->ox, sizeof(double) * M); cudaMalloc(&D->oy, sizeof(double) * M);
  cudaMalloc(&D->oz, sizeof(double) * M); cudaMalloc(&D->w, sizeof(double) * M);
  cudaMemcpy(D->ox, ox, sizeof(double) * M, cudaMemcpyHostToDevice);
  cudaMemcpy(D->oy, oy, sizeof(double) * M, cudaMemcpyHostToDevice);
  cudaMemcpy(D->oz, oz, sizeof(double) * M, cudaMemcpyHostToDevice);
  cudaMemcpy(D->w, w, sizeof(double) * M, cudaMemcpyHostToDevice);
  cudaMalloc(&D->I, sizeof(double) * N * M);
  cudaMemset(D->I, 0, sizeof(double) * N * M);
  cudaMalloc(&D->G, sizeof(double) * N); cudaMalloc(&D->Gp, sizeof(double) * N);
  cudaMemset(D->G, 0, sizeof(double) * N);
  cudaMalloc(&D->ks, sizeof(double) * N); cudaMalloc(&D->kg, sizeof(double) * N);
  cudaMalloc(&D->ksafe, sizeof(double) * N); cudaMalloc(&D->B, sizeof(double) * N);
  cudaMalloc(&D->Ig_out, sizeof(double) * n2); cudaMalloc(&D->Isoil, sizeof(double) * n2);
  cudaMalloc(&D->qin, sizeof(double) * n2);
  cudaMalloc(&D->keys, sizeof(unsigned long long) * 4);
  cudaMallocHost(&D->h_keys, sizeof(unsigned long long) * 4);
  D->eps_w = 0.85; D->tol = 1.0e-3; D->relax = 0.7; D->kgmax = kgmax; D->max_iter = 30;
  D->last_iters = 0;
  D->timing = 0; D->sweep_ms = 0.0; D->sweep_count = 0;
  for (int q = 0; q < 32; ++q) {
    cudaEventCreate(&D->ev0[q]);
    cudaEventCreate(&D->ev1[q]);
  }
  if (cudaGetLastError() != cudaSuccess) {
    dom_destroy(D);
    return nullptr;
  }
  return D;
}

void dom_destroy(void* h) {
  DomCtx* D = (DomCtx*)h;
  if (!D) return;
  cudaFree(D->ox); cudaFree(D->oy); cudaFree(D->oz); cudaFree(D->w); cudaFree(D->I);
  cudaFree(D->G); cudaFree(D->Gp); cudaFree(D->ks); cudaFree(D->kg); cudaFree(D->ksafe);
  cudaFree(D->B); cudaFree(D->Ig_out); cudaFree(D->Isoil); cudaFree(D->qin); cudaFree(D->keys);
  cudaFreeHost(D->h_keys);
  for (int q = 0; q < 32; ++q) {
    cudaEventDestroy(D->ev0[q]);
    cudaEventDestroy(D->ev1[q]);
  }
  delete D;
}

void dom_set_timing(void* h, int on) {
  DomCtx* D = (DomCtx*)h;
  D->timing = on;
  D->sweep_ms = 0.0;
  D->sweep_count = 0;
}

void dom_sweep_stats(void* h, double* ms, long long* count) {
  DomCtx* D = (DomCtx*)h;
  *ms = D->sweep_ms;
  *count = D->sweep_count;
}

double* dom_intensity(void* h) { return ((DomCtx*)h)->I; }
double* dom_G(void* h) { return ((DomCtx*)h)->G; }
int dom_last_iters(void* h) { return ((DomCtx*)h)->last_iters; }

static double key_to_double(unsigned long long k) {
  double d;
  memcpy(&d, &k, sizeof(double));
  return d;
}

int dom_solve(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH, const double* rho,
              const double* Mloc, double* q_solid, double* q_gas, double* q_in_soil,
              cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const int M = D->M;
  const double Tamb4 = pow(T_amb, 4.0);
  k_dom_setup<<<blocks_for(N, 256), 256, 0, st>>>(g, Ts, Tg, as, om, YH, rho, Mloc, sigma, Tamb4,
                                                  D->kgmax, D->ks, D->kg, D->ksafe, D->B); fs_count_launch();
  const double I_amb = SIGMA_SB_D * Tamb4 / PI_D;
  k_dom_ground_init<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, Tsoil0, D->eps_w, I_amb, D->Isoil,
                                                        D->Ig_out); fs_count_launch();
  SweepArgs a{};
  a.ox = D->ox; a.oy = D->oy; a.oz = D->oz; a.I = D->I; a.ksafe = D->ksafe; a.B = D->B;
  a.Ig = D->Ig_out; a.I_amb = I_amb; a.inv_dx = 1.0 / g.dx; a.inv_dy = 1.0 / g.dy; a.M = M;
  a.periodic = 1;
  const int nplanes = g.nx + g.ny + g.nz - 2;
  const int64_t nthr = (int64_t)g.ny * g.nz * M;
  const double refl = (1.0 - D->eps_w) / PI_D;
  int it;
  const size_t smem = sizeof(double) * 2 * (size_t)g.ny * g.nz;
  int max_smem = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const bool block_sweep = smem <= (size_t)max_smem;
  if (block_sweep)
    cudaFuncSetAttribute(k_dom_sweep_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  for (it = 0; it < D->max_iter; ++it) {
    std::swap(D->G, D->Gp);
    if (block_sweep) {
      if (D->timing) cudaEventRecord(D->ev0[it], st);
      k_dom_sweep_block<<<M, 1024, smem, st>>>(g, a); fs_count_launch();
      if (D->timing) cudaEventRecord(D->ev1[it], st);
    } else {
      for (int d = 0; d < nplanes; ++d) {
        a.plane = d;
        k_dom_plane<<<blocks_for(nthr, 256), 256, 0, st>>>(g, a); fs_count_launch();
      }
    }
    cudaMemsetAsync(D->keys, 0, sizeof(unsigned long long) * 2, st);
    unsigned nb = blocks_for(N, 256);
    if (nb > 1184) nb = 1184;
    k_dom_G<<<nb, 256, 0, st>>>(N, M, D->w, D->I, D->G, D->Gp, D->keys); fs_count_launch();
    k_dom_ground<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, M, D->oz, D->w, D->I, N, D->Isoil,
                                                      refl, D->relax, D->Ig_out, D->qin); fs_count_launch();
    if (it > 0) {
      cudaMemcpyAsync(D->h_keys, D->keys, sizeof(unsigned long long) * 2, cudaMemcpyDeviceToHost,
                      st);
      if (cudaStreamSynchronize(st) != cudaSuccess) return FS_ECUDA;
      double Gmax = key_to_double(D->h_keys[0]);
      double dmax = key_to_double(D->h_keys[1]);
      if (Gmax != Gmax || dmax != dmax) return FS_ENONFINITE;
      if (Gmax < 1e-12) Gmax = 1e-12;
      if (dmax / Gmax < D->tol) { ++it; break; }
    }
  }
  D->last_iters = it;
  if (D->timing && block_sweep) {
    cudaEventSynchronize(D->ev1[it - 1]);
    for (int q = 0; q < it; ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, D->ev0[q], D->ev1[q]);
      D->sweep_ms += ms;
      D->sweep_count += 1;
    }
  }
  k_dom_finish<<<blocks_for(N, 256), 256, 0, st>>>(g, D->ks, D->kg, D->ksafe, D->B, D->G, q_solid,
                                                   q_gas); fs_count_launch();
  if (q_in_soil) {
    k_scale2<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, D->qin, D->eps_w, q_in_soil); fs_count_launch(); }
  return cuda_status();
}
