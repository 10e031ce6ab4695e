// Discrete-ordinates radiation (dom_3d.py:286-473 DOMRadiationSolver.solve).
//
// Each source iteration sweeps every ordinate with step differencing
// (dom_3d.py:147-211).  Within one ordinate the upwind dependencies run along
// +-x, +-y, +-z, so all cells on a hyperplane i'+j'+k' = d (sweep-direction
// coordinates) are independent.  The y-periodic inflow at the first row reads
// the intensity left by the previous sweep at the other end of the row, as
// the reference's in-place sweep does (that cell lies on a later hyperplane).
// That wrap row is the only part of the intensities that a later sweep reads,
// and it persists across calls as the reference's I_set does.
//
// Sweep paths (chosen at the first solve, or forced by fs_dom_set_sweep_mode):
//   1 octant clusters: one thread-block cluster per octant, the
//     cluster's CTAs split the k' rows; every thread owns one pencil (j',k')
//     and advances all ordinates of the octant on each hyperplane, reading
//     the previous hyperplane from shared memory.  The row below a CTA's
//     first row arrives from the upstream CTA through distributed shared
//     memory, handed over with mbarriers (point to point, so the CTAs run
//     as a skewed pipeline).  Kappa and kappa*B are loaded once per cell for
//     all ordinates of the octant, and the sweep emits the octant's partial
//     G (and ground flux) instead of storing intensities.
//   4 as 1, with one cluster-wide barrier per hyperplane instead.
//   2 one CTA per ordinate with the full intensity field stored (then G is
//     summed over ordinates in ordinate order).
//   3 one launch per hyperplane (any grid size).
//   5 one CTA per ordinate (as 2) with fixed pencils per thread, the inputs
//     of a hyperplane loaded in batches and the inflow rows staged ahead.
//   7 as 4 without clusters: a cooperative launch of self-timed CTAs that
//     hand their last row downstream through a ring in global memory.
//   8 (default where it fits) as 4 with clusters small enough that all eight
//     octants are resident at once, two pencils per thread where needed,
//     inputs prefetched by cp.async and ghost cells for the inflow.
// G in paths 1, 4, 6, 7 and 8 is summed within each octant in ordinate order and then over
// octants in octant order (the reference sums all ordinates in one sequence;
// the two orders differ only by rounding).
#include <vector>
#include <cstring>
#include <utility>
#include <cooperative_groups.h>
#include "common.cuh"
#include "kernels.h"

#define PI_D 3.141592653589793
#define SIGMA_SB_D 5.67e-8

struct DomCtx {
  GridDev g;
  int M;
  double *ox, *oy, *oz, *w;  // device ordinates and weights
  std::vector<double> hox, hoy, hoz, hw;
  double* I;                  // M * N (paths 2/3 only)
  double* wrap;               // M * Nz * Nx y-periodic inflow rows (path 1)
  double2* kb;                // (kappa, kappa*B) per cell (path 1)
  double* Goct;               // 8 * N octant partial G (path 1)
  double* Qoct;               // 8 * (Ny*Nx) octant partial ground flux (path 1)
  int mode;                   // resolved path: 0 not yet, 1 clusters, 2 block/ordinate, 3 planes
  int mode_req, force_C;      // requested path (0 auto) and cluster size (0 auto)
  int groups;                 // ordinate groups per octant (clusters per octant), paths 4/6
  int fp32;                   // single-precision sweep (path 4 only)
  float2* kb32;
  float *Goct32, *Qoct32, *wrap32;
  int Mo, cl_C, cl_rows, cl_threads, cl_lg_ring, cl_ppt, cl_active;
  int force_groups;            // path 8: ordinate groups per octant (0 automatic)
  int begun;                  // dom_begin done, dom_end due
  double pend_I_amb;          // ambient intensity of the begun solve
  void* st_ring;              // path 7 hand-off ring, then the read counters
  size_t st_ring_bytes;       // ring and counters (filled with 0xff before each sweep)
  size_t st_cnt_offset;
  size_t cl_smem;
  int down_slot[8];
  double *G, *Gp;             // current / previous G
  double *ks, *kg, *ksafe, *B;
  double *Ig_out, *Isoil, *qin;  // (Ny, Nx)
  unsigned long long* keys;      // reduction slots
  unsigned long long* h_keys;
  int* dstate;                   // path 8's device-side test: done, iterations, error
  int* h_dstate;
  double eps_w, tol, relax, kgmax;
  int max_iter;
  int last_iters;
  // optional per-sweep timing (CUDA events on the launching stream)
  int timing;
  cudaEvent_t ev0[32], ev1[32];
  double sweep_ms;
  long long sweep_count;
};

// L2 eviction-priority hints: (kappa, kappa*B) is re-read by every ordinate of
// a sweep and should stay in L2, while intensities and partial sums are
// written once per sweep and should leave it first.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double2 ld_hint(const double2* p, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(v.x), "=d"(v.y)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_stream(double* p, double v) {
  asm volatile("st.global.cs.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

__device__ __forceinline__ double clip01(double x) {
  if (x < 0.0) x = 0.0;
  if (x > 1.0) x = 1.0;
  return x;
}

__global__ void k_dom_setup(GridDev g, const double* __restrict__ Ts, const double* __restrict__ Tg,
                            const double* __restrict__ as, const double* __restrict__ om,
                            const double* __restrict__ YH, const double* __restrict__ rho,
                            const double* __restrict__ Mloc, double sigma, double Tamb4,
                            double kgmax, double* ks, double* kg, double* ksafe, double* B,
                            double2* kb, float2* kb32) {
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
  const double Bc = SIGMA_SB_D * T4 / PI_D;
  ks[c] = ksol;
  kg[c] = kgas;
  ksafe[c] = ksf;
  B[c] = Bc;
  if (kb) kb[c] = make_double2(ksf, ksf * Bc);
  if (kb32) kb32[c] = make_float2((float)ksf, (float)(ksf * Bc));
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
  const double ix = fabs(xi) / g.dx;
  const double iy = fabs(eta) / g.dy;
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
  const double ix = fabs(xi) / g.dx;
  const double iy = fabs(eta) / g.dy;
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

// Path 5: one CTA per ordinate (as path 2) with every thread owning a fixed
// set of PPT pencils.  Per hyperplane each thread first loads its cells'
// kappa and kappa*B (all pencils at once, one load latency), then the upwind
// values from the shared previous-plane buffer, and writes the new values to
// the shared current-plane buffer and to the intensity field; the y-periodic
// inflow of the first row and the ground intensity of the bottom row are
// staged in shared memory one hyperplane ahead by the first threads.  One
// __syncthreads per hyperplane, no cross-CTA traffic; G is then summed over
// all ordinates in ordinate order, as the reference does.
struct OrdArgs {
  const double *ox, *oy, *oz;
  double* I;                // M x N intensities (natural layout)
  const double2* kb;        // (kappa, kappa*B)
  const double* Ig;         // ground intensity (ny, nx)
  double I_amb;
  int periodic;
};

__host__ __device__ inline size_t ord_smem_bytes(int ny, int nz) {
  return sizeof(double) * ((size_t)2 * ny * nz + (size_t)nz + 2 * (size_t)nz + 2 * (size_t)ny);
}

template <int PPT, int TPB>
__global__ void __launch_bounds__(TPB, 1) k_dom_ord(GridDev g, OrdArgs a) {
  extern __shared__ double sh[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int npen = ny * nz;
  double* bufA = sh;
  double* bufB = sh + npen;
  double* izt = bufB + npen;            // |mu| / dz_k
  double* wrapbuf = izt + nz;           // 2 x nz: y inflow of the row (kp, jp = 0)
  double* igbuf = wrapbuf + 2 * nz;     // 2 x ny: ground intensity under (kp = 0, jp)
  const int n = blockIdx.x;
  const double xi = a.ox[n], eta = a.oy[n], mu = a.oz[n];
  const bool fx = xi >= 0.0, fy = eta >= 0.0, fz = mu >= 0.0;
  const double ix = fabs(xi) / g.dx;
  const double iy = fabs(eta) / g.dy;
  for (int k = threadIdx.x; k < nz; k += TPB) izt[k] = fabs(mu) / g.dz[k];
  // cell index of sweep coordinates (ip, jp, kp) = base + ip*si + jp*sj + kp*sk (32-bit; the
  // host checks that Nx*Ny*Nz fits)
  const int si = fx ? 1 : -1;
  const int sj = fy ? nx : -nx;
  const int sk = fz ? nx * ny : -(nx * ny);
  const int base = (fz ? 0 : (nz - 1) * nx * ny) + (fy ? 0 : (ny - 1) * nx) + (fx ? 0 : nx - 1);
  const int wrap_off = fy ? (ny - 1) * nx : -(ny - 1) * nx;   // jp = 0 -> far end of the row
  double* I = a.I + (int64_t)n * ncells_dev(g);
  const int nplanes = nx + ny + nz - 2;
  const int kp0 = threadIdx.x / ny, jp0 = threadIdx.x - kp0 * ny;
  const int dkp = TPB / ny, djp = TPB - dkp * ny;
  constexpr int CH = PPT < 4 ? PPT : 4;   // pencils whose loads are in flight together
  const uint64_t keep = l2_policy_evict_last();
  for (int d = -1; d < nplanes; ++d) {
    // stage the inflow values of plane d+1 (plane 0 before the loop proper)
    {
      const int dn = d + 1;
      const int t = threadIdx.x;
      if (dn < nplanes) {
        if (t < nz && a.periodic) {
          const int ip = dn - t;
          if (ip >= 0 && ip < nx) wrapbuf[(dn & 1) * nz + t] = I[base + ip * si + t * sk + wrap_off];
        }
        if (fz && t >= nz && t < nz + ny) {
          const int jp = t - nz;
          const int ip = dn - jp;
          if (ip >= 0 && ip < nx) {
            const int i = fx ? ip : nx - 1 - ip;
            const int j = fy ? jp : ny - 1 - jp;
            igbuf[(dn & 1) * ny + jp] = a.Ig[j * nx + i];
          }
        }
      }
    }
    if (d >= 0) {
      double* cur = (d & 1) ? bufB : bufA;
      const double* prev = (d & 1) ? bufA : bufB;
      const double* wrp = wrapbuf + (d & 1) * nz;
      const double* igp = igbuf + (d & 1) * ny;
      int kp = kp0, jp = jp0;
#pragma unroll
      for (int r0 = 0; r0 < PPT; r0 += CH) {
        double2 kab[CH];
        int cc[CH];
        {
          int kq = kp, jq = jp;
#pragma unroll
          for (int r = 0; r < CH; ++r) {
            const int ip = d - jq - kq;
            cc[r] = (kq < nz && ip >= 0 && ip < nx) ? base + ip * si + jq * sj + kq * sk : -1;
            if (cc[r] >= 0) kab[r] = ld_hint(a.kb + cc[r], keep);
            kq += dkp; jq += djp;
            if (jq >= ny) { jq -= ny; ++kq; }
          }
        }
#pragma unroll
        for (int r = 0; r < CH; ++r) {
          if (cc[r] >= 0) {
            const int ip = d - jp - kp;
            const int q = threadIdx.x + (r0 + r) * TPB;
            const double Ix = ip > 0 ? prev[q] : a.I_amb;
            const double Iy = jp > 0 ? prev[q - 1] : (a.periodic ? wrp[kp] : a.I_amb);
            double Iz;
            if (kp > 0) Iz = prev[q - ny];
            else Iz = fz ? (mu > 0.0 ? igp[jp] : 0.0) : a.I_amb;
            const double iz = izt[fz ? kp : nz - 1 - kp];
            const double num = kab[r].y + ix * Ix + iy * Iy + iz * Iz;
            const double den = kab[r].x + ix + iy + iz;
            const double v = num / den;
            cur[q] = v;
            st_stream(I + cc[r], v);
          }
          kp += dkp; jp += djp;
          if (jp >= ny) { jp -= ny; ++kp; }
        }
      }
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

// ---- path 1: octant clusters -------------------------------------------------
namespace cg = cooperative_groups;

struct OctArgs {
  const double2* kb;
  const double *ox, *oy, *oz, *w;
  const double* Ig;
  double *Goct, *Qoct, *wrap;
  double I_amb;
  int Mo, C, rows, periodic;
  unsigned down_slots;  // 4 bits per octant: ground-flux slot, 15 = upward octant
  int* err;             // set when a bounded wait gives up (pipelined sweep)
  int groups;           // clusters per octant, each with MO of its ordinates (barrier path)
};

// Dynamic shared memory: two hyperplane buffers of Mo x (rows*Ny) doubles,
// then |mu|/dz_k (Mo x Nz), |xi|/dx, |eta|/dy, w, w*|mu| (Mo each).
__host__ __device__ inline size_t oct_smem_bytes(int Mo, int rows, int ny, int nz) {
  return sizeof(double) * ((size_t)2 * Mo * rows * ny + (size_t)Mo * nz + 4 * (size_t)Mo);
}
// pipelined sweep: mbarriers (2 x OCT_RING) + inbox ring (OCT_RING x Mo x Ny) in front
#define OCT_RING 4
// and a ring of OCT_AHEAD hyperplanes of prefetched inputs per thread:
// (kappa, kappa*B) 16 B, the y-inflow wrap values Mo x 8 B, the ground intensity 8 B
#define OCT_AHEAD 4
__host__ __device__ inline size_t oct_pipe_smem_bytes(int Mo, int rows, int ny, int nz) {
  const size_t nthr = (size_t)rows * ny;
  return 16 * (size_t)OCT_RING + sizeof(double) * (size_t)OCT_RING * Mo * ny +
         (size_t)OCT_AHEAD * nthr * 16 + (size_t)OCT_AHEAD * rows * Mo * 8 +
         (size_t)OCT_AHEAD * ny * 8 + oct_smem_bytes(Mo, rows, ny, nz);
}

__device__ __forceinline__ void cluster_arrive_release() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

#define OCT_MAX_THREADS 512
// One thread per pencil (rows*Ny <= OCT_MAX_THREADS).  Per hyperplane:
// wait for the previous plane of the whole cluster, compute all MO
// ordinates of the thread's cell from shared memory (the neighbour CTA's
// last row through DSMEM), arrive, then store the octant partials and
// prefetch the next plane's kappa / inflow values while the others finish.
template <int MO, int MINB = 1>
__global__ void __launch_bounds__(OCT_MAX_THREADS, MINB) k_dom_octant(GridDev g, OctArgs a) {
  extern __shared__ double sh[];
  cg::cluster_group cl = cg::this_cluster();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int rank = (int)cl.block_rank();
  const int part = blockIdx.x / a.C;      // (octant, ordinate group)
  const int oct = part / a.groups;
  const int grp = part - oct * a.groups;
  const int n0 = (oct * a.groups + grp) * MO;
  const int S = a.rows * ny;
  double* buf0 = sh;
  double* buf1 = sh + (size_t)MO * S;
  double* izt = buf1 + (size_t)MO * S;
  double* cix = izt + (size_t)MO * nz;
  double* ciy = cix + MO;
  double* cw = ciy + MO;
  double* cwm = cw + MO;
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int m = t / nz, k = t - m * nz;
    izt[t] = fabs(a.oz[n0 + m]) / g.dz[k];
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    cix[m] = fabs(a.ox[n0 + m]) / g.dx;
    ciy[m] = fabs(a.oy[n0 + m]) / g.dy;
    cw[m] = a.w[n0 + m];
    cwm[m] = a.w[n0 + m] * fabs(a.oz[n0 + m]);
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * a.rows;
  const int nrows = min(a.rows, nz - r0);
  const int npen = nrows > 0 ? nrows * ny : 0;
  const int q = threadIdx.x;
  const bool has = q < npen;
  const int kl = has ? q / ny : 0;
  const int jp = has ? q - kl * ny : 0;
  const int kp = r0 + kl;
  const int j = fy ? jp : ny - 1 - jp;
  const int k = fz ? kp : nz - 1 - kp;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits * a.groups + grp;
  double* Go = a.Goct + (int64_t)part * N;
  const int64_t wstride = (int64_t)nz * nx;
  double* wrap0 = a.wrap + (int64_t)n0 * wstride;
  const bool ground_out = has && !fz && k == 0 && slot >= 0;
  const bool z_in_ground = has && fz && kp == 0;
  const bool z_remote = has && kl == 0 && kp > 0;
  const bool y_wrap = has && jp == 0 && a.periodic;
  const bool y_wrap_out = has && jp == ny - 1 && a.periodic;
  const double* nbase = nullptr;
  const int nplanes = nx + ny + nz - 2;
  const uint64_t keep = l2_policy_evict_last();
  // prefetched values for the coming plane
  double2 kab = make_double2(0.0, 0.0);
  double win[MO];
  double Igc = 0.0;
  auto prefetch = [&](int d) {
    const int ip = d - jp - kp;
    if (!has || ip < 0 || ip >= nx) return;
    const int i = fx ? ip : nx - 1 - ip;
    kab = ld_hint(a.kb + ((int64_t)k * ny + j) * nx + i, keep);
    if (y_wrap) {
#pragma unroll
      for (int m = 0; m < MO; ++m) win[m] = wrap0[m * wstride + (int64_t)k * nx + i];
    }
    if (z_in_ground) Igc = a.Ig[(int64_t)j * nx + i];
  };
#pragma unroll
  for (int m = 0; m < MO; ++m) win[m] = a.I_amb;
  __syncthreads();
  prefetch(0);
  for (int d = 0; d < nplanes; ++d) {
    double* cur = (d & 1) ? buf1 : buf0;
    const double* prev = (d & 1) ? buf0 : buf1;
    if (d > 0) cluster_wait_acquire();
    const int ip = d - jp - kp;
    const bool act = has && ip >= 0 && ip < nx;
    double v[MO];
    double gs = 0.0, qs = 0.0;
    if (act) {
      if (z_remote) nbase = cl.map_shared_rank(const_cast<double*>(prev), rank - 1) +
                            (size_t)(a.rows - 1) * ny + jp;
      double zr[MO];
      if (z_remote) {
#pragma unroll
        for (int m = 0; m < MO; ++m) zr[m] = nbase[(size_t)m * S];
      }
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        const double* pm = prev + (size_t)m * S;
        const double Ix = ip > 0 ? pm[q] : a.I_amb;
        const double Iy = jp > 0 ? pm[q - 1] : (a.periodic ? win[m] : a.I_amb);
        double Iz;
        if (kl > 0) Iz = pm[q - ny];
        else if (kp > 0) Iz = zr[m];
        else Iz = fz ? Igc : a.I_amb;
        const double ix = cix[m], iy = ciy[m], iz = izt[m * nz + k];
        const double num = kab.y + ix * Ix + iy * Iy + iz * Iz;
        const double den = kab.x + ix + iy + iz;
        v[m] = num / den;
        cur[(size_t)m * S + q] = v[m];
        gs = gs + cw[m] * v[m];
        if (ground_out) qs = qs + cwm[m] * v[m];
      }
    }
    cluster_arrive_release();
    if (act) {
      const int i = fx ? ip : nx - 1 - ip;
      st_stream(Go + ((int64_t)k * ny + j) * nx + i, gs);
      if (y_wrap_out) {
#pragma unroll
        for (int m = 0; m < MO; ++m) wrap0[m * wstride + (int64_t)k * nx + i] = v[m];
      }
      if (ground_out) a.Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qs;
    }
    if (d + 1 < nplanes) prefetch(d + 1);
  }
  cluster_wait_acquire();
}

// The division of the sweep: correctly rounded in FP64 (the reference's
// arithmetic); in the single-precision form the reciprocal-based quotient of
// __fdividef (about 2 ulp), which keeps each ordinate's dependent chain short.
__device__ __forceinline__ double sweep_div(double a, double b) { return a / b; }
__device__ __forceinline__ float sweep_div(float a, float b) { return __fdividef(a, b); }

// ---- single-precision form of path 4 (the mixed-precision solver) -----------
// Same sweep, with kappa, kappa*B, the hyperplane buffers, the inflow rows and
// the octant partials in FP32; the octant partials are summed into G in FP64.
struct OctArgs32 {
  const float2* kb;
  const double *ox, *oy, *oz, *w;
  const double* Ig;
  float *Goct, *Qoct, *wrap;
  float I_amb;
  int C, rows, periodic;
  unsigned down_slots;
};

__device__ __forceinline__ float2 ld_hint_f2(const float2* p, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
               : "=f"(v.x), "=f"(v.y)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_stream_f(float* p, float v) {
  asm volatile("st.global.cs.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

template <int MO>
__global__ void __launch_bounds__(OCT_MAX_THREADS, 1) k_dom_octant_f32(GridDev g, OctArgs32 a) {
  extern __shared__ float shf[];
  cg::cluster_group cl = cg::this_cluster();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int rank = (int)cl.block_rank();
  const int oct = blockIdx.x / a.C;
  const int n0 = oct * MO;
  const int S = a.rows * ny;
  float* buf0 = shf;
  float* buf1 = shf + (size_t)MO * S;
  float* izt = buf1 + (size_t)MO * S;
  float* cix = izt + (size_t)MO * nz;
  float* ciy = cix + MO;
  float* cw = ciy + MO;
  float* cwm = cw + MO;
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int m = t / nz, k = t - m * nz;
    izt[t] = (float)(fabs(a.oz[n0 + m]) / g.dz[k]);
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    cix[m] = (float)(fabs(a.ox[n0 + m]) / g.dx);
    ciy[m] = (float)(fabs(a.oy[n0 + m]) / g.dy);
    cw[m] = (float)a.w[n0 + m];
    cwm[m] = (float)(a.w[n0 + m] * fabs(a.oz[n0 + m]));
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * a.rows;
  const int nrows = min(a.rows, nz - r0);
  const int npen = nrows > 0 ? nrows * ny : 0;
  const int q = threadIdx.x;
  const bool has = q < npen;
  const int kl = has ? q / ny : 0;
  const int jp = has ? q - kl * ny : 0;
  const int kp = r0 + kl;
  const int j = fy ? jp : ny - 1 - jp;
  const int k = fz ? kp : nz - 1 - kp;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits;
  float* Go = a.Goct + (int64_t)oct * N;
  const int64_t wstride = (int64_t)nz * nx;
  float* wrap0 = a.wrap + (int64_t)n0 * wstride;
  const bool ground_out = has && !fz && k == 0 && slot >= 0;
  const bool z_in_ground = has && fz && kp == 0;
  const bool z_remote = has && kl == 0 && kp > 0;
  const bool y_wrap = has && jp == 0 && a.periodic;
  const bool y_wrap_out = has && jp == ny - 1 && a.periodic;
  const float* nbase = nullptr;
  const int nplanes = nx + ny + nz - 2;
  const uint64_t keep = l2_policy_evict_last();
  float2 kab = make_float2(0.f, 0.f);
  float win[MO];
  float Igc = 0.f;
  auto prefetch = [&](int d) {
    const int ip = d - jp - kp;
    if (!has || ip < 0 || ip >= nx) return;
    const int i = fx ? ip : nx - 1 - ip;
    kab = ld_hint_f2(a.kb + ((int64_t)k * ny + j) * nx + i, keep);
    if (y_wrap) {
#pragma unroll
      for (int m = 0; m < MO; ++m) win[m] = wrap0[m * wstride + (int64_t)k * nx + i];
    }
    if (z_in_ground) Igc = (float)a.Ig[(int64_t)j * nx + i];
  };
#pragma unroll
  for (int m = 0; m < MO; ++m) win[m] = a.I_amb;
  __syncthreads();
  prefetch(0);
  for (int d = 0; d < nplanes; ++d) {
    float* cur = (d & 1) ? buf1 : buf0;
    const float* prev = (d & 1) ? buf0 : buf1;
    if (d > 0) cluster_wait_acquire();
    const int ip = d - jp - kp;
    const bool act = has && ip >= 0 && ip < nx;
    float v[MO];
    float gs = 0.f, qs = 0.f;
    if (act) {
      if (z_remote) nbase = cl.map_shared_rank(const_cast<float*>(prev), rank - 1) +
                            (size_t)(a.rows - 1) * ny + jp;
      float zr[MO];
      if (z_remote) {
#pragma unroll
        for (int m = 0; m < MO; ++m) zr[m] = nbase[(size_t)m * S];
      }
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        const float* pm = prev + (size_t)m * S;
        const float Ix = ip > 0 ? pm[q] : a.I_amb;
        const float Iy = jp > 0 ? pm[q - 1] : (a.periodic ? win[m] : a.I_amb);
        float Iz;
        if (kl > 0) Iz = pm[q - ny];
        else if (kp > 0) Iz = zr[m];
        else Iz = fz ? Igc : a.I_amb;
        const float ix = cix[m], iy = ciy[m], iz = izt[m * nz + k];
        const float num = kab.y + ix * Ix + iy * Iy + iz * Iz;
        const float den = kab.x + ix + iy + iz;
        v[m] = sweep_div(num, den);
        cur[(size_t)m * S + q] = v[m];
        gs = gs + cw[m] * v[m];
        if (ground_out) qs = qs + cwm[m] * v[m];
      }
    }
    cluster_arrive_release();
    if (act) {
      const int i = fx ? ip : nx - 1 - ip;
      st_stream_f(Go + ((int64_t)k * ny + j) * nx + i, gs);
      if (y_wrap_out) {
#pragma unroll
        for (int m = 0; m < MO; ++m) wrap0[m * wstride + (int64_t)k * nx + i] = v[m];
      }
      if (ground_out) a.Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qs;
    }
    if (d + 1 < nplanes) prefetch(d + 1);
  }
  cluster_wait_acquire();
}

static const void* octant_f32_ptr(int Mo) {
  switch (Mo) {
    case 3: return (const void*)k_dom_octant_f32<3>;
    case 6: return (const void*)k_dom_octant_f32<6>;
    case 10: return (const void*)k_dom_octant_f32<10>;
    default: return nullptr;
  }
}

// G (FP64) from FP32 octant partials; max G and max |G - G_prev|
__global__ void k_dom_G_oct32(int64_t N, int nparts, const float* __restrict__ Goct, double* G,
                              const double* __restrict__ Gp, unsigned long long* keys,
                              const int* done = nullptr) {
  if (done && *done) return;
  unsigned long long bg = 0, bd = 0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N;
       c += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int o = 0; o < nparts; ++o) s += (double)Goct[(int64_t)o * N + c];
    G[c] = s;
    double d = fabs(s - Gp[c]);
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

__global__ void k_dom_ground_oct32(int n2, int nslots, const float* __restrict__ Qoct,
                                   const double* __restrict__ Isoil, double refl, double relax,
                                   double* Ig, double* qin, const int* done = nullptr) {
  if (done && *done) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  double s = 0.0;
  for (int o = 0; o < nslots; ++o) s += (double)Qoct[(int64_t)o * n2 + q];
  qin[q] = s;
  double Inew = Isoil[q] + refl * s;
  Ig[q] = relax * Inew + (1.0 - relax) * Ig[q];
}

__global__ void k_f32_to_f64(int64_t n, const float* __restrict__ a, double* b) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) b[t] = (double)a[t];
}
__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ a, float* b) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) b[t] = (float)a[t];
}

// ---- pipelined variant: point-to-point hand-off between neighbouring CTAs ----
// CTA r needs, on hyperplane d, the last row of CTA r-1 from hyperplane d-1.
// Instead of a cluster-wide barrier per hyperplane, CTA r-1's last-row
// threads store those values straight into an inbox ring in CTA r's shared
// memory (distributed shared memory) and arrive on that slot's "full"
// mbarrier; CTA r's first-row threads wait on it, read, and arrive on the
// producer's "empty" mbarrier for the slot.  Each CTA then only waits for
// its upstream neighbour and the CTAs run as a skewed pipeline; inside a
// CTA one __syncthreads per hyperplane orders the shared buffers.  Every
// wait is bounded: on expiry the kernel records the failure in *err and
// runs to completion without waiting further.
#define OCT_WAIT_LIMIT 2000000
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t cluster_map_u32(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t remote_a) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote_a)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false (and *err set) if it gave up or an earlier wait had
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t a, uint32_t parity, int* err) {
  if (mbar_try_wait(a, parity)) return true;
  for (int it = 1; it < OCT_WAIT_LIMIT; ++it) {
    if (mbar_try_wait(a, parity)) return true;
    if ((it & 1023) == 0 && *(volatile int*)err) return false;  // another wait gave up
  }
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int MO>
__global__ void __launch_bounds__(OCT_MAX_THREADS, 1) k_dom_octant_pipe(GridDev g, OctArgs a) {
  extern __shared__ __align__(16) unsigned char shraw[];
  cg::cluster_group cl = cg::this_cluster();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int rank = (int)cl.block_rank();
  const int C = a.C;
  const int oct = blockIdx.x / C;
  const int n0 = oct * MO;
  const int rows = a.rows;
  const int S = rows * ny;
  unsigned long long* mb_full = (unsigned long long*)shraw;   // this CTA's inbox slots
  unsigned long long* mb_empty = mb_full + OCT_RING;          // this CTA's outbox slots
  double* inbox = (double*)(shraw + 16 * OCT_RING);           // OCT_RING x MO x ny
  double2* kab_ring = (double2*)(inbox + (size_t)OCT_RING * MO * ny);  // OCT_AHEAD x S
  double* wrap_ring = (double*)(kab_ring + (size_t)OCT_AHEAD * S);     // OCT_AHEAD x MO x rows
  double* ig_ring = wrap_ring + (size_t)OCT_AHEAD * MO * rows;         // OCT_AHEAD x ny
  double* buf0 = ig_ring + (size_t)OCT_AHEAD * ny;
  double* buf1 = buf0 + (size_t)MO * S;
  double* izt = buf1 + (size_t)MO * S;
  double* cix = izt + (size_t)MO * nz;
  double* ciy = cix + MO;
  double* cw = ciy + MO;
  double* cwm = cw + MO;
  if (threadIdx.x == 0) {
    for (int s = 0; s < OCT_RING; ++s) {
      mbar_init(smem_u32(mb_full + s), (uint32_t)ny);
      mbar_init(smem_u32(mb_empty + s), (uint32_t)ny);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int m = t / nz, k = t - m * nz;
    izt[t] = fabs(a.oz[n0 + m]) / g.dz[k];
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    cix[m] = fabs(a.ox[n0 + m]) / g.dx;
    ciy[m] = fabs(a.oy[n0 + m]) / g.dy;
    cw[m] = a.w[n0 + m];
    cwm[m] = a.w[n0 + m] * fabs(a.oz[n0 + m]);
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * rows;
  const int nrows = min(rows, nz - r0);
  const int npen = nrows > 0 ? nrows * ny : 0;
  const int q = threadIdx.x;
  const bool has = q < npen;
  const int kl = has ? q / ny : 0;
  const int jp = has ? q - kl * ny : 0;
  const int kp = r0 + kl;
  const int j = fy ? jp : ny - 1 - jp;
  const int k = fz ? kp : nz - 1 - kp;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits;
  double* Go = a.Goct + (int64_t)oct * N;
  const int64_t wstride = (int64_t)nz * nx;
  double* wrap0 = a.wrap + (int64_t)n0 * wstride;
  const bool ground_out = has && !fz && k == 0 && slot >= 0;
  const bool z_in_ground = has && fz && kp == 0;
  const bool consumer = has && kl == 0 && rank > 0;
  const bool producer = has && kl == rows - 1 && rank < C - 1;
  const bool y_wrap = has && jp == 0 && a.periodic;
  const bool y_wrap_out = has && jp == ny - 1 && a.periodic;
  double* down_inbox = producer ? cl.map_shared_rank(inbox, rank + 1) : nullptr;
  const uint32_t full_u32 = smem_u32(mb_full), empty_u32 = smem_u32(mb_empty);
  const uint32_t down_full = producer ? cluster_map_u32(full_u32, rank + 1) : 0u;
  const uint32_t up_empty = consumer ? cluster_map_u32(empty_u32, rank - 1) : 0u;
  const int nplanes = nx + ny + nz - 2;
  const int64_t row_base = ((int64_t)k * ny + j) * nx;
  // asynchronous copies of plane d's inputs into ring slot d % OCT_AHEAD (one group per plane)
  auto prefetch = [&](int d) {
    const int ip = d - jp - kp;
    if (has && ip >= 0 && ip < nx) {
      const int i = fx ? ip : nx - 1 - ip;
      const int sl = d % OCT_AHEAD;
      cp_async16(&kab_ring[(size_t)sl * S + q], &a.kb[row_base + i]);
      if (y_wrap) {
#pragma unroll
        for (int m = 0; m < MO; ++m)
          cp_async8(&wrap_ring[((size_t)sl * MO + m) * rows + kl],
                    &wrap0[m * wstride + (int64_t)k * nx + i]);
      }
      if (z_in_ground) cp_async8(&ig_ring[(size_t)sl * ny + jp], &a.Ig[(int64_t)j * nx + i]);
    }
    cp_async_commit();
  };
  for (int d = 0; d < OCT_AHEAD - 1; ++d) prefetch(d);
  // every CTA's barriers are initialised before anyone arrives remotely
  cluster_arrive_release();
  cluster_wait_acquire();
  for (int d = 0; d < nplanes; ++d) {
    prefetch(d + OCT_AHEAD - 1);   // an empty group past the last plane
    double* cur = (d & 1) ? buf1 : buf0;
    const double* prev = (d & 1) ? buf0 : buf1;
    const int ip = d - jp - kp;
    const bool act = has && ip >= 0 && ip < nx;
    double zr[MO];
    if (consumer && d > 0) {
      const int sl = (d - 1) % OCT_RING;
      mbar_wait_bounded(full_u32 + 8u * sl, (uint32_t)(((d - 1) / OCT_RING) & 1), a.err);
      if (act) {
#pragma unroll
        for (int m = 0; m < MO; ++m) zr[m] = inbox[((size_t)sl * MO + m) * ny + jp];
      }
      mbar_arrive_cluster(up_empty + 8u * sl);
    }
    cp_async_wait<OCT_AHEAD - 1>();   // this plane's group has landed
    double v[MO];
    double gs = 0.0, qs = 0.0;
    if (act) {
      const int sl = d % OCT_AHEAD;
      const double2 kab = kab_ring[(size_t)sl * S + q];
      double den[MO];
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        const double* pm = prev + (size_t)m * S;
        const double Ix = ip > 0 ? pm[q] : a.I_amb;
        double Iy;
        if (jp > 0) Iy = pm[q - 1];
        else Iy = a.periodic ? wrap_ring[((size_t)sl * MO + m) * rows + kl] : a.I_amb;
        double Iz;
        if (kl > 0) Iz = pm[q - ny];
        else if (kp > 0) Iz = zr[m];
        else Iz = fz ? ig_ring[(size_t)sl * ny + jp] : a.I_amb;
        const double ix = cix[m], iy = ciy[m], iz = izt[m * nz + k];
        v[m] = kab.y + ix * Ix + iy * Iy + iz * Iz;
        den[m] = kab.x + ix + iy + iz;
      }
#pragma unroll
      for (int m = 0; m < MO; ++m) v[m] = v[m] / den[m];
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        cur[(size_t)m * S + q] = v[m];
        gs = gs + cw[m] * v[m];
        if (ground_out) qs = qs + cwm[m] * v[m];
      }
    }
    if (producer) {
      const int sl = d % OCT_RING;
      if (d >= OCT_RING)
        mbar_wait_bounded(empty_u32 + 8u * sl, (uint32_t)(((d / OCT_RING) - 1) & 1), a.err);
      if (act) {
#pragma unroll
        for (int m = 0; m < MO; ++m) down_inbox[((size_t)sl * MO + m) * ny + jp] = v[m];
      }
      mbar_arrive_cluster(down_full + 8u * sl);
    }
    if (act) {
      const int i = fx ? ip : nx - 1 - ip;
      Go[row_base + i] = gs;
      if (y_wrap_out) {
#pragma unroll
        for (int m = 0; m < MO; ++m) wrap0[m * wstride + (int64_t)k * nx + i] = v[m];
      }
      if (ground_out) a.Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qs;
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  // nobody leaves while a neighbour may still touch its shared memory
  cluster_arrive_release();
  cluster_wait_acquire();
}

// ---- path 7: self-timed octant pipeline (global-memory hand-off) -------------
// The row split of path 4 (CTAs of an octant split the k' rows, one thread per
// pencil, all ordinates of the octant per thread), without clusters and
// without any barrier between CTAs.  The only value a CTA needs from another
// is the upstream CTA's last row of the previous hyperplane.  The upstream
// CTA's last-row threads store that row into a ring of R slots in global
// memory (L2), and the downstream CTA's first-row threads load it from there.
// No fence is issued on the hand-off: every word carries its own state.  The
// intensities are never negative, so the sign bit of each stored word is free
// and holds the lap parity ((p - a0) / R) mod 2 of hyperplane p, a0 being the
// first hyperplane of that pencil; the ring is filled with sign-bit-set words
// before every sweep, so the first lap (parity 0) can never be mistaken for
// stale contents, and a word two laps old cannot be present when a lap is
// awaited because the reader has already read the lap in between.  The
// writer may overwrite a slot once the reader's CTA has published (one
// relaxed store per hyperplane) that it has read it; those reads have
// completed by then.  Each CTA therefore runs at its own pace with one
// __syncthreads per hyperplane, the latency between SMs is paid once per CTA
// in the pipeline fill, and no cluster has to fit in one GPC, so all eight
// octants run at once.  The arithmetic of every cell is that of path 4, so the
// results are identical.  Every wait is bounded as in path 1.
template <typename T> struct Vec2Of;
template <> struct Vec2Of<double> { using type = double2; };
template <> struct Vec2Of<float> { using type = float2; };
template <typename T> struct WordOf;
template <> struct WordOf<double> { using type = unsigned long long; };
template <> struct WordOf<float> { using type = unsigned; };

template <typename T>
struct StArgs {
  const typename Vec2Of<T>::type* kb;
  const double *ox, *oy, *oz, *w;
  const double* Ig;
  T *Goct, *Qoct, *wrap;
  typename WordOf<T>::type* ring;  // 8 x (C-1) x R x Mo x Ny words
  int* consumed;                   // 8 x (C-1): last hyperplane read by each downstream CTA
  T I_amb;
  int C, rows, periodic, lg_ring;
  unsigned down_slots;
  int* err;
};
#define ST_RING_LG 3  // R = 8 slots

__host__ __device__ inline size_t st_up16(size_t x) { return (x + 15) & ~(size_t)15; }
// Shared-memory layout of path 7 (byte offsets, each 16-byte aligned): the
// prefetch rings (OCT_AHEAD hyperplanes of kappa/kappa*B and ground
// intensity), the y-inflow and y-outflow rows staged in chunks of ST_CHUNK
// hyperplanes (two chunks each), the z-inflow row from the upstream CTA, the
// two hyperplane buffers and the per-ordinate constants.
#define ST_CHUNK 32
struct StLayout {
  size_t kab, ig, win, wout, zin, buf0, buf1, izt, cix, total;
};
__host__ __device__ inline StLayout st_layout(int tsize, int Mo, int rows, int ny, int nz) {
  StLayout L;
  const size_t S = (size_t)rows * ny;
  const size_t chunk = (size_t)2 * Mo * rows * ST_CHUNK * tsize;
  size_t o = 0;
  L.kab = o; o = st_up16(o + (size_t)OCT_AHEAD * S * 2 * tsize);
  L.ig = o; o = st_up16(o + (size_t)OCT_AHEAD * ny * sizeof(double));
  L.win = o; o = st_up16(o + chunk);
  L.wout = o; o = st_up16(o + chunk);
  L.zin = o; o = st_up16(o + (size_t)Mo * ny * tsize);
  L.buf0 = o; o = st_up16(o + (size_t)Mo * S * tsize);
  L.buf1 = o; o = st_up16(o + (size_t)Mo * S * tsize);
  L.izt = o; o = st_up16(o + (size_t)Mo * nz * tsize);
  L.cix = o; o = st_up16(o + 4 * (size_t)Mo * tsize);
  L.total = o;
  return L;
}

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(int* p, int v) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long word_of(double v) {
  return (unsigned long long)__double_as_longlong(v);
}
__device__ __forceinline__ unsigned word_of(float v) { return __float_as_uint(v); }
__device__ __forceinline__ double value_of(unsigned long long w) {
  return __longlong_as_double((long long)(w & 0x7fffffffffffffffull));
}
__device__ __forceinline__ float value_of(unsigned w) { return __uint_as_float(w & 0x7fffffffu); }
__device__ __forceinline__ unsigned sign_of(unsigned long long w) { return (unsigned)(w >> 63); }
__device__ __forceinline__ unsigned sign_of(unsigned w) { return w >> 31; }
__device__ __forceinline__ unsigned long long with_sign(unsigned long long w, unsigned s) {
  return (w & 0x7fffffffffffffffull) | ((unsigned long long)s << 63);
}
__device__ __forceinline__ unsigned with_sign(unsigned w, unsigned s) {
  return (w & 0x7fffffffu) | (s << 31);
}
__device__ __forceinline__ void cp_async_kb(void* dst, const double2* src, uint64_t pol) {
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(
                   smem_u32(dst)),
               "l"(src), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async_kb(void* dst, const float2* src, uint64_t pol) {
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(
                   smem_u32(dst)),
               "l"(src), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async_val(void* dst, const double* src) { cp_async8(dst, src); }
__device__ __forceinline__ void cp_async_val(void* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void st_cs(double* p, double v) { st_stream(p, v); }
__device__ __forceinline__ void st_cs(float* p, float v) {
  asm volatile("st.global.cs.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// One thread per pencil.  The y-periodic inflow of a row (read by its first
// pencil) and outflow (written by its last) run along x over the hyperplanes,
// so they move through shared memory in chunks of ST_CHUNK hyperplanes with
// contiguous loads and stores by the whole CTA.  A location's inflow is read
// (from the previous sweep) before its chunk starts and its outflow is
// written after the outflow's chunk ends, ny-1 hyperplanes later, so the
// previous sweep's value is always the one read, as in the reference's
// in-place sweep.
template <typename T, int MO>
__global__ void __launch_bounds__(OCT_MAX_THREADS, 1) k_dom_octant_st(GridDev g, StArgs<T> a) {
  using T2 = typename Vec2Of<T>::type;
  using W = typename WordOf<T>::type;
  extern __shared__ __align__(16) unsigned char shraw[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int C = a.C;
  const int oct = blockIdx.x / C;
  const int rank = blockIdx.x - oct * C;
  const int n0 = oct * MO;
  const int rows = a.rows;
  const int S = rows * ny;
  const int lg = a.lg_ring;
  const int R = 1 << lg;
  const StLayout L = st_layout((int)sizeof(T), MO, rows, ny, nz);
  T2* kab_ring = (T2*)(shraw + L.kab);
  double* ig_ring = (double*)(shraw + L.ig);
  T* win = (T*)(shraw + L.win);    // [2 chunks][MO][rows][ST_CHUNK]
  T* wout = (T*)(shraw + L.wout);  // [2 chunks][MO][rows][ST_CHUNK]
  T* zin = (T*)(shraw + L.zin);
  T* buf0 = (T*)(shraw + L.buf0);
  T* buf1 = (T*)(shraw + L.buf1);
  T* izt = (T*)(shraw + L.izt);
  T* cix = (T*)(shraw + L.cix);
  T* ciy = cix + MO;
  T* cw = ciy + MO;
  T* cwm = cw + MO;
  const int nplanes = nx + ny + nz - 2;
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int m = t / nz, k = t - m * nz;
    izt[t] = (T)(fabs(a.oz[n0 + m]) / g.dz[k]);
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    cix[m] = (T)(fabs(a.ox[n0 + m]) / g.dx);
    ciy[m] = (T)(fabs(a.oy[n0 + m]) / g.dy);
    cw[m] = (T)a.w[n0 + m];
    cwm[m] = (T)(a.w[n0 + m] * fabs(a.oz[n0 + m]));
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * rows;
  const int nrows = min(rows, nz - r0);
  const int npen = nrows > 0 ? nrows * ny : 0;
  const int q = threadIdx.x;
  const bool has = q < npen;
  const int kl = has ? q / ny : 0;
  const int jp = has ? q - kl * ny : 0;
  const int kp = r0 + kl;
  const int j = fy ? jp : ny - 1 - jp;
  const int k = fz ? kp : nz - 1 - kp;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits;
  T* Go = a.Goct + (int64_t)oct * N;
  const int64_t wstride = (int64_t)nz * nx;
  T* wrap0 = a.wrap + (int64_t)n0 * wstride;
  const bool ground_out = has && !fz && k == 0 && slot >= 0;
  const bool z_in_ground = has && fz && kp == 0;
  const bool consumer = has && kl == 0 && rank > 0;
  // only a full CTA (every CTA but the last) has a downstream neighbour
  const bool producer = has && kl == rows - 1 && rank < C - 1;
  const bool periodic = a.periodic != 0;
  const bool y_out = has && jp == ny - 1 && periodic;
  // ring of the boundary below this CTA (read) and above it (written)
  const size_t slot_words = (size_t)MO * ny;
  const W* ring_in = consumer
      ? a.ring + ((size_t)oct * (C - 1) + (rank - 1)) * R * slot_words + jp : nullptr;
  W* ring_out = producer
      ? a.ring + ((size_t)oct * (C - 1) + rank) * R * slot_words + jp : nullptr;
  int* cnt_in = (rank > 0) ? a.consumed + oct * (C - 1) + (rank - 1) : nullptr;
  const int* cnt_out = producer ? a.consumed + oct * (C - 1) + rank : nullptr;
  // first hyperplane of a pencil's hand-off words (the row below the consumer's
  // first row, and the producer's own row): laps are counted from there.  A
  // one-row CTA is consumer and producer at once.
  const int a0_in = jp + kp - 1, a0_out = jp + kp;
  const int64_t row_base = ((int64_t)k * ny + j) * nx;
  const uint64_t keep = l2_policy_evict_last();
  const int chunk_elems = MO * rows * ST_CHUNK;
  // the y-inflow rows of chunk c (hyperplanes c*ST_CHUNK ...), by the whole CTA
  auto load_inflow = [&](int c) {
    T* dst = win + (size_t)(c & 1) * chunk_elems;
    for (int e = threadIdx.x; e < chunk_elems; e += blockDim.x) {
      const int t = e % ST_CHUNK, rm = e / ST_CHUNK;
      const int rl = rm % rows, m = rm / rows;
      const int ip = c * ST_CHUNK + t - (r0 + rl);  // pencil jp = 0 of row rl
      if (rl < nrows && ip >= 0 && ip < nx) {
        const int kk = fz ? r0 + rl : nz - 1 - (r0 + rl);
        const int i = fx ? ip : nx - 1 - ip;
        cp_async_val(&dst[e], &wrap0[m * wstride + (int64_t)kk * nx + i]);
      }
    }
  };
  // the y-outflow rows of chunk c, to global memory by the whole CTA
  auto store_outflow = [&](int c) {
    const T* src = wout + (size_t)(c & 1) * chunk_elems;
    for (int e = threadIdx.x; e < chunk_elems; e += blockDim.x) {
      const int t = e % ST_CHUNK, rm = e / ST_CHUNK;
      const int rl = rm % rows, m = rm / rows;
      const int ip = c * ST_CHUNK + t - (ny - 1) - (r0 + rl);  // pencil jp = ny-1 of row rl
      if (rl < nrows && ip >= 0 && ip < nx) {
        const int kk = fz ? r0 + rl : nz - 1 - (r0 + rl);
        const int i = fx ? ip : nx - 1 - ip;
        wrap0[m * wstride + (int64_t)kk * nx + i] = src[e];
      }
    }
  };
  // the inputs of hyperplane d (one commit group per hyperplane); the group of
  // the last hyperplane before a chunk also carries that chunk's inflow rows
  auto prefetch = [&](int d) {
    const int ip = d - jp - kp;
    if (has && ip >= 0 && ip < nx) {
      const int i = fx ? ip : nx - 1 - ip;
      const int sl = d % OCT_AHEAD;
      cp_async_kb(&kab_ring[(size_t)sl * S + q], &a.kb[row_base + i], keep);
      if (z_in_ground) cp_async8(&ig_ring[(size_t)sl * ny + jp], &a.Ig[(int64_t)j * nx + i]);
    }
    if (periodic && (d + 1) % ST_CHUNK == 0 && d + 1 < nplanes) load_inflow((d + 1) / ST_CHUNK);
    cp_async_commit();
  };
  if (periodic) load_inflow(0);
  for (int d = 0; d < OCT_AHEAD - 1; ++d) prefetch(d);
  cp_async_wait<OCT_AHEAD - 2>();  // group 0, which holds chunk 0 of the inflow rows
  __syncthreads();
  const int Rm = R - 1;
  W raw[MO];  // the z-inflow words of the coming hyperplane (consumer row)
#pragma unroll
  for (int m = 0; m < MO; ++m) raw[m] = 0;
  int known = -1;    // last hyperplane the downstream CTA is known to have read
  int pending = -1;  // a load of that count issued on the previous hyperplane
  for (int d = 0; d < nplanes; ++d) {
    prefetch(d + OCT_AHEAD - 1);  // an empty group past the last plane
    // a finished chunk of outflow rows leaves for global memory
    if (periodic && d > 0 && d % ST_CHUNK == 0) store_outflow(d / ST_CHUNK - 1);
    T* cur = (d & 1) ? buf1 : buf0;
    const T* prev = (d & 1) ? buf0 : buf1;
    const int ip = d - jp - kp;
    const bool act = has && ip >= 0 && ip < nx;
    if (consumer) {
      if (act) {
        // words of hyperplane d-1, loaded one hyperplane ago; re-read any not yet written
        const int p = d - 1;
        const unsigned par = (unsigned)((p - a0_in) >> lg) & 1u;
        const W* src = ring_in + (size_t)(p & Rm) * slot_words;
        unsigned bad = 0;
#pragma unroll
        for (int m = 0; m < MO; ++m) bad |= sign_of(raw[m]) ^ par;
        for (int it = 0; bad; ++it) {
          if (it >= OCT_WAIT_LIMIT) { atomicExch(a.err, 1); break; }
          if ((it & 1023) == 1023 && *(volatile int*)a.err) break;
          // all stale words re-read at once
#pragma unroll
          for (int m = 0; m < MO; ++m)
            if (sign_of(raw[m]) != par) raw[m] = ld_relaxed(src + (size_t)m * ny);
          bad = 0;
#pragma unroll
          for (int m = 0; m < MO; ++m) bad |= sign_of(raw[m]) ^ par;
        }
#pragma unroll
        for (int m = 0; m < MO; ++m) zin[(size_t)m * ny + jp] = value_of(raw[m]);
      }
      // start loading hyperplane d's words, used on the next hyperplane
      const int ipn = d + 1 - jp - kp;
      if (d + 1 < nplanes && ipn >= 0 && ipn < nx) {
        const W* src = ring_in + (size_t)(d & Rm) * slot_words;
#pragma unroll
        for (int m = 0; m < MO; ++m) raw[m] = ld_relaxed(src + (size_t)m * ny);
      }
    }
    cp_async_wait<OCT_AHEAD - 1>();  // this plane's group has landed
    T v[MO];
    T gs = (T)0, qs = (T)0;
    if (act) {
      const int sl = d % OCT_AHEAD;
      const int ch = (d / ST_CHUNK) & 1, tt = d % ST_CHUNK;
      const T2 kab = kab_ring[(size_t)sl * S + q];
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        const T* pm = prev + (size_t)m * S;
        const T Ix = ip > 0 ? pm[q] : a.I_amb;
        T Iy;
        if (jp > 0) Iy = pm[q - 1];
        else Iy = periodic ? win[((size_t)(ch * MO + m) * rows + kl) * ST_CHUNK + tt] : a.I_amb;
        T Iz;
        if (kl > 0) Iz = pm[q - ny];
        else if (kp > 0) Iz = zin[(size_t)m * ny + jp];
        else Iz = fz ? (T)ig_ring[(size_t)sl * ny + jp] : a.I_amb;
        const T ix = cix[m], iy = ciy[m], iz = izt[m * nz + k];
        const T num = kab.y + ix * Ix + iy * Iy + iz * Iz;
        const T den = kab.x + ix + iy + iz;
        v[m] = sweep_div(num, den);
        cur[(size_t)m * S + q] = v[m];
        gs = gs + cw[m] * v[m];
        if (ground_out) qs = qs + cwm[m] * v[m];
      }
      if (y_out) {
#pragma unroll
        for (int m = 0; m < MO; ++m) wout[((size_t)(ch * MO + m) * rows + kl) * ST_CHUNK + tt] = v[m];
      }
    }
    if (producer) {
      if (pending > known) known = pending;
      if (act) {
        // the slot held hyperplane d-R, which the downstream CTA must have read
        if (d - R > known) {
          int it = 0;
          do {
            known = ld_relaxed(cnt_out);
          } while (d - R > known && ++it < OCT_WAIT_LIMIT &&
                   !((it & 1023) == 0 && *(volatile int*)a.err));
          if (d - R > known && it >= OCT_WAIT_LIMIT) atomicExch(a.err, 1);
        }
        const unsigned par = (unsigned)((d - a0_out) >> lg) & 1u;
        W* dst = ring_out + (size_t)(d & Rm) * slot_words;
#pragma unroll
        for (int m = 0; m < MO; ++m)
          st_relaxed(dst + (size_t)m * ny, with_sign(word_of(v[m]), par));
      }
      pending = ld_relaxed(cnt_out);  // used on the next hyperplane
    }
    if (act) {
      const int i = fx ? ip : nx - 1 - ip;
      st_cs(Go + row_base + i, gs);
      if (ground_out) a.Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qs;
    }
    __syncthreads();
    // every read of hyperplane d-1's words in this CTA has completed
    if (threadIdx.x == 0 && rank > 0 && d > 0) st_relaxed(cnt_in, d - 1);
  }
  // the last (partial) chunk of outflow rows
  if (periodic) store_outflow((nplanes - 1) / ST_CHUNK);
  cp_async_wait<0>();
}

static const void* octant_st_ptr(bool fp32, int Mo) {
  switch (Mo) {
    case 3: return fp32 ? (const void*)k_dom_octant_st<float, 3> : (const void*)k_dom_octant_st<double, 3>;
    case 6: return fp32 ? (const void*)k_dom_octant_st<float, 6> : (const void*)k_dom_octant_st<double, 6>;
    case 10: return fp32 ? (const void*)k_dom_octant_st<float, 10> : (const void*)k_dom_octant_st<double, 10>;
    default: return nullptr;
  }
}

// ---- path 8: octant clusters sized to run all eight octants at once ----------
// Path 4's lockstep scheme (a cluster per octant, one cluster barrier per
// hyperplane, the upstream CTA's last row read through distributed shared
// memory), with the inputs prefetched into shared memory by cp.async and the
// y-wrap rows staged in chunks as in path 7, and with PPT pencils per thread
// so that a cluster can take more k' rows.  A thread-block cluster must fit
// in one GPC: with one CTA per SM at most 7 clusters of 11-16 CTAs are
// resident on a B200, but 11 of 10 and 15 of 9, so eight octant clusters of
// up to 10 CTAs run in one wave instead of two.  Every cell's arithmetic is
// that of path 4.
struct ClArgs {
  const void* kb;
  const double *ox, *oy, *oz, *w;
  const double* Ig;
  void *Goct, *Qoct, *wrap;
  double I_amb;
  int C, rows, periodic;
  int groups;  // clusters (ordinate groups of MO) per octant
  unsigned down_slots;
  const int* done;  // device flag: nonzero = the source iteration has converged, do nothing
};
// The hyperplane buffers carry a ghost row below the CTA's first row and a
// ghost column left of every row (rows+1 by ny+1 per ordinate): the first
// row's threads put the z-inflow (upstream CTA, ground or ambient) into the
// ghost row and the first column's threads the y-inflow into the ghost
// column, and a pencil's own slot holds the ambient intensity until its
// first cell, so every cell reads its three upwind neighbours the same way.
#define CL_CHUNK 16
// one pencil per thread up to this many pencils per CTA (80 registers a thread),
// else two pencils per thread up to twice this many (at most 96 registers)
#define CL_MAX_THREADS_1 768
#define CL_MAX_THREADS_2 640
struct ClLayout {
  size_t kab, ig, win, wout, buf0, buf1, izt, cix, total;
};
__host__ __device__ inline ClLayout cl_layout(int tsize, int Mo, int rows, int ny, int nz) {
  ClLayout L;
  const size_t S = (size_t)rows * ny;
  const size_t P = (size_t)(rows + 1) * (ny + 1);
  const size_t chunk = (size_t)2 * Mo * rows * CL_CHUNK * tsize;
  size_t o = 0;
  L.kab = o; o = st_up16(o + (size_t)OCT_AHEAD * S * 2 * tsize);
  L.ig = o; o = st_up16(o + (size_t)OCT_AHEAD * ny * sizeof(double));
  L.win = o; o = st_up16(o + chunk);
  L.wout = o; o = st_up16(o + chunk);
  L.buf0 = o; o = st_up16(o + (size_t)Mo * P * tsize);
  L.buf1 = o; o = st_up16(o + (size_t)Mo * P * tsize);
  L.izt = o; o = st_up16(o + (size_t)Mo * nz * tsize);
  L.cix = o; o = st_up16(o + 4 * (size_t)Mo * tsize);
  L.total = o;
  return L;
}

template <typename T, int MO, int PPT>
__global__ void __launch_bounds__(PPT == 1 ? CL_MAX_THREADS_1 : CL_MAX_THREADS_2, 1)
    k_dom_octant_cl(GridDev g, ClArgs a) {
  using T2 = typename Vec2Of<T>::type;
  extern __shared__ __align__(16) unsigned char shraw[];
  // an iteration queued past convergence: every CTA leaves before any
  // cluster barrier or shared-memory traffic
  if (a.done && *(volatile const int*)a.done) return;
  cg::cluster_group cl = cg::this_cluster();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int C = a.C;
  const int rank = (int)cl.block_rank();
  const int part = blockIdx.x / C;  // (octant, ordinate group)
  const int oct = part / a.groups;
  const int grp = part - oct * a.groups;
  const int n0 = part * MO;
  const int rows = a.rows;
  const int S = rows * ny;
  const int RS = ny + 1;           // padded row stride
  const int P = (rows + 1) * RS;   // padded plane per ordinate
  const ClLayout L = cl_layout((int)sizeof(T), MO, rows, ny, nz);
  T2* kab_ring = (T2*)(shraw + L.kab);
  double* ig_ring = (double*)(shraw + L.ig);
  T* win = (T*)(shraw + L.win);
  T* wout = (T*)(shraw + L.wout);
  T* buf0 = (T*)(shraw + L.buf0);
  T* buf1 = (T*)(shraw + L.buf1);
  T* izt = (T*)(shraw + L.izt);
  T* cix = (T*)(shraw + L.cix);
  T* ciy = cix + MO;
  T* cw = ciy + MO;
  T* cwm = cw + MO;
  const T2* kb = (const T2*)a.kb;
  T* Goct = (T*)a.Goct;
  T* Qoct = (T*)a.Qoct;
  T* wrap = (T*)a.wrap;
  const T I_amb = (T)a.I_amb;
  const int nplanes = nx + ny + nz - 2;
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int m = t / nz, k = t - m * nz;
    izt[t] = (T)(fabs(a.oz[n0 + m]) / g.dz[k]);
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    cix[m] = (T)(fabs(a.ox[n0 + m]) / g.dx);
    ciy[m] = (T)(fabs(a.oy[n0 + m]) / g.dy);
    cw[m] = (T)a.w[n0 + m];
    cwm[m] = (T)(a.w[n0 + m] * fabs(a.oz[n0 + m]));
  }
  for (int t = threadIdx.x; t < MO * P; t += blockDim.x) {
    buf0[t] = I_amb;
    buf1[t] = I_amb;
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * rows;
  const int nrows = min(rows, nz - r0);
  const int npen = nrows > 0 ? nrows * ny : 0;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits * a.groups + grp;
  T* Go = Goct + (int64_t)part * N;
  const int64_t wstride = (int64_t)nz * nx;
  T* wrap0 = wrap + (int64_t)n0 * wstride;
  const bool periodic = a.periodic != 0;
  const int TT = blockDim.x;
  const uint64_t keep = l2_policy_evict_last();
  const int chunk_elems = MO * rows * CL_CHUNK;
  auto load_inflow = [&](int c) {
    T* dst = win + (size_t)(c & 1) * chunk_elems;
    for (int e = threadIdx.x; e < chunk_elems; e += TT) {
      const int t = e % CL_CHUNK, rm = e / CL_CHUNK;
      const int rl = rm % rows, m = rm / rows;
      const int ip = c * CL_CHUNK + t - (r0 + rl);
      if (rl < nrows && ip >= 0 && ip < nx) {
        const int kk = fz ? r0 + rl : nz - 1 - (r0 + rl);
        const int i = fx ? ip : nx - 1 - ip;
        cp_async_val(&dst[e], &wrap0[m * wstride + (int64_t)kk * nx + i]);
      }
    }
  };
  auto store_outflow = [&](int c) {
    const T* src = wout + (size_t)(c & 1) * chunk_elems;
    for (int e = threadIdx.x; e < chunk_elems; e += TT) {
      const int t = e % CL_CHUNK, rm = e / CL_CHUNK;
      const int rl = rm % rows, m = rm / rows;
      const int ip = c * CL_CHUNK + t - (ny - 1) - (r0 + rl);
      if (rl < nrows && ip >= 0 && ip < nx) {
        const int kk = fz ? r0 + rl : nz - 1 - (r0 + rl);
        const int i = fx ? ip : nx - 1 - ip;
        wrap0[m * wstride + (int64_t)kk * nx + i] = src[e];
      }
    }
  };
  // per-pencil constants: pencil index, row and column, global row base, roles
  int pq[PPT], pjp[PPT], pkp[PPT], pk[PPT], pqi[PPT];
  int64_t prb[PPT];
  unsigned prole[PPT];  // 1 has, 2 first row, 16 ground flux, 32 ground inflow, 64 last row with a CTA above
#pragma unroll
  for (int pp = 0; pp < PPT; ++pp) {
    const int q = threadIdx.x + pp * TT;
    const bool has = q < npen;
    const int kl = has ? q / ny : 0;
    const int jp = has ? q - kl * ny : 0;
    const int kp = r0 + kl;
    const int k = fz ? kp : nz - 1 - kp;
    const int j = fy ? jp : ny - 1 - jp;
    pq[pp] = q; pjp[pp] = jp; pkp[pp] = kp; pk[pp] = k;
    pqi[pp] = (kl + 1) * RS + jp + 1;
    prb[pp] = ((int64_t)k * ny + j) * nx;
    prole[pp] = (has ? 1u : 0u) | (has && kl == 0 ? 2u : 0u) |
                (has && !fz && k == 0 && slot >= 0 ? 16u : 0u) | (has && fz && kp == 0 ? 32u : 0u) |
                (has && kl == rows - 1 && rank < C - 1 ? 64u : 0u);
  }
  auto prefetch = [&](int d) {
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int ip = d - pjp[pp] - pkp[pp];
      if ((prole[pp] & 1u) && ip >= 0 && ip < nx) {
        const int i = fx ? ip : nx - 1 - ip;
        const int sl = d % OCT_AHEAD;
        cp_async_kb(&kab_ring[(size_t)sl * S + pq[pp]], &kb[prb[pp] + i], keep);
        if (prole[pp] & 32u) {
          const int j = fy ? pjp[pp] : ny - 1 - pjp[pp];
          cp_async8(&ig_ring[(size_t)sl * ny + pjp[pp]], &a.Ig[(int64_t)j * nx + i]);
        }
      }
    }
    // a chunk of inflow rows two hyperplanes before it starts: the first
    // column's ghosts of hyperplane c*CL_CHUNK are written on the one before
    if (periodic && (d + 2) % CL_CHUNK == 0 && d + 2 < nplanes) load_inflow((d + 2) / CL_CHUNK);
    cp_async_commit();
  };
  // Threads t < rows*MO move the y-wrap values between the staged chunks and
  // the hyperplane buffers' first and last columns, one value each, so that no
  // pencil carries that work: the ghost column of hyperplane dn (in the buffer
  // that is then the previous one), and the last column of hyperplane dp.
  const int nmove = rows * MO;
  auto fill_ghost_col = [&](T* buf, int dn) {
    const int t = threadIdx.x;
    if (t < nmove) {
      const int m = t / rows, kl = t - m * rows;
      if (kl < nrows)
        buf[(size_t)m * P + (kl + 1) * RS] =
            periodic ? win[((size_t)(((dn / CL_CHUNK) & 1) * MO + m) * rows + kl) * CL_CHUNK +
                           dn % CL_CHUNK]
                     : I_amb;
    }
  };
  auto copy_last_col = [&](const T* buf, int dp) {
    const int t = threadIdx.x;
    if (periodic && t < nmove) {
      const int m = t / rows, kl = t - m * rows;
      if (kl < nrows)
        wout[((size_t)(((dp / CL_CHUNK) & 1) * MO + m) * rows + kl) * CL_CHUNK + dp % CL_CHUNK] =
            buf[(size_t)m * P + (kl + 1) * RS + ny];
    }
  };
  if (periodic) load_inflow(0);
  for (int d = 0; d < OCT_AHEAD - 1; ++d) prefetch(d);
  cp_async_wait<OCT_AHEAD - 2>();  // group 0, which holds chunk 0 of the inflow rows
  __syncthreads();
  fill_ghost_col(buf1, 0);  // hyperplane 0 reads buf1 as its previous one
  // the first cluster barrier also publishes the ambient-filled buffers
  cluster_arrive_release();
  // the downstream CTA's buffers: this CTA's last row goes straight into their
  // ghost row below the first row (a store before the barrier's release, not
  // a load after its acquire, so its latency is not on the next hyperplane)
  T* dn0 = rank < C - 1 ? cl.map_shared_rank(buf0, rank + 1) : nullptr;
  T* dn1 = rank < C - 1 ? cl.map_shared_rank(buf1, rank + 1) : nullptr;
  for (int d = 0; d < nplanes; ++d) {
    prefetch(d + OCT_AHEAD - 1);  // an empty group past the last plane
    T* cur = (d & 1) ? buf1 : buf0;
    T* prev = (d & 1) ? buf0 : buf1;
    T* dcur = (d & 1) ? dn1 : dn0;
    cp_async_wait<OCT_AHEAD - 1>();  // this plane's group has landed
    cluster_wait_acquire();
    // the last column of hyperplane d-1 into its chunk; a chunk whose last
    // column arrived on the previous hyperplane leaves for global memory
    if (d > 0) copy_last_col(prev, d - 1);
    if (periodic && d > 1 && (d - 1) % CL_CHUNK == 0) store_outflow((d - 1) / CL_CHUNK - 1);
    if (d + 1 < nplanes) fill_ghost_col(cur, d + 1);
    const int sl = d % OCT_AHEAD;
    T gsv[PPT], qsv[PPT];
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int jp = pjp[pp], kp = pkp[pp], qi = pqi[pp];
      const int ip = d - jp - kp;
      const bool act = (prole[pp] & 1u) && ip >= 0 && ip < nx;
      T gs = (T)0, qs = (T)0;
      if (act) {
        // the ground's (or the ambient) z-inflow below the first CTA's first row;
        // the other CTAs' got it from the CTA below on the previous hyperplane
        if ((prole[pp] & 2u) && kp == 0) {
          const T z = fz ? (T)ig_ring[(size_t)sl * ny + jp] : I_amb;
#pragma unroll
          for (int m = 0; m < MO; ++m) prev[(size_t)m * P + jp + 1] = z;
        }
        const T2 kab = kab_ring[(size_t)sl * S + pq[pp]];
        const bool ground_out = (prole[pp] & 16u) != 0;
        const int k = pk[pp];
#pragma unroll
        for (int m = 0; m < MO; ++m) {
          const T* pm = prev + (size_t)m * P + qi;
          const T Ix = pm[0], Iy = pm[-1], Iz = pm[-RS];
          const T ix = cix[m], iy = ciy[m], iz = izt[m * nz + k];
          const T num = kab.y + ix * Ix + iy * Iy + iz * Iz;
          const T den = kab.x + ix + iy + iz;
          const T v = sweep_div(num, den);
          cur[(size_t)m * P + qi] = v;
          if (prole[pp] & 64u) dcur[(size_t)m * P + jp + 1] = v;
          gs = gs + cw[m] * v;
          if (ground_out) qs = qs + cwm[m] * v;
        }
      } else if (prole[pp] & 1u) {
        // before its first cell a pencil's x-inflow is the ambient intensity
#pragma unroll
        for (int m = 0; m < MO; ++m) cur[(size_t)m * P + qi] = I_amb;
      }
      gsv[pp] = gs;
      qsv[pp] = qs;
    }
    cluster_arrive_release();
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int ip = d - pjp[pp] - pkp[pp];
      if ((prole[pp] & 1u) && ip >= 0 && ip < nx) {
        const int i = fx ? ip : nx - 1 - ip;
        st_cs(Go + prb[pp] + i, gsv[pp]);
        if (prole[pp] & 16u) {
          const int j = fy ? pjp[pp] : ny - 1 - pjp[pp];
          Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qsv[pp];
        }
      }
    }
  }
  cluster_wait_acquire();
  // the last hyperplane's last column, then every chunk not yet flushed
  copy_last_col(((nplanes - 1) & 1) ? buf1 : buf0, nplanes - 1);
  __syncthreads();
  if (periodic) {
    for (int c = max(0, (nplanes - 1) / CL_CHUNK - 1); c <= (nplanes - 1) / CL_CHUNK; ++c)
      if ((c + 1) * CL_CHUNK + 1 > nplanes - 1) store_outflow(c);
  }
  cp_async_wait<0>();
}

static const void* octant_cl_ptr(bool fp32, int Mo, int ppt) {
#define CLP(T, M, P) (const void*)k_dom_octant_cl<T, M, P>
  if (ppt == 1) {
    switch (Mo) {
      case 3: return fp32 ? CLP(float, 3, 1) : CLP(double, 3, 1);
      case 5: return fp32 ? CLP(float, 5, 1) : CLP(double, 5, 1);
      case 6: return fp32 ? CLP(float, 6, 1) : CLP(double, 6, 1);
      case 10: return fp32 ? CLP(float, 10, 1) : CLP(double, 10, 1);
    }
  } else if (ppt == 2) {
    switch (Mo) {
      case 3: return fp32 ? CLP(float, 3, 2) : CLP(double, 3, 2);
      case 5: return fp32 ? CLP(float, 5, 2) : CLP(double, 5, 2);
      case 6: return fp32 ? CLP(float, 6, 2) : CLP(double, 6, 2);
      case 10: return fp32 ? CLP(float, 10, 2) : CLP(double, 10, 2);
    }
  }
#undef CLP
  return nullptr;
}

template <int MO, int MINB = 1>
static cudaError_t launch_octant_kernel(const GridDev& g, const OctArgs& a, cudaLaunchConfig_t* cfg) {
  return cudaLaunchKernelEx(cfg, k_dom_octant<MO, MINB>, g, a);
}

template <int MO>
static cudaError_t launch_octant_pipe_kernel(const GridDev& g, const OctArgs& a,
                                             cudaLaunchConfig_t* cfg) {
  return cudaLaunchKernelEx(cfg, k_dom_octant_pipe<MO>, g, a);
}

// pipe: the point-to-point pipelined kernel (path 1), else the cluster-barrier one (paths 4
// and 6, the latter with two clusters per octant of half the ordinates, two CTAs per SM)
static const void* octant_kernel_ptr(int Mo, bool pipe, int groups = 1) {
  if (pipe) {
    switch (Mo) {
      case 3: return (const void*)k_dom_octant_pipe<3>;
      case 6: return (const void*)k_dom_octant_pipe<6>;
      case 10: return (const void*)k_dom_octant_pipe<10>;
      default: return nullptr;
    }
  }
  if (groups == 2) {
    switch (Mo / 2) {
      case 3: return (const void*)k_dom_octant<3, 2>;
      case 5: return (const void*)k_dom_octant<5, 2>;
      default: return nullptr;
    }
  }
  switch (Mo) {
    case 3: return (const void*)k_dom_octant<3>;
    case 6: return (const void*)k_dom_octant<6>;
    case 10: return (const void*)k_dom_octant<10>;
    default: return nullptr;
  }
}

// G = sum over octants of the octant partials (octant order); max G and max |G - G_prev|
__global__ void k_dom_G_oct(int64_t N, int nparts, const double* __restrict__ Goct, double* G,
                            const double* __restrict__ Gp, unsigned long long* keys,
                            const int* done = nullptr) {
  if (done && *done) return;
  unsigned long long bg = 0, bd = 0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N;
       c += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int o = 0; o < nparts; ++o) s += Goct[(int64_t)o * N + c];
    G[c] = s;
    double d = fabs(s - Gp[c]);
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

// q_in at the ground from the downward octants' partial fluxes; ground intensity relaxation
__global__ void k_dom_ground_oct(int n2, int nslots, const double* __restrict__ Qoct,
                                 const double* __restrict__ Isoil, double refl, double relax,
                                 double* Ig, double* qin, const int* done = nullptr) {
  if (done && *done) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  double s = 0.0;
  for (int o = 0; o < nslots; ++o) s += Qoct[(int64_t)o * n2 + q];
  qin[q] = s;
  double Inew = Isoil[q] + refl * s;
  Ig[q] = relax * Inew + (1.0 - relax) * Ig[q];
}

// wrap rows from a full intensity field: wrap[n][k][i] = I[n][k][j_far][i]
// inverse of k_dom_extract_wrap: write the wrap rows into a full intensity field
__global__ void k_dom_scatter_wrap(GridDev g, int M, const double* __restrict__ oy,
                                   const double* __restrict__ wrap, double* I) {
  const int64_t tot = (int64_t)M * g.nz * g.nx;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= tot) return;
  const int n = (int)(t / ((int64_t)g.nz * g.nx));
  const int64_t r = t - (int64_t)n * g.nz * g.nx;
  const int k = (int)(r / g.nx);
  const int i = (int)(r - (int64_t)k * g.nx);
  const int jf = oy[n] >= 0.0 ? g.ny - 1 : 0;
  I[(int64_t)n * ncells_dev(g) + cidx(g, k, jf, i)] = wrap[t];
}

template <typename T>
__global__ void k_dom_extract_wrap(GridDev g, int M, const double* __restrict__ oy,
                                   const double* __restrict__ I, T* wrap) {
  const int64_t tot = (int64_t)M * g.nz * g.nx;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= tot) return;
  const int n = (int)(t / ((int64_t)g.nz * g.nx));
  const int64_t r = t - (int64_t)n * g.nz * g.nx;
  const int k = (int)(r / g.nx);
  const int i = (int)(r - (int64_t)k * g.nx);
  const int jf = oy[n] >= 0.0 ? g.ny - 1 : 0;
  wrap[t] = (T)I[(int64_t)n * ncells_dev(g) + cidx(g, k, jf, i)];
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
  D->I = nullptr; D->wrap = nullptr; D->kb = nullptr; D->Goct = nullptr; D->Qoct = nullptr;
  D->mode = 0; D->mode_req = 0; D->force_C = 0; D->groups = 1;
  D->fp32 = 0; D->kb32 = nullptr; D->Goct32 = nullptr; D->Qoct32 = nullptr; D->wrap32 = nullptr;
  D->st_ring = nullptr; D->st_ring_bytes = 0; D->st_cnt_offset = 0;
  D->cl_ppt = 1; D->cl_active = 0; D->force_groups = 0; D->begun = 0; D->pend_I_amb = 0.0;
  cudaMalloc(&D->G, sizeof(double) * N); cudaMalloc(&D->Gp, sizeof(double) * N);
  cudaMemset(D->G, 0, sizeof(double) * N);
  cudaMalloc(&D->ks, sizeof(double) * N); cudaMalloc(&D->kg, sizeof(double) * N);
  cudaMalloc(&D->ksafe, sizeof(double) * N); cudaMalloc(&D->B, sizeof(double) * N);
  cudaMalloc(&D->Ig_out, sizeof(double) * n2); cudaMalloc(&D->Isoil, sizeof(double) * n2);
  cudaMalloc(&D->qin, sizeof(double) * n2);
  cudaMalloc(&D->keys, sizeof(unsigned long long) * 4);
  cudaMallocHost(&D->h_keys, sizeof(unsigned long long) * 4);
  cudaMalloc(&D->dstate, sizeof(int) * 4);
  cudaMallocHost(&D->h_dstate, sizeof(int) * 4);
  D->eps_w = 0.85; D->tol = 1.0e-3; D->relax = 0.7; D->kgmax = kgmax; D->max_iter = 30;
  D->last_iters = 0;
  D->timing = 0; D->sweep_ms = 0.0; D->sweep_count = 0;
  for (int q = 0; q < 32; ++q) {
    cudaEventCreate(&D->ev0[q]);
    cudaEventCreate(&D->ev1[q]);
  }
  // the copies and the clearing above run on the legacy default stream; wait
  // for them here, since the solves run on streams that do not order after it
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    dom_destroy(D);
    return nullptr;
  }
  return D;
}

void dom_destroy(void* h) {
  DomCtx* D = (DomCtx*)h;
  if (!D) return;
  cudaFree(D->ox); cudaFree(D->oy); cudaFree(D->oz); cudaFree(D->w); cudaFree(D->I);
  cudaFree(D->wrap); cudaFree(D->kb); cudaFree(D->Goct); cudaFree(D->Qoct);
  cudaFree(D->kb32); cudaFree(D->Goct32); cudaFree(D->Qoct32); cudaFree(D->wrap32);
  cudaFree(D->st_ring);
  cudaFree(D->G); cudaFree(D->Gp); cudaFree(D->ks); cudaFree(D->kg); cudaFree(D->ksafe);
  cudaFree(D->B); cudaFree(D->Ig_out); cudaFree(D->Isoil); cudaFree(D->qin); cudaFree(D->keys);
  cudaFreeHost(D->h_keys);
  cudaFree(D->dstate);
  cudaFreeHost(D->h_dstate);
  for (int q = 0; q < 32; ++q) {
    cudaEventDestroy(D->ev0[q]);
    cudaEventDestroy(D->ev1[q]);
  }
  delete D;
}

// Octant grouping required by path 1: M = 8*Mo, ordinates octant-major, every
// ordinate of a group with the same signs and no zero component.
static bool octant_grouping(const DomCtx* D) {
  if (D->M % 8 != 0) return false;
  const int Mo = D->M / 8;
  for (int o = 0; o < 8; ++o) {
    const int n0 = o * Mo;
    for (int m = 0; m < Mo; ++m) {
      const int n = n0 + m;
      if (D->hox[n] == 0.0 || D->hoy[n] == 0.0 || D->hoz[n] == 0.0) return false;
      if ((D->hox[n] > 0) != (D->hox[n0] > 0) || (D->hoy[n] > 0) != (D->hoy[n0] > 0) ||
          (D->hoz[n] > 0) != (D->hoz[n0] > 0))
        return false;
    }
  }
  return true;
}

// Pick the cluster size (CTAs per octant) and launch shape for path 1; false if none fits.
// kind: 4 cluster barrier per hyperplane, 1 mbarrier pipeline
static bool plan_clusters(DomCtx* D, int force_C, int kind, int groups = 1) {
  const GridDev& g = D->g;
  const int Mo = D->M / 8 / groups;
  const bool pipe = kind == 1;
  int dev = 0, optin = 0, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  const void* fn = D->fp32 ? octant_f32_ptr(Mo) : octant_kernel_ptr(Mo * groups, pipe, groups);
  if (!fn) return false;
  cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  double best = 1e300;
  bool found = false;
  for (int C = 16; C >= 1; --C) {
    if (force_C > 0 && C != force_C) continue;
    const int rows = (g.nz + C - 1) / C;
    if ((g.nz + rows - 1) / rows != C) continue;  // same split as a smaller cluster
    int threads = ((rows * g.ny + 31) / 32) * 32;
    if (threads > OCT_MAX_THREADS) continue;
    const size_t need = pipe ? oct_pipe_smem_bytes(Mo, rows, g.ny, g.nz)
                             : (D->fp32 ? oct_smem_bytes(Mo, rows, g.ny, g.nz) / 2
                                        : oct_smem_bytes(Mo, rows, g.ny, g.nz));
    if (need > (size_t)optin) continue;
    // ask for more than half an SM's shared memory so that no two CTAs share an SM,
    // unless that leaves fewer than 8 clusters resident
    size_t pad = groups > 1 ? need : (size_t)smem_sm / 2 + 1024;
    size_t trial[2] = {need > pad ? need : (pad <= (size_t)optin ? pad : need), need};
    for (int t = 0; t < 2; ++t) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(8 * groups * C); cfg.blockDim = dim3(threads);
      cfg.dynamicSmemBytes = trial[t]; cfg.attrs = at; cfg.numAttrs = 1;
      int active = 0;
      if (cudaOccupancyMaxActiveClusters(&active, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        active = 0;
      }
      if (active < 1) continue;
      const int waves = (8 + active - 1) / active;
      const int per_thread = (rows * g.ny + threads - 1) / threads;
      double cost = (double)waves * per_thread * (t == 0 ? 1.0 : (active >= 8 ? 1.5 : 2.0));
      if (groups > 1) cost = (double)((8 * groups + active - 1) / active) * 0.5;
      if (cost < best) {
        best = cost; found = true;
        D->cl_C = C; D->cl_rows = rows; D->cl_threads = threads; D->cl_smem = trial[t];
      }
      if (t == 0 && active >= 8) break;
    }
  }
  return found;
}

// Launch shape of path 7: CTAs per octant C (k' rows split as in path 4), one
// CTA per SM, and all 8*C CTAs resident at once (the hand-off waits on other
// CTAs, so the grid is launched cooperatively); false if it does not fit.
static bool plan_st(DomCtx* D, int force_C) {
  const GridDev& g = D->g;
  const int Mo = D->M / 8;
  const int tsize = D->fp32 ? (int)sizeof(float) : (int)sizeof(double);
  if (g.nx + g.ny + g.nz - 2 >= (1 << 30)) return false;
  int dev = 0, optin = 0, smem_sm = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const void* fn = octant_st_ptr(D->fp32 != 0, Mo);
  if (!fn) return false;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  // the largest C (fewest rows per CTA) whose 8*C CTAs fit one per SM
  for (int C = 64; C >= 1; --C) {
    if (force_C > 0 && C != force_C) continue;
    const int rows = (g.nz + C - 1) / C;
    if ((g.nz + rows - 1) / rows != C) continue;
    const int threads = ((rows * g.ny + 31) / 32) * 32;
    if (threads > OCT_MAX_THREADS || 8 * C > nsm) continue;
    const size_t need = st_layout(tsize, Mo, rows, g.ny, g.nz).total;
    const size_t pad = (size_t)smem_sm / 2 + 1024;  // no two CTAs on one SM
    const size_t smem = need > pad ? need : pad;
    if (smem > (size_t)optin) continue;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (per_sm < 1 || (int64_t)per_sm * nsm < 8 * C) continue;
    D->cl_C = C; D->cl_rows = rows; D->cl_threads = threads; D->cl_smem = smem;
    D->cl_lg_ring = ST_RING_LG;
    return true;
  }
  return false;
}

// Launch shape of path 8: ordinate groups per octant (1, or 2 when the octant's
// ordinates split evenly), cluster size C (k' rows per CTA), pencils per
// thread (1 or 2), one CTA per SM.  One cluster per octant is kept whenever
// all eight clusters are resident at once: two clusters per octant take more
// SMs for about the same sweep time, and the SMs left free are the ones the
// concurrent projection and k-epsilon run on (measured: 23.4 against 22.8 ms
// per step).  Otherwise the configuration with the fewest waves times work per
// CTA per hyperplane (pencils x ordinates) wins.  force_C / D->force_groups
// pin C / the grouping (0: free).
static bool plan_cl(DomCtx* D, int force_C) {
  const int force_groups = D->force_groups;
  const GridDev& g = D->g;
  const int MoAll = D->M / 8;
  const int tsize = D->fp32 ? (int)sizeof(float) : (int)sizeof(double);
  int dev = 0, optin = 0, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  double best = 1e300;
  bool found = false;
  for (int groups = 1; groups <= 2; ++groups) {
    if (force_groups > 0 && groups != force_groups) continue;
    if (MoAll % groups != 0) continue;
    if (found && D->cl_active >= 8) break;  // one cluster per octant, all resident
    const int Mo = MoAll / groups;
    for (int C = 16; C >= 1; --C) {
      if (force_C > 0 && C != force_C) continue;
      const int rows = (g.nz + C - 1) / C;
      if ((g.nz + rows - 1) / rows != C) continue;
      const int pencils = rows * g.ny;
      const int ppt = pencils <= CL_MAX_THREADS_1 ? 1 : (pencils <= 2 * CL_MAX_THREADS_2 ? 2 : 0);
      if (ppt == 0) continue;
      const int threads = ((pencils + ppt - 1) / ppt + 31) / 32 * 32;
      const void* fn = octant_cl_ptr(D->fp32 != 0, Mo, ppt);
      if (!fn) continue;
      cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
      const size_t need = cl_layout(tsize, Mo, rows, g.ny, g.nz).total;
      const size_t pad = (size_t)smem_sm / 2 + 1024;  // no two CTAs on one SM
      const size_t smem = need > pad ? need : pad;
      if (smem > (size_t)optin) continue;
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(8 * groups * C); cfg.blockDim = dim3(threads);
      cfg.dynamicSmemBytes = smem; cfg.attrs = at; cfg.numAttrs = 1;
      int active = 0;
      if (cudaOccupancyMaxActiveClusters(&active, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        active = 0;
      }
      if (active < 1) continue;
      const int waves = (8 * groups + active - 1) / active;
      const double cost = (double)waves * pencils * Mo;
      if (cost < best) {
        best = cost; found = true;
        D->cl_C = C; D->cl_rows = rows; D->cl_threads = threads; D->cl_smem = smem;
        D->cl_ppt = ppt; D->groups = groups;
        D->cl_active = waves == 1 ? 8 : 0;  // 8: every cluster resident at once
      }
    }
  }
  return found;
}

static void alloc_st_ring(DomCtx* D) {
  const int tsize = D->fp32 ? (int)sizeof(float) : (int)sizeof(double);
  const size_t bounds = (size_t)8 * (D->cl_C - 1);
  const size_t words = bounds * ((size_t)1 << D->cl_lg_ring) * D->Mo * D->g.ny;
  D->st_cnt_offset = (words * tsize + 255) & ~(size_t)255;
  D->st_ring_bytes = D->st_cnt_offset + sizeof(int) * (bounds > 0 ? bounds : 1);
  cudaMalloc(&D->st_ring, D->st_ring_bytes);
}

// The first call (at the first solve or intensity access) allocates the
// sweep's buffers and clears the y-inflow rows on the caller's stream, so the
// clearing is ordered before that stream's first sweep (a plain cudaMemset
// runs on the legacy default stream, which does not order work on streams
// created non-blocking, such as torch's side streams).
static int dom_prepare(DomCtx* D, cudaStream_t st) {
  if (D->mode != 0) return FS_OK;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const int want = D->mode_req;
  // auto: path 8 when all eight octant clusters can be resident at once, else path 4
  const bool auto8 = want == 0 && octant_grouping(D) && plan_cl(D, D->force_C) && D->cl_active >= 8;
  if (D->fp32) {
    const int kind = auto8 ? 8 : ((want == 7 || want == 8) ? want : 4);
    if ((want != 0 && want != 4 && want != 7 && want != 8) || !octant_grouping(D) ||
        !(kind == 7 ? plan_st(D, D->force_C)
                    : (kind == 8 ? plan_cl(D, D->force_C) : plan_clusters(D, D->force_C, kind)))) {
      fs_set_error("single-precision sweep needs an octant path (4, 7 or 8) on this grid");
      return FS_EARG;
    }
    D->mode = kind;
    if (kind != 8) D->groups = 1;  // path 8 planned its own grouping
    D->Mo = D->M / 8;
    int slot = 0;
    for (int o = 0; o < 8; ++o) D->down_slot[o] = D->hoz[o * D->Mo] < 0.0 ? slot++ : -1;
    cudaMalloc(&D->kb32, sizeof(float2) * N);
    cudaMalloc(&D->Goct32, sizeof(float) * 8 * D->groups * N);
    cudaMalloc(&D->Qoct32, sizeof(float) * 8 * D->groups * n2);
    cudaMalloc(&D->wrap32, sizeof(float) * D->M * g.nz * g.nx);
    cudaMemsetAsync(D->wrap32, 0, sizeof(float) * D->M * g.nz * g.nx, st);
    if (D->mode == 7) alloc_st_ring(D);
    return cuda_status();
  }
  // auto picks the cluster-barrier sweep (path 4), measured faster than path 1
  const int groups = (want == 6 && D->M % 16 == 0) ? 2 : 1;
  const int kind = auto8 ? 8 : ((want == 1 || want == 7 || want == 8) ? want : 4);
  if ((want == 0 || want == 1 || want == 4 || want == 6 || want == 7 || want == 8) &&
      octant_grouping(D) &&
      (kind == 7 ? plan_st(D, D->force_C)
                 : (kind == 8 ? plan_cl(D, D->force_C) : plan_clusters(D, D->force_C, kind, groups)))) {
    D->mode = kind == 8 ? 8 : (want == 1 ? 1 : (want == 6 ? 6 : (want == 7 ? 7 : 4)));
    if (kind != 8) D->groups = groups;  // path 8 planned its own grouping
    D->Mo = D->M / 8;
    int slot = 0;
    for (int o = 0; o < 8; ++o) D->down_slot[o] = D->hoz[o * D->Mo] < 0.0 ? slot++ : -1;
    cudaMalloc(&D->kb, sizeof(double2) * N);
    cudaMalloc(&D->Goct, sizeof(double) * 8 * D->groups * N);
    cudaMalloc(&D->Qoct, sizeof(double) * 8 * D->groups * n2);
    cudaMalloc(&D->wrap, sizeof(double) * D->M * g.nz * g.nx);
    cudaMemsetAsync(D->wrap, 0, sizeof(double) * D->M * g.nz * g.nx, st);
    if (D->mode == 7) alloc_st_ring(D);
    return cuda_status();
  }
  if (want == 1 || want == 4 || want == 6 || want == 7 || want == 8) {
    fs_set_error("octant-cluster sweep not possible for this grid or quadrature");
    return FS_EARG;
  }
  const size_t smem = sizeof(double) * 2 * (size_t)g.ny * g.nz;
  int max_smem = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const bool ord_ok = ord_smem_bytes(g.ny, g.nz) <= (size_t)max_smem &&
                      (int64_t)g.ny * g.nz <= 8 * 1024 && g.ny + g.nz <= 1024;
  if (want == 5 && !ord_ok) {
    fs_set_error("per-ordinate register sweep not possible for this grid");
    return FS_EARG;
  }
  if (want == 5) {
    D->mode = 5;
    cudaMalloc(&D->kb, sizeof(double2) * N);
  } else {
    D->mode = (want == 3 || smem > (size_t)max_smem) ? 3 : 2;
  }
  cudaMalloc(&D->I, sizeof(double) * N * D->M);
  cudaMemsetAsync(D->I, 0, sizeof(double) * N * D->M, st);
  return cuda_status();
}

int dom_set_mode(void* h, int mode, int cluster_ctas) {
  DomCtx* D = (DomCtx*)h;
  if (mode < 0 || mode > 8 || cluster_ctas < 0 || cluster_ctas > (mode == 7 ? 64 : 16))
    return FS_EARG;
  if (D->mode != 0) {
    fs_set_error("sweep mode must be set before the first solve or intensity load");
    return FS_EARG;
  }
  D->mode_req = mode;
  D->force_C = cluster_ctas;
  return FS_OK;
}

int dom_mode(void* h) { return ((DomCtx*)h)->mode; }

int dom_set_groups(void* h, int groups) {
  DomCtx* D = (DomCtx*)h;
  if (groups < 0 || groups > 2) return FS_EARG;
  if (D->mode != 0) {
    fs_set_error("ordinate groups must be set before the first solve or intensity load");
    return FS_EARG;
  }
  D->force_groups = groups;
  return FS_OK;
}

int dom_set_precision(void* h, int fp32) {
  DomCtx* D = (DomCtx*)h;
  if (D->mode != 0) {
    fs_set_error("precision must be set before the first solve or intensity load");
    return FS_EARG;
  }
  D->fp32 = fp32 ? 1 : 0;
  return FS_OK;
}

int dom_load_intensity(void* h, const double* I_full, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  int rc = dom_prepare(D, st);
  if (rc != FS_OK) return rc;
  const GridDev& g = D->g;
  if (D->fp32) {
    const int64_t tot = (int64_t)D->M * g.nz * g.nx;
    k_dom_extract_wrap<float><<<blocks_for(tot, 256), 256, 0, st>>>(g, D->M, D->oy, I_full,
                                                                   D->wrap32);
    fs_count_launch();
  } else if (D->mode == 1 || D->mode == 4 || D->mode == 6 || D->mode == 7 || D->mode == 8) {
    const int64_t tot = (int64_t)D->M * g.nz * g.nx;
    k_dom_extract_wrap<double><<<blocks_for(tot, 256), 256, 0, st>>>(g, D->M, D->oy, I_full,
                                                                    D->wrap);
    fs_count_launch();
  } else {
    cudaMemcpyAsync(D->I, I_full, sizeof(double) * ncells(g) * D->M, cudaMemcpyDeviceToDevice,
                    st);
  }
  return cuda_status();
}

int64_t dom_wrap_size(void* h) {
  DomCtx* D = (DomCtx*)h;
  return (int64_t)D->M * D->g.nz * D->g.nx;
}

// The persistent part of the intensities (the y-inflow rows a later sweep
// reads), M x Nz x Nx, out of or into whichever storage the sweep path uses.
int dom_get_wrap(void* h, double* dst, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  int rc = dom_prepare(D, st);
  if (rc != FS_OK) return rc;
  const int64_t tot = dom_wrap_size(h);
  if (D->fp32) {
    k_f32_to_f64<<<blocks_for(tot, 256), 256, 0, st>>>(tot, D->wrap32, dst);
    fs_count_launch();
  } else if (D->mode == 1 || D->mode == 4 || D->mode == 6 || D->mode == 7 || D->mode == 8) {
    cudaMemcpyAsync(dst, D->wrap, sizeof(double) * tot, cudaMemcpyDeviceToDevice, st);
  } else {
    k_dom_extract_wrap<double><<<blocks_for(tot, 256), 256, 0, st>>>(D->g, D->M, D->oy, D->I,
                                                                    dst);
    fs_count_launch();
  }
  return cuda_status();
}

int dom_set_wrap(void* h, const double* src, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  int rc = dom_prepare(D, st);
  if (rc != FS_OK) return rc;
  const int64_t tot = dom_wrap_size(h);
  if (D->fp32) {
    k_f64_to_f32<<<blocks_for(tot, 256), 256, 0, st>>>(tot, src, D->wrap32);
    fs_count_launch();
  } else if (D->mode == 1 || D->mode == 4 || D->mode == 6 || D->mode == 7 || D->mode == 8) {
    cudaMemcpyAsync(D->wrap, src, sizeof(double) * tot, cudaMemcpyDeviceToDevice, st);
  } else {
    k_dom_scatter_wrap<<<blocks_for(tot, 256), 256, 0, st>>>(D->g, D->M, D->oy, src, D->I);
    fs_count_launch();
  }
  return cuda_status();
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

static int launch_octant_sweep(DomCtx* D, const OctArgs& a, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = D->cl_C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(8 * D->groups * D->cl_C);
  cfg.blockDim = dim3(D->cl_threads);
  cfg.dynamicSmemBytes = D->cl_smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e;
  const bool pipe = D->mode == 1;
  if (D->groups == 2) {
    switch (D->Mo / 2) {
      case 3: e = launch_octant_kernel<3, 2>(D->g, a, &cfg); break;
      case 5: e = launch_octant_kernel<5, 2>(D->g, a, &cfg); break;
      default: e = cudaErrorInvalidValue;
    }
    fs_count_launch();
    return e == cudaSuccess ? FS_OK : FS_ECUDA;
  }
  switch (D->Mo) {
    case 3: e = pipe ? launch_octant_pipe_kernel<3>(D->g, a, &cfg)
                     : launch_octant_kernel<3>(D->g, a, &cfg); break;
    case 6: e = pipe ? launch_octant_pipe_kernel<6>(D->g, a, &cfg)
                     : launch_octant_kernel<6>(D->g, a, &cfg); break;
    case 10: e = pipe ? launch_octant_pipe_kernel<10>(D->g, a, &cfg)
                      : launch_octant_kernel<10>(D->g, a, &cfg); break;
    default: e = cudaErrorInvalidValue;
  }
  fs_count_launch();
  return e == cudaSuccess ? FS_OK : FS_ECUDA;
}

static int launch_cl_sweep(DomCtx* D, const ClArgs& a, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = D->cl_C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(8 * D->groups * D->cl_C);
  cfg.blockDim = dim3(D->cl_threads);
  cfg.dynamicSmemBytes = D->cl_smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = cudaErrorInvalidValue;
  const bool f = D->fp32 != 0;
#define CLL(T, M, P) e = cudaLaunchKernelEx(&cfg, k_dom_octant_cl<T, M, P>, D->g, a)
  switch ((D->Mo / D->groups) * 4 + D->cl_ppt) {
    case 3 * 4 + 1: if (f) CLL(float, 3, 1); else CLL(double, 3, 1); break;
    case 5 * 4 + 1: if (f) CLL(float, 5, 1); else CLL(double, 5, 1); break;
    case 6 * 4 + 1: if (f) CLL(float, 6, 1); else CLL(double, 6, 1); break;
    case 10 * 4 + 1: if (f) CLL(float, 10, 1); else CLL(double, 10, 1); break;
    case 3 * 4 + 2: if (f) CLL(float, 3, 2); else CLL(double, 3, 2); break;
    case 5 * 4 + 2: if (f) CLL(float, 5, 2); else CLL(double, 5, 2); break;
    case 6 * 4 + 2: if (f) CLL(float, 6, 2); else CLL(double, 6, 2); break;
    case 10 * 4 + 2: if (f) CLL(float, 10, 2); else CLL(double, 10, 2); break;
  }
#undef CLL
  fs_count_launch();
  return e == cudaSuccess ? FS_OK : FS_ECUDA;
}

template <typename T>
static int launch_st_sweep(DomCtx* D, StArgs<T> a, cudaStream_t st) {
  // every word of the ring back to "sign bit set" and every read count to -1
  if (cudaMemsetAsync(D->st_ring, 0xff, D->st_ring_bytes, st) != cudaSuccess) return FS_ECUDA;
  a.ring = (typename WordOf<T>::type*)D->st_ring;
  a.consumed = (int*)((char*)D->st_ring + D->st_cnt_offset);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.gridDim = dim3(8 * D->cl_C);
  cfg.blockDim = dim3(D->cl_threads);
  cfg.dynamicSmemBytes = D->cl_smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e;
  switch (D->Mo) {
    case 3: e = cudaLaunchKernelEx(&cfg, k_dom_octant_st<T, 3>, D->g, a); break;
    case 6: e = cudaLaunchKernelEx(&cfg, k_dom_octant_st<T, 6>, D->g, a); break;
    case 10: e = cudaLaunchKernelEx(&cfg, k_dom_octant_st<T, 10>, D->g, a); break;
    default: e = cudaErrorInvalidValue;
  }
  fs_count_launch();
  return e == cudaSuccess ? FS_OK : FS_ECUDA;
}

template <int PPT, int TPB>
static void ord_launch(DomCtx* D, const OrdArgs& oa, size_t smem, cudaStream_t st) {
  cudaFuncSetAttribute(k_dom_ord<PPT, TPB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  k_dom_ord<PPT, TPB><<<D->M, TPB, smem, st>>>(D->g, oa);
}

static int launch_ord_sweep(DomCtx* D, double I_amb, cudaStream_t st) {
  const GridDev& g = D->g;
  const int npen = g.ny * g.nz;
  OrdArgs oa{};
  oa.ox = D->ox; oa.oy = D->oy; oa.oz = D->oz; oa.I = D->I; oa.kb = D->kb; oa.Ig = D->Ig_out;
  oa.I_amb = I_amb; oa.periodic = 1;
  const size_t smem = ord_smem_bytes(g.ny, g.nz);
  // pencils per thread at 1024 threads per ordinate (the staging threads need ny+nz)
  if (g.ny + g.nz > 1024 || ncells(g) >= (int64_t)1 << 31) return FS_EARG;
  const int need = (npen + 1023) / 1024;
  if (need <= 1) ord_launch<1, 1024>(D, oa, smem, st);
  else if (need <= 2) ord_launch<2, 1024>(D, oa, smem, st);
  else if (need <= 4) ord_launch<4, 1024>(D, oa, smem, st);
  else if (need <= 8) ord_launch<8, 1024>(D, oa, smem, st);
  else return FS_EARG;
  fs_count_launch();
  return cudaGetLastError() == cudaSuccess ? FS_OK : FS_ECUDA;
}

// The first half of a solve: absorption, emission and the ground's own
// emission from the caller's fields.  Once this work has run on the stream,
// the solve reads none of those fields again, so the caller may change them
// while dom_end's sweeps run.
int dom_begin(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH,
              const double* rho, const double* Mloc, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  int rc = dom_prepare(D, st);
  if (rc != FS_OK) return rc;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const bool octp = D->mode == 1 || D->mode == 4 || D->mode == 6 || D->mode == 7 || D->mode == 8;
  const double Tamb4 = pow(T_amb, 4.0);
  k_dom_setup<<<blocks_for(N, 256), 256, 0, st>>>(g, Ts, Tg, as, om, YH, rho, Mloc, sigma, Tamb4,
                                                  D->kgmax, D->ks, D->kg, D->ksafe, D->B,
                                                  (!D->fp32 && (octp || D->mode == 5)) ? D->kb : nullptr,
                                                  D->fp32 ? D->kb32 : nullptr);
  fs_count_launch();
  const double I_amb = SIGMA_SB_D * Tamb4 / PI_D;
  k_dom_ground_init<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, Tsoil0, D->eps_w, I_amb, D->Isoil,
                                                        D->Ig_out);
  fs_count_launch();
  D->pend_I_amb = I_amb;
  D->begun = 1;
  return cuda_status();
}

int dom_solve(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH, const double* rho,
              const double* Mloc, double* q_solid, double* q_gas, double* q_in_soil,
              cudaStream_t st) {
  int rc = dom_begin(h, Ts, Tg, as, om, sigma, T_amb, Tsoil0, YH, rho, Mloc, st);
  if (rc != FS_OK) return rc;
  return dom_end(h, q_solid, q_gas, q_in_soil, st);
}

// The second half: the source iterations and the radiative sources.
// End of queued source iteration q: the host loop's test (dom_end) on the
// device.  st: [0] done, [1] iterations run, [2] error (1 stalled hand-off,
// 2 non-finite G).
__global__ void k_dom_check(const unsigned long long* __restrict__ keys, double tol, int q,
                            int* st) {
  if (st[0]) return;
  // a stalled hand-off or a non-finite G ends the solve on every iteration,
  // the first included; only the convergence ratio waits for a second one
  if (keys[2] != 0) { st[2] = 1; st[1] = q + 1; st[0] = 1; return; }
  double Gmax = __longlong_as_double((long long)keys[0]);
  const double dmax = __longlong_as_double((long long)keys[1]);
  if (Gmax != Gmax || dmax != dmax) { st[2] = 2; st[1] = q + 1; st[0] = 1; return; }
  if (q == 0) return;
  if (Gmax < 1e-12) Gmax = 1e-12;
  if (dmax / Gmax < tol) { st[1] = q + 1; st[0] = 1; }
}

// Path 8's source iterations without a host round trip between sweeps: the
// iterations are queued in batches (the first as long as the previous solve),
// every kernel of an iteration queued past convergence returns at once (the
// flag k_dom_check sets), and the host reads the flag once per batch.  The
// iterations that run, their order and their results are the host loop's.
static int dom_iterate_dev(DomCtx* D, const ClArgs& base, int nslots, double refl,
                           cudaStream_t st, int* iters_out) {
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  unsigned nb = blocks_for(N, 256);
  if (nb > 1184) nb = 1184;
  cudaMemsetAsync(D->dstate, 0, sizeof(int) * 4, st);
  int queued = 0;
  int batch = D->last_iters > 2 ? D->last_iters : 2;
  int it = 0;
  while (true) {
    for (int q = 0; q < batch && queued < D->max_iter; ++q, ++queued) {
      std::swap(D->G, D->Gp);
      if (D->timing) cudaEventRecord(D->ev0[queued], st);
      ClArgs ca = base;
      ca.done = D->dstate;
      int rc = launch_cl_sweep(D, ca, st);
      if (rc != FS_OK) return rc;
      if (D->timing) cudaEventRecord(D->ev1[queued], st);
      cudaMemsetAsync(D->keys, 0, sizeof(unsigned long long) * 2, st);
      if (D->fp32) {
        k_dom_G_oct32<<<nb, 256, 0, st>>>(N, 8 * D->groups, D->Goct32, D->G, D->Gp, D->keys,
                                          D->dstate);
        k_dom_ground_oct32<<<blocks_for(n2, 128), 128, 0, st>>>(
            (int)n2, nslots, D->Qoct32, D->Isoil, refl, D->relax, D->Ig_out, D->qin, D->dstate);
      } else {
        k_dom_G_oct<<<nb, 256, 0, st>>>(N, 8 * D->groups, D->Goct, D->G, D->Gp, D->keys,
                                        D->dstate);
        k_dom_ground_oct<<<blocks_for(n2, 128), 128, 0, st>>>(
            (int)n2, nslots, D->Qoct, D->Isoil, refl, D->relax, D->Ig_out, D->qin, D->dstate);
      }
      k_dom_check<<<1, 1, 0, st>>>(D->keys, D->tol, queued, D->dstate);
      fs_count_launch(); fs_count_launch(); fs_count_launch();
    }
    cudaMemcpyAsync(D->h_dstate, D->dstate, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
    if (D->h_dstate[2] == 1) {
      fs_set_error("fs_dom_solve: pipelined sweep wait gave up (hand-off between CTAs stalled)");
      return FS_ETIMEOUT;
    }
    if (D->h_dstate[2] == 2) return FS_ENONFINITE;
    if (D->h_dstate[0]) { it = D->h_dstate[1]; break; }
    if (queued >= D->max_iter) { it = queued; break; }
    batch = 1;
  }
  // the host swapped G and Gp once per queued iteration; undo the swaps of
  // the iterations that returned at once
  if ((queued - it) & 1) std::swap(D->G, D->Gp);
  *iters_out = it;
  return FS_OK;
}

int dom_end(void* h, double* q_solid, double* q_gas, double* q_in_soil, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  if (!D->begun) {
    fs_set_error("dom_end without a dom_begin");
    return FS_EARG;
  }
  D->begun = 0;
  int rc = FS_OK;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const int M = D->M;
  const bool octp = D->mode == 1 || D->mode == 4 || D->mode == 6 || D->mode == 7 || D->mode == 8;
  const double I_amb = D->pend_I_amb;
  SweepArgs a{};
  a.ox = D->ox; a.oy = D->oy; a.oz = D->oz; a.I = D->I; a.ksafe = D->ksafe; a.B = D->B;
  a.Ig = D->Ig_out; a.I_amb = I_amb; a.inv_dx = 1.0 / g.dx; a.inv_dy = 1.0 / g.dy; a.M = M;
  a.periodic = 1;
  OctArgs oa{};
  if (octp) {
    oa.kb = D->kb; oa.ox = D->ox; oa.oy = D->oy; oa.oz = D->oz; oa.w = D->w; oa.Ig = D->Ig_out;
    oa.Goct = D->Goct; oa.Qoct = D->Qoct; oa.wrap = D->wrap; oa.I_amb = I_amb; oa.Mo = D->Mo;
    oa.C = D->cl_C; oa.rows = D->cl_rows; oa.periodic = 1;
    oa.groups = D->groups;
    oa.err = (int*)(D->keys + 2);
    oa.down_slots = 0;
    for (int o = 0; o < 8; ++o)
      oa.down_slots |= (unsigned)(D->down_slot[o] >= 0 ? D->down_slot[o] : 15) << (4 * o);
  }
  int nslots = 0;
  for (int o = 0; o < 8; ++o) nslots += (octp && D->down_slot[o] >= 0) ? D->groups : 0;
  const int nplanes = g.nx + g.ny + g.nz - 2;
  const int64_t nthr = (int64_t)g.ny * g.nz * M;
  const double refl = (1.0 - D->eps_w) / PI_D;
  const size_t smem = sizeof(double) * 2 * (size_t)g.ny * g.nz;
  if (D->mode == 2)
    cudaFuncSetAttribute(k_dom_sweep_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  cudaMemsetAsync(D->keys + 2, 0, sizeof(unsigned long long), st);
  int it = 0;
  if (D->mode == 8) {
    ClArgs ca{};
    ca.kb = D->fp32 ? (const void*)D->kb32 : (const void*)D->kb;
    ca.Goct = D->fp32 ? (void*)D->Goct32 : (void*)D->Goct;
    ca.Qoct = D->fp32 ? (void*)D->Qoct32 : (void*)D->Qoct;
    ca.wrap = D->fp32 ? (void*)D->wrap32 : (void*)D->wrap;
    ca.I_amb = I_amb;
    ca.ox = D->ox; ca.oy = D->oy; ca.oz = D->oz; ca.w = D->w; ca.Ig = D->Ig_out;
    ca.C = D->cl_C; ca.rows = D->cl_rows; ca.periodic = 1; ca.down_slots = oa.down_slots;
    ca.groups = D->groups;
    rc = dom_iterate_dev(D, ca, nslots, refl, st, &it);
    if (rc != FS_OK) return rc;
  } else
  for (it = 0; it < D->max_iter; ++it) {
    std::swap(D->G, D->Gp);
    if (D->timing) cudaEventRecord(D->ev0[it], st);
    if (D->mode == 8) {
      ClArgs ca{};
      ca.kb = D->fp32 ? (const void*)D->kb32 : (const void*)D->kb;
      ca.Goct = D->fp32 ? (void*)D->Goct32 : (void*)D->Goct;
      ca.Qoct = D->fp32 ? (void*)D->Qoct32 : (void*)D->Qoct;
      ca.wrap = D->fp32 ? (void*)D->wrap32 : (void*)D->wrap;
      ca.I_amb = I_amb;
      ca.ox = D->ox; ca.oy = D->oy; ca.oz = D->oz; ca.w = D->w; ca.Ig = D->Ig_out;
      ca.C = D->cl_C; ca.rows = D->cl_rows; ca.periodic = 1; ca.down_slots = oa.down_slots;
      ca.groups = D->groups;
      rc = launch_cl_sweep(D, ca, st);
      if (rc != FS_OK) return rc;
    } else if (D->mode == 7) {
      if (D->fp32) {
        StArgs<float> sa{};
        sa.kb = D->kb32; sa.Goct = D->Goct32; sa.Qoct = D->Qoct32; sa.wrap = D->wrap32;
        sa.I_amb = (float)I_amb;
        sa.ox = D->ox; sa.oy = D->oy; sa.oz = D->oz; sa.w = D->w; sa.Ig = D->Ig_out;
        sa.C = D->cl_C; sa.rows = D->cl_rows; sa.periodic = 1; sa.lg_ring = D->cl_lg_ring;
        sa.down_slots = oa.down_slots; sa.err = oa.err;
        rc = launch_st_sweep(D, sa, st);
      } else {
        StArgs<double> sa{};
        sa.kb = D->kb; sa.Goct = D->Goct; sa.Qoct = D->Qoct; sa.wrap = D->wrap;
        sa.I_amb = I_amb;
        sa.ox = D->ox; sa.oy = D->oy; sa.oz = D->oz; sa.w = D->w; sa.Ig = D->Ig_out;
        sa.C = D->cl_C; sa.rows = D->cl_rows; sa.periodic = 1; sa.lg_ring = D->cl_lg_ring;
        sa.down_slots = oa.down_slots; sa.err = oa.err;
        rc = launch_st_sweep(D, sa, st);
      }
      if (rc != FS_OK) return rc;
    } else if (D->fp32) {
      OctArgs32 o3{};
      o3.kb = D->kb32; o3.ox = D->ox; o3.oy = D->oy; o3.oz = D->oz; o3.w = D->w;
      o3.Ig = D->Ig_out; o3.Goct = D->Goct32; o3.Qoct = D->Qoct32; o3.wrap = D->wrap32;
      o3.I_amb = (float)I_amb; o3.C = D->cl_C; o3.rows = D->cl_rows; o3.periodic = 1;
      o3.down_slots = oa.down_slots;
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = D->cl_C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(8 * D->cl_C); cfg.blockDim = dim3(D->cl_threads);
      cfg.dynamicSmemBytes = D->cl_smem; cfg.stream = st; cfg.attrs = at; cfg.numAttrs = 1;
      cudaError_t e;
      switch (D->Mo) {
        case 3: e = cudaLaunchKernelEx(&cfg, k_dom_octant_f32<3>, g, o3); break;
        case 6: e = cudaLaunchKernelEx(&cfg, k_dom_octant_f32<6>, g, o3); break;
        case 10: e = cudaLaunchKernelEx(&cfg, k_dom_octant_f32<10>, g, o3); break;
        default: e = cudaErrorInvalidValue;
      }
      fs_count_launch();
      if (e != cudaSuccess) return FS_ECUDA;
    } else if (octp) {
      rc = launch_octant_sweep(D, oa, st);
      if (rc != FS_OK) return rc;
    } else if (D->mode == 5) {
      rc = launch_ord_sweep(D, I_amb, st);
      if (rc != FS_OK) return rc;
    } else if (D->mode == 2) {
      k_dom_sweep_block<<<M, 1024, smem, st>>>(g, a);
      fs_count_launch();
    } else {
      for (int d = 0; d < nplanes; ++d) {
        a.plane = d;
        k_dom_plane<<<blocks_for(nthr, 256), 256, 0, st>>>(g, a);
        fs_count_launch();
      }
    }
    if (D->timing) cudaEventRecord(D->ev1[it], st);
    cudaMemsetAsync(D->keys, 0, sizeof(unsigned long long) * 2, st);  // keys[2] keeps the wait flag
    unsigned nb = blocks_for(N, 256);
    if (nb > 1184) nb = 1184;
    if (D->fp32) {
      k_dom_G_oct32<<<nb, 256, 0, st>>>(N, 8 * D->groups, D->Goct32, D->G, D->Gp, D->keys);
      fs_count_launch();
      k_dom_ground_oct32<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, nslots, D->Qoct32,
                                                              D->Isoil, refl, D->relax,
                                                              D->Ig_out, D->qin);
      fs_count_launch();
    } else if (octp) {
      k_dom_G_oct<<<nb, 256, 0, st>>>(N, 8 * D->groups, D->Goct, D->G, D->Gp, D->keys);
      fs_count_launch();
      k_dom_ground_oct<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, nslots, D->Qoct, D->Isoil,
                                                            refl, D->relax, D->Ig_out, D->qin);
      fs_count_launch();
    } else {
      k_dom_G<<<nb, 256, 0, st>>>(N, M, D->w, D->I, D->G, D->Gp, D->keys);
      fs_count_launch();
      k_dom_ground<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, M, D->oz, D->w, D->I, N,
                                                        D->Isoil, refl, D->relax, D->Ig_out,
                                                        D->qin);
      fs_count_launch();
    }
    // the error checks run on every iteration (a single-iteration solve
    // included); the convergence test, as the reference's, from the second
    {
      cudaMemcpyAsync(D->h_keys, D->keys, sizeof(unsigned long long) * 3, cudaMemcpyDeviceToHost,
                      st);
      if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
      if ((int)D->h_keys[2] != 0) {
        fs_set_error("fs_dom_solve: pipelined sweep wait gave up (hand-off between CTAs stalled)");
        return FS_ETIMEOUT;
      }
      double Gmax = key_to_double(D->h_keys[0]);
      double dmax = key_to_double(D->h_keys[1]);
      if (Gmax != Gmax || dmax != dmax) return FS_ENONFINITE;
      if (Gmax < 1e-12) Gmax = 1e-12;
      if (it > 0 && dmax / Gmax < D->tol) { ++it; break; }
    }
  }
  D->last_iters = it;
  if (D->timing) {
    cudaEventSynchronize(D->ev1[it - 1]);
    for (int q = 0; q < it; ++q) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, D->ev0[q], D->ev1[q]);
      D->sweep_ms += ms;
      D->sweep_count += 1;
    }
  }
  k_dom_finish<<<blocks_for(N, 256), 256, 0, st>>>(g, D->ks, D->kg, D->ksafe, D->B, D->G, q_solid,
                                                   q_gas);
  fs_count_launch();
  if (q_in_soil) {
    k_scale2<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, D->qin, D->eps_w, q_in_soil);
    fs_count_launch();
  }
  return cuda_status();
}
