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
//   8 (default for quadratures grouped by octant) octant clusters: one
//     thread-block cluster per octant (or per half of an octant's ordinates),
//     the cluster's CTAs split the k' rows and every thread owns one or two
//     pencils (j',k') and advances all the group's ordinates of its cell on
//     each hyperplane, reading the previous hyperplane from shared memory.
//     The CTAs form a pipeline, not a lock-step: each stores its last row of
//     every hyperplane into a ring in the next CTA's shared memory
//     (distributed shared memory) and signals the slot's "full" mbarrier; the
//     next CTA's helper warp waits for it, and after the hyperplane that
//     read it signals the slot's "empty" mbarrier back, so a CTA waits only
//     for its neighbours, and only when it runs ahead of them by more than
//     the ring's slack.  Within a CTA one __syncthreads per hyperplane.  All
//     waits are bounded (an error flag, then FS_ETIMEOUT on the host).  Inputs
//     arrive by cp.async a few hyperplanes ahead; the sweep emits the
//     octant's partial G and ground flux and never stores intensities.  The
//     cluster shape is planned so that all clusters are resident at once
//     where the part allows it.
//   3 (any quadrature) one launch per hyperplane over all ordinates, with the
//     full intensity field stored; G summed over ordinates in ordinate order.
// Path 8 sums G within each octant in ordinate order and then over octants in
// octant order (the reference sums all ordinates in one sequence; the two
// orders differ only by rounding).
#include <vector>
#include <cstring>
#include <utility>
#include <type_traits>
#include <cooperative_groups.h>
#include "common.cuh"
#include "kernels.h"

#define PI_D 3.141592653589793
#define SIGMA_SB_D 5.67e-8

namespace cg = cooperative_groups;

struct DomCtx {
  GridDev g;
  int M;
  double *ox, *oy, *oz, *w;  // device ordinates and weights
  std::vector<double> hox, hoy, hoz, hw;
  double* I;                  // M * N full intensities (path 3 only)
  int mode;                   // resolved path: 0 not yet, 3 or 8
  int mode_req, force_C;      // requested path (0 auto) and cluster size (0 auto)
  int groups;                 // ordinate groups per octant (clusters per octant)
  int force_groups;           // requested groups (0 automatic)
  int withhold_plane;         // test switch: hyperplane whose ring fill is withheld (-1 none)
  int fp32;                   // single-precision sweep (path 8)
  // path 8 buffers (FP64 or FP32, by fp32): (kappa, kappa*B) per cell, octant
  // partial G (8*groups x N), octant partial ground flux (8*groups x Ny*Nx),
  // y-periodic inflow rows (M x Nz x Nx)
  void *kb, *Goct, *Qoct, *wrap;
  int Mo, cl_C, cl_rows, cl_threads, cl_ppt, cl_waves;
  size_t cl_smem;
  int sweep_kernel;           // requested path-8 kernel: 0/1 pencil per thread, 2 lane column
  int cl_lane;                // resolved: 1 = the lane-column kernel
  int begun;                  // dom_begin done, dom_end due
  double pend_I_amb;          // ambient intensity of the begun solve
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

// ---- device helpers ----------------------------------------------------------
// L2 eviction-priority hint: (kappa, kappa*B) is re-read by every ordinate
// group of a sweep and should stay in L2.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
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
// streaming stores of the octant partials (read once, by the G reduction)
__device__ __forceinline__ void st_cs(double* p, double v) {
  asm volatile("st.global.cs.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
// two adjacent values in one 16-byte (8-byte for FP32) streaming store
__device__ __forceinline__ void st_cs2(double* p, double lo, double hi) {
  asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(lo), "d"(hi) : "memory");
}
__device__ __forceinline__ void st_cs2(float* p, float lo, float hi) {
  asm volatile("st.global.cs.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(lo), "f"(hi) : "memory");
}
__device__ __forceinline__ void st_cs(float* p, float v) {
  asm volatile("st.global.cs.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void cluster_arrive_release() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ double clip01(double x) {
  if (x < 0.0) x = 0.0;
  if (x > 1.0) x = 1.0;
  return x;
}

// The cell update of one ordinate, I = (kappa*B + ax*Ix + ay*Iy + az*Iz) /
// (kappa + ax + ay + az) (dom_3d.py:147-211), with the numerator by fused
// multiply-adds and the constant part of the denominator, ax + ay + az,
// tabulated per ordinate and level.
// FP64: the quotient from the hardware's approximate reciprocal refined by
// one Newton-Raphson iteration (r <- r + r (1 - den r), which squares its
// relative error), then one Markstein correction of the quotient
// (q <- q + r (num - den q), Markstein 1990), whose error is the square of
// the reciprocal's plus the final rounding: within about one ulp of the
// correctly rounded quotient (den > 0 always: kappa >= 1e-3).  FP32 (mixed
// form): __fdividef (about 2 ulp).
__device__ __forceinline__ double rcp_approx(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}
__device__ __forceinline__ double sweep_quot(double num, double den) {
  const double r0 = rcp_approx(den);
  const double e = __fma_rn(-den, r0, 1.0);
  const double r1 = __fma_rn(r0, e, r0);
  const double q0 = num * r1;
  const double res = __fma_rn(-den, q0, num);
  return __fma_rn(r1, res, q0);
}
__device__ __forceinline__ float sweep_quot(float num, float den) { return __fdividef(num, den); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmat(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__host__ __device__ inline size_t up16(size_t x) { return (x + 15) & ~(size_t)15; }

template <typename T> struct Vec2Of;
template <> struct Vec2Of<double> { using type = double2; };
template <> struct Vec2Of<float> { using type = float2; };

// ---- set-up: absorption, emission, ground ------------------------------------
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

// ---- path 3: one launch per hyperplane, full intensities -----------------------
struct SweepArgs {
  const double *ox, *oy, *oz;
  double* I;
  const double *ksafe, *B, *Ig;
  double I_amb;
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

// ---- path 8: octant clusters ---------------------------------------------------
struct ClArgs {
  const void* kb;
  const double *ox, *oy, *oz, *w;
  const double* Ig;
  void *Goct, *Qoct, *wrap;
  double I_amb;
  int C, rows, periodic;
  int groups;  // clusters (ordinate groups of MO) per octant
  unsigned down_slots;  // 4 bits per octant: ground-flux slot, 15 = upward octant
  const int* done;  // device flag: nonzero = the source iteration has converged, do nothing
  int* err;         // device flag: set when a bounded hand-off wait gave up
  int withhold;     // test switch: the first CTA withholds its fill of this hyperplane (-1 none)
};
// Inputs (kappa, kappa*B, the ground intensity and the y-inflow of a row's
// first pencil) arrive this many hyperplanes ahead through cp.async commit
// groups.
#define CL_AHEAD 4
// Slots of the ring through which a CTA hands the last row of each
// hyperplane to the next CTA of the cluster: the upstream CTA runs up to
// CL_RING - 1 hyperplanes ahead of the downstream one (CL_RING - 2 in the
// lane-column kernel, which sends a row before the barrier that ends its
// hyperplane instead of after it).
#define CL_RING 3
// Threads per CTA (the helper warp included): one pencil per thread up to
// CL_MAX_THREADS_1 (80 registers a thread), else two pencils per thread up to
// CL_MAX_THREADS_2 (96 registers).
#define CL_MAX_THREADS_1 768
#define CL_MAX_THREADS_2 640
// bounded hand-off waits: try_wait rounds before a thread gives up
#define CL_WAIT_LIMIT (1 << 20)
// Shared memory of a CTA: the hyperplane buffers (current and previous,
// [pencil][ordinate]), the ring of the upstream CTA's last rows
// ([slot][pencil][ordinate]), the prefetched inputs and the per-ordinate
// tables.  A pencil's ordinates are contiguous and padded to an odd count
// (cl_mpad), so that the per-ordinate offsets of the cell update are
// immediates and a warp's 32 pencils fall in distinct shared-memory banks.  A pencil's own slot holds the ambient intensity until its first
// cell; the z-inflow of the first row comes from the ring or, in the first
// CTA, from the ground (or the ambient intensity); the y-inflow of a row's
// first pencil is the value the previous sweep left at the other end of the
// row, prefetched from the y-wrap array.
struct ClLayout {
  size_t bars, kab, ig, yin, buf0, buf1, ring, kz, cxy, cwq, total;
};
__host__ __device__ constexpr int cl_mpad(int Mo) { return Mo | 1; }
__host__ __device__ inline ClLayout cl_layout(int tsize, int Mo, int rows, int ny, int nz) {
  ClLayout L;
  const size_t S = (size_t)rows * ny;
  const size_t Mp = (size_t)cl_mpad(Mo);
  size_t o = 0;
  L.bars = o; o = up16(o + 2 * CL_RING * sizeof(unsigned long long));
  L.kab = o; o = up16(o + (size_t)CL_AHEAD * S * 2 * tsize);
  L.ig = o; o = up16(o + (size_t)CL_AHEAD * ny * sizeof(double));
  L.yin = o; o = up16(o + (size_t)CL_AHEAD * rows * Mo * tsize);
  L.buf0 = o; o = up16(o + Mp * S * tsize);
  L.buf1 = o; o = up16(o + Mp * S * tsize);
  L.ring = o; o = up16(o + (size_t)CL_RING * Mp * ny * tsize);
  L.kz = o; o = up16(o + (size_t)nz * Mo * 2 * tsize);
  L.cxy = o; o = up16(o + (size_t)Mo * 2 * tsize);
  L.cwq = o; o = up16(o + (size_t)Mo * 2 * tsize);
  L.total = o;
  return L;
}

// mbarriers of the row hand-off (cluster scope)
__device__ __forceinline__ void cl_mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// this CTA's arrival on its own barrier, announcing the bytes the phase awaits
__device__ __forceinline__ void cl_arrive_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// the shared::cluster address of the same location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cl_mapa(uint32_t addr, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
// arrive on another CTA's mbarrier, releasing this thread's earlier writes
__device__ __forceinline__ void cl_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
// a value into another CTA's shared memory; its bytes count towards the
// transaction count of that CTA's mbarrier (no fence or arrival needed)
__device__ __forceinline__ void cl_st_async(uint32_t a, double v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(a),
               "d"(v), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void cl_st_async(uint32_t a, float v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];" ::"r"(a),
               "f"(v), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool cl_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity; a thread whose wait gave up
// records it in *err and from then on neither waits nor signals nor stores
// into the ring (so no barrier phase is re-armed before it completed, and no
// bytes arrive for a phase nobody announced); its neighbours' waits then give
// up in turn, every CTA reaches the final cluster barrier, and the host
// reports FS_ETIMEOUT (the sweep's results are not to be trusted).
__device__ __forceinline__ void cl_wait(uint32_t addr, uint32_t parity, bool& failed, int* err) {
  if (failed) return;
  for (int it = 0; it < CL_WAIT_LIMIT; ++it)
    if (cl_try_wait(addr, parity)) return;
  failed = true;
  if (err) atomicExch(err, 1);
}

// Shared-memory loads and stores of the sweep's hot loop by 32-bit address;
// volatile, so they stay in program order (a batch's loads before its stores).
template <typename T> __device__ __forceinline__ T sh_ld(uint32_t a);
template <> __device__ __forceinline__ double sh_ld<double>(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
  return v;
}
template <> __device__ __forceinline__ float sh_ld<float>(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
  return v;
}
template <typename T2> __device__ __forceinline__ T2 sh_ld2(uint32_t a);
template <> __device__ __forceinline__ double2 sh_ld2<double2>(uint32_t a) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
  return v;
}
template <> __device__ __forceinline__ float2 sh_ld2<float2>(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ void sh_st(uint32_t a, double v) {
  asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void sh_st(uint32_t a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

template <typename T, int MO, int PPT>
__global__ void __launch_bounds__(PPT == 1 ? CL_MAX_THREADS_1 : CL_MAX_THREADS_2, 1)
    k_dom_octant_cl(GridDev g, ClArgs a) {
  using T2 = typename Vec2Of<T>::type;
  // ordinates per batch of the cell update (the FP64 ten-ordinate groups in
  // two batches of five, to stay within the register budget)
  constexpr int CB = (sizeof(T) == 4 || MO <= 6) ? MO : (MO % 5 == 0 ? 5 : MO);
  constexpr int MP = cl_mpad(MO);  // a pencil's padded ordinate stride
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
  const int S = rows * ny;  // pencils per CTA; also the plane per ordinate
  const ClLayout L = cl_layout((int)sizeof(T), MO, rows, ny, nz);
  unsigned long long* full = (unsigned long long*)(shraw + L.bars);
  unsigned long long* empty = full + CL_RING;
  T2* kab_ring = (T2*)(shraw + L.kab);
  double* ig_ring = (double*)(shraw + L.ig);
  T* yin = (T*)(shraw + L.yin);
  T* buf0 = (T*)(shraw + L.buf0);
  T* buf1 = (T*)(shraw + L.buf1);
  T* ring = (T*)(shraw + L.ring);
  T2* kz = (T2*)(shraw + L.kz);
  T2* cxy = (T2*)(shraw + L.cxy);
  T2* cwq = (T2*)(shraw + L.cwq);
  const T2* kb = (const T2*)a.kb;
  T* Goct = (T*)a.Goct;
  T* Qoct = (T*)a.Qoct;
  T* wrap = (T*)a.wrap;
  const T I_amb = (T)a.I_amb;
  const int nplanes = nx + ny + nz - 2;
  // the last warp is the helper: the hand-off signals only
  const int TT = (int)blockDim.x - 32;
  const bool helper = (int)threadIdx.x >= TT;
  const int hl = (int)threadIdx.x - TT;
  // per level and ordinate: (az, ax + ay + az); per ordinate (ax, ay) and
  // (weight, weight * |mu|)
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int k = t / MO, m = t - k * MO;
    const double ax = fabs(a.ox[n0 + m]) / g.dx, ay = fabs(a.oy[n0 + m]) / g.dy;
    const double az = fabs(a.oz[n0 + m]) / g.dz[k];
    T2 v;
    v.x = (T)az;
    v.y = (T)(ax + ay + az);
    kz[t] = v;
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    T2 xy, wq;
    xy.x = (T)(fabs(a.ox[n0 + m]) / g.dx);
    xy.y = (T)(fabs(a.oy[n0 + m]) / g.dy);
    wq.x = (T)a.w[n0 + m];
    wq.y = (T)(a.w[n0 + m] * fabs(a.oz[n0 + m]));
    cxy[m] = xy;
    cwq[m] = wq;
  }
  for (int t = threadIdx.x; t < MP * S; t += blockDim.x) {
    buf0[t] = I_amb;
    buf1[t] = I_amb;
  }
  for (int t = threadIdx.x; t < CL_RING * MP * ny; t += blockDim.x) ring[t] = I_amb;
  // a full slot: the ring slot's bytes (ny pencils x MO ordinates) have
  // arrived from the upstream CTA and this CTA's helper has announced them; an
  // empty slot: the helper of the downstream CTA has seen the hyperplane that
  // read it complete
  const uint32_t fill_bytes = (uint32_t)(ny * MO * sizeof(T));
  if (threadIdx.x == 0) {
    for (int s = 0; s < CL_RING; ++s) {
      cl_mbar_init(&full[s], 1u);
      cl_mbar_init(&empty[s], 1u);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
  const uint64_t keep = l2_policy_evict_last();
  // per-pencil constants: pencil index, row and column, global row base, roles
  int pq[PPT], pjp[PPT], pkp[PPT], pk[PPT];
  int64_t prb[PPT];
  // 1 has, 2 first row, 4 first column (y-inflow), 8 last column (y-outflow),
  // 16 ground flux, 32 ground inflow
  unsigned prole[PPT];
#pragma unroll
  for (int pp = 0; pp < PPT; ++pp) {
    const int q = threadIdx.x + pp * TT;
    const bool has = !helper && q < npen;
    const int kl = has ? q / ny : 0;
    const int jp = has ? q - kl * ny : 0;
    const int kp = r0 + kl;
    const int k = fz ? kp : nz - 1 - kp;
    const int j = fy ? jp : ny - 1 - jp;
    pq[pp] = q; pjp[pp] = jp; pkp[pp] = kp; pk[pp] = k;
    prb[pp] = ((int64_t)k * ny + j) * nx;
    prole[pp] = (has ? 1u : 0u) | (has && kl == 0 ? 2u : 0u) | (has && jp == 0 ? 4u : 0u) |
                (has && jp == ny - 1 && periodic ? 8u : 0u) |
                (has && !fz && k == 0 && slot >= 0 ? 16u : 0u) | (has && fz && kp == 0 ? 32u : 0u);
  }
  auto prefetch = [&](int d) {
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int ip = d - pjp[pp] - pkp[pp];
      if ((prole[pp] & 1u) && ip >= 0 && ip < nx) {
        const int i = fx ? ip : nx - 1 - ip;
        const int sl = d % CL_AHEAD;
        cp_async_kb(&kab_ring[(size_t)sl * S + pq[pp]], &kb[prb[pp] + i], keep);
        if (prole[pp] & 32u) {
          const int j = fy ? pjp[pp] : ny - 1 - pjp[pp];
          cp_async8(&ig_ring[(size_t)sl * ny + pjp[pp]], &a.Ig[(int64_t)j * nx + i]);
        }
        if (prole[pp] & 4u) {
          // the y-inflow of this row's first pencil, ordinate by ordinate
          T* dst = yin + ((size_t)sl * rows + (pkp[pp] - r0)) * MO;
          const T* src = wrap0 + (int64_t)pk[pp] * nx + i;
#pragma unroll
          for (int m = 0; m < MO; ++m) {
            if (periodic)
              cp_async_val(&dst[m], src + m * wstride);
            else
              dst[m] = I_amb;
          }
        }
      }
    }
    cp_async_commit();
  };
  for (int d = 0; d < CL_AHEAD - 1; ++d) prefetch(d);
  __syncthreads();
  // the barriers' initialisation, the filled buffers and the first CL_RING
  // fills announced, cluster-wide
  if (helper && hl == 0 && rank > 0)
    for (int s = 0; s < CL_RING; ++s) cl_arrive_expect(smem_u32(&full[s]), fill_bytes);
  cluster_arrive_release();
  cluster_wait_acquire();
  // shared-memory addresses (32-bit) of the hot loop's arrays; the
  // downstream CTA's ring and full barriers, the upstream CTA's empty barriers
  constexpr uint32_t TS = (uint32_t)sizeof(T);
  constexpr uint32_t PS = (uint32_t)MP * TS;  // bytes per pencil
  const uint32_t a_buf0 = smem_u32(buf0), a_buf1 = smem_u32(buf1), a_ring = smem_u32(ring);
  const uint32_t a_yin = smem_u32(yin);
  const uint32_t a_kz = smem_u32(kz), a_cxy = smem_u32(cxy), a_cwq = smem_u32(cwq);
  const uint32_t a_dring = rank < C - 1 ? cl_mapa(a_ring, (unsigned)(rank + 1)) : 0u;
  const uint32_t full_dn = rank < C - 1 ? cl_mapa(smem_u32(full), (unsigned)(rank + 1)) : 0u;
  const uint32_t empty_up = rank > 0 ? cl_mapa(smem_u32(empty), (unsigned)(rank - 1)) : 0u;
  bool failed = false;
  // With an even nx a pencil's octant-partial G goes out in aligned pairs of
  // x-adjacent cells, which it visits on consecutive hyperplanes: the first
  // value of a pair waits in a register for the second (every pair
  // completes, the first and last cells included).
  const bool gpair = (nx & 1) == 0;
  T gpend[PPT];
#pragma unroll
  for (int pp = 0; pp < PPT; ++pp) gpend[pp] = (T)0;
  // The last row of hyperplane r (in the buffer at abuf) into the downstream
  // CTA's ring slot r % CL_RING, once the downstream CTA is done with what the
  // slot held: ny x MO values spread over all pencil threads, two or fewer
  // each, right after the barrier that completed hyperplane r, so that no warp
  // carries the hand-off alone.  The test switch withholds the first CTA's
  // fill of hyperplane a.withhold, so the next CTA's bounded wait runs out.
  auto push_row = [&](int r, uint32_t abuf) {
    if (rank >= C - 1 || (int)threadIdx.x >= ny * MO || (rank == 0 && r == a.withhold)) return;
    const int ps = r % CL_RING;
    if (r >= CL_RING)
      cl_wait(smem_u32(&empty[ps]), (uint32_t)((r / CL_RING - 1) & 1), failed, a.err);
    if (failed) return;
    const uint32_t src = abuf + (uint32_t)((rows - 1) * ny) * PS;
    const uint32_t dst = a_dring + (uint32_t)(ps * ny) * PS;
    const uint32_t bar = full_dn + 8u * ps;
    for (int idx = threadIdx.x; idx < ny * MO; idx += TT) {
      const int jq = idx / MO, m = idx - jq * MO;
      const uint32_t off = (uint32_t)jq * PS + (uint32_t)m * TS;
      cl_st_async(dst + off, sh_ld<T>(src + off), bar);
    }
  };
  for (int d = 0; d < nplanes; ++d) {
    prefetch(d + CL_AHEAD - 1);  // an empty group past the last plane
    cp_async_wait<CL_AHEAD - 1>();  // this plane's group has landed
    // the upstream CTA's last row of hyperplane d-1 is in the ring
    if (helper && hl == 0 && rank > 0 && d > 0)
      cl_wait(smem_u32(&full[(d - 1) % CL_RING]), (uint32_t)(((d - 1) / CL_RING) & 1), failed,
              a.err);
    __syncthreads();  // hyperplane d-1 complete in this CTA
    if (helper) {
      // the slot read on hyperplane d-1 awaits its next fill, and the
      // upstream CTA may write it
      // (after a wait that gave up, no barrier is touched again: a phase that
      // did not complete is never re-armed)
      if (hl == 0 && rank > 0 && d >= 2 && !failed) {
        cl_arrive_expect(smem_u32(&full[(d - 2) % CL_RING]), fill_bytes);
        cl_arrive_remote(empty_up + 8u * ((d - 2) % CL_RING));
      }
      continue;
    }
    const int sl = d % CL_AHEAD;
    const int zslot = (d + CL_RING - 1) % CL_RING;
    const uint32_t a_prev = (d & 1) ? a_buf0 : a_buf1;
    const uint32_t a_cur = (d & 1) ? a_buf1 : a_buf0;
    if (d > 0) push_row(d - 1, a_prev);
    T gsv[PPT], qsv[PPT];
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int jp = pjp[pp], kp = pkp[pp];
      const uint32_t qo = (uint32_t)pq[pp] * PS;
      const int ip = d - jp - kp;
      const bool act = (prole[pp] & 1u) && ip >= 0 && ip < nx;
      T gs = (T)0, qs = (T)0;
      if (act) {
        const uint32_t ap = a_prev + qo;  // Ix at ap + m*TS
        const uint32_t ac = a_cur + qo;
        // y-inflow: the pencil to the left, or the prefetched wrap values
        uint32_t ay = ap - PS;
        if (prole[pp] & 4u) ay = a_yin + (uint32_t)((sl * rows + (kp - r0)) * MO) * TS;
        // z-inflow: the row below in this CTA, else the ring; in the first
        // CTA the ground's (or the ambient) intensity, put in the ring slot
        uint32_t az = ap - (uint32_t)ny * PS;
        if (prole[pp] & 2u) {
          az = a_ring + (uint32_t)(zslot * ny + jp) * PS;
          if (rank == 0) {
            const T z = fz ? (T)ig_ring[(size_t)sl * ny + jp] : I_amb;
#pragma unroll
            for (int m = 0; m < MO; ++m) sh_st(az + (uint32_t)m * TS, z);
          } else {
            // this thread's own acquire of the slot the helper waited for
            cl_wait(smem_u32(&full[zslot]), (uint32_t)(((d - 1) / CL_RING) & 1), failed, a.err);
          }
        }
        const T2 kab = kab_ring[(size_t)sl * S + pq[pp]];
        const uint32_t akz = a_kz + (uint32_t)(pk[pp] * MO) * (2 * TS);
        // The cell update of the group's ordinates, in batches of CB: every
        // shared-memory load of a batch is issued before its stores, so the
        // batch's updates overlap instead of waiting on one another's stores.
        // Every per-ordinate offset is an immediate; only a pencil over the
        // ground sums the ground flux (one instance of the loop per role, so
        // neither has a branch inside).
        auto update = [&](auto ground_tag) {
          constexpr bool GROUND = decltype(ground_tag)::value;  // the ground-flux sum too
#pragma unroll
          for (int m0 = 0; m0 < MO; m0 += CB) {
            T Ix[CB], Iy[CB], Iz[CB], v[CB];
#pragma unroll
            for (int b = 0; b < CB; ++b) {
              const uint32_t mo = (uint32_t)(m0 + b) * TS;
              Ix[b] = sh_ld<T>(ap + mo);
              Iy[b] = sh_ld<T>(ay + mo);
              Iz[b] = sh_ld<T>(az + mo);
            }
#pragma unroll
            for (int b = 0; b < CB; ++b) {
              const uint32_t mo = (uint32_t)(m0 + b) * (2 * TS);
              const T2 zc = sh_ld2<T2>(akz + mo);
              const T2 xy = sh_ld2<T2>(a_cxy + mo);
              const T num = fmat(zc.x, Iz[b], fmat(xy.y, Iy[b], fmat(xy.x, Ix[b], kab.y)));
              v[b] = sweep_quot(num, kab.x + zc.y);
            }
#pragma unroll
            for (int b = 0; b < CB; ++b) {
              const T2 wq = sh_ld2<T2>(a_cwq + (uint32_t)(m0 + b) * (2 * TS));
              gs = fmat(wq.x, v[b], gs);
              if (GROUND) qs = fmat(wq.y, v[b], qs);
            }
#pragma unroll
            for (int b = 0; b < CB; ++b) {
              const uint32_t mo = (uint32_t)(m0 + b) * TS;
              sh_st(ac + mo, v[b]);
            }
          }
        };
        if (prole[pp] & 16u)
          update(std::true_type{});
        else
          update(std::false_type{});
        if (prole[pp] & 8u) {
          // the y-outflow, read by the next sweep at the row's other end
          T* wo = wrap0 + (int64_t)pk[pp] * nx + (fx ? ip : nx - 1 - ip);
#pragma unroll
          for (int m = 0; m < MO; ++m) wo[m * wstride] = sh_ld<T>(ac + (uint32_t)m * TS);
        }
      } else {
        if ((prole[pp] & 1u) && ip == -1) {
          // the hyperplane before a pencil's first cell: its x-inflow there
          // is the ambient intensity
          const uint32_t ac = a_cur + qo;
#pragma unroll
          for (int m = 0; m < MO; ++m) sh_st(ac + (uint32_t)m * TS, I_amb);
        }
      }
      gsv[pp] = gs;
      qsv[pp] = qs;
    }
#pragma unroll
    for (int pp = 0; pp < PPT; ++pp) {
      const int ip = d - pjp[pp] - pkp[pp];
      if ((prole[pp] & 1u) && ip >= 0 && ip < nx) {
        const int i = fx ? ip : nx - 1 - ip;
        if (!gpair) {
          st_cs(Go + prb[pp] + i, gsv[pp]);
        } else if (((i & 1) == 0) == fx) {
          gpend[pp] = gsv[pp];  // first of its pair in visiting order
        } else if (fx) {
          st_cs2(Go + prb[pp] + (i - 1), gpend[pp], gsv[pp]);
        } else {
          st_cs2(Go + prb[pp] + i, gsv[pp], gpend[pp]);
        }
        if (prole[pp] & 16u) {
          const int j = fy ? pjp[pp] : ny - 1 - pjp[pp];
          Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qsv[pp];
        }
      }
    }
  }
  __syncthreads();  // the last hyperplane complete in this CTA
  if (!helper) push_row(nplanes - 1, ((nplanes - 1) & 1) ? a_buf1 : a_buf0);
  cp_async_wait<0>();
  // the last hyperplane's fill (read by no one) has landed too: no store of
  // the upstream CTA is in flight to this CTA when it leaves
  if (helper && hl == 0 && rank > 0)
    cl_wait(smem_u32(&full[(nplanes - 1) % CL_RING]), (uint32_t)(((nplanes - 1) / CL_RING) & 1),
            failed, a.err);
  // no CTA leaves while another may still signal its barriers
  cluster_arrive_release();
  cluster_wait_acquire();
}

// ---- path 8, lane-column form ------------------------------------------------
// The same sweep (cluster per octant, CTAs splitting the k' rows, the ring
// hand-off between CTAs, the same inputs, outputs and arithmetic, so the same
// results bit for bit) with another mapping of pencils to threads: lane jp of
// the CTA owns the pencils (jp, kp) of all of the CTA's rows and keeps their
// latest intensities (rows x ordinates) in registers.  Within a hyperplane all
// cells are independent; a cell's x-inflow is its own pencil's latest value,
// its z-inflow the latest value of the pencil below (same lane; the first row
// takes the ring or the ground), its y-inflow the latest value of the pencil
// to the left: the lane below by a warp shuffle, for a warp's first lane the
// previous warp's last lane through a two-slot exchange buffer, for the first
// column the row's y-inflow.  A hyperplane costs one barrier over ny/32
// compute warps and the helper, and each lane has rows x ordinates
// independent updates per hyperplane, where the pencil-per-thread form moves
// every intensity through shared memory and waits at a barrier over 24 warps
// that each have ten.  Measured on the 400 x 120 x 60 S8 workload it is the
// slower of the two (3.85 ms per FP64 sweep, twice the other): with one warp per
// scheduler a lane's updates do not overlap enough to cover the latency of
// the reciprocal and its corrections, which the other form hides with six
// warps per scheduler.  It is built for comparison and chosen only on request.
#define LC_MAX_WARPS 4  // compute warps (ny <= 128)
struct LcLayout {
  size_t bars, kab, ig, yin, xb, ring, kz, cxy, cwq, total;
};
__host__ __device__ inline LcLayout lc_layout(int tsize, int Mo, int rows, int nw, int ny, int nz) {
  LcLayout L;
  const size_t NWL = (size_t)nw * 32;
  const size_t Mp = (size_t)cl_mpad(Mo);
  size_t o = 0;
  L.bars = o; o = up16(o + 2 * CL_RING * sizeof(unsigned long long));
  L.kab = o; o = up16(o + (size_t)CL_AHEAD * rows * NWL * 2 * tsize);
  L.ig = o; o = up16(o + (size_t)CL_AHEAD * NWL * sizeof(double));
  L.yin = o; o = up16(o + (size_t)CL_AHEAD * rows * Mo * tsize);
  L.xb = o; o = up16(o + (size_t)2 * nw * rows * Mo * tsize);
  L.ring = o; o = up16(o + (size_t)CL_RING * Mp * ny * tsize);
  L.kz = o; o = up16(o + (size_t)nz * Mo * 2 * tsize);
  L.cxy = o; o = up16(o + (size_t)Mo * 2 * tsize);
  L.cwq = o; o = up16(o + (size_t)Mo * 2 * tsize);
  L.total = o;
  return L;
}

template <typename T, int MO, int ROWS>
__global__ void __launch_bounds__(32 * (LC_MAX_WARPS + 1), 1)
    k_dom_octant_lc(GridDev g, ClArgs a) {
  using T2 = typename Vec2Of<T>::type;
  constexpr int MP = cl_mpad(MO);
  extern __shared__ __align__(16) unsigned char shraw[];
  if (a.done && *(volatile const int*)a.done) return;
  cg::cluster_group cl = cg::this_cluster();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int C = a.C;
  const int rank = (int)cl.block_rank();
  const int part = blockIdx.x / C;
  const int oct = part / a.groups;
  const int grp = part - oct * a.groups;
  const int n0 = part * MO;
  const int nw = (int)(blockDim.x >> 5) - 1;  // compute warps; the last warp is the helper
  const int NWL = nw * 32;
  const LcLayout L = lc_layout((int)sizeof(T), MO, ROWS, nw, ny, nz);
  unsigned long long* full = (unsigned long long*)(shraw + L.bars);
  unsigned long long* empty = full + CL_RING;
  T2* kab_ring = (T2*)(shraw + L.kab);
  double* ig_ring = (double*)(shraw + L.ig);
  T* yin = (T*)(shraw + L.yin);
  T* xb = (T*)(shraw + L.xb);
  T* ring = (T*)(shraw + L.ring);
  T2* kz = (T2*)(shraw + L.kz);
  T2* cxy = (T2*)(shraw + L.cxy);
  T2* cwq = (T2*)(shraw + L.cwq);
  const T2* kb = (const T2*)a.kb;
  T* Goct = (T*)a.Goct;
  T* Qoct = (T*)a.Qoct;
  T* wrap = (T*)a.wrap;
  const T I_amb = (T)a.I_amb;
  const int nplanes = nx + ny + nz - 2;
  const int lane = (int)threadIdx.x & 31, wid = (int)threadIdx.x >> 5;
  const bool helper = wid == nw;
  const int jp = (int)threadIdx.x;  // the lane's column (compute warps)
  const bool has = !helper && jp < ny;
  for (int t = threadIdx.x; t < MO * nz; t += blockDim.x) {
    const int k = t / MO, m = t - k * MO;
    const double ax = fabs(a.ox[n0 + m]) / g.dx, ay = fabs(a.oy[n0 + m]) / g.dy;
    const double az = fabs(a.oz[n0 + m]) / g.dz[k];
    T2 v;
    v.x = (T)az;
    v.y = (T)(ax + ay + az);
    kz[t] = v;
  }
  for (int m = threadIdx.x; m < MO; m += blockDim.x) {
    T2 xy, wq;
    xy.x = (T)(fabs(a.ox[n0 + m]) / g.dx);
    xy.y = (T)(fabs(a.oy[n0 + m]) / g.dy);
    wq.x = (T)a.w[n0 + m];
    wq.y = (T)(a.w[n0 + m] * fabs(a.oz[n0 + m]));
    cxy[m] = xy;
    cwq[m] = wq;
  }
  for (int t = threadIdx.x; t < 2 * nw * ROWS * MO; t += blockDim.x) xb[t] = I_amb;
  for (int t = threadIdx.x; t < CL_RING * MP * ny; t += blockDim.x) ring[t] = I_amb;
  const uint32_t fill_bytes = (uint32_t)(ny * MO * sizeof(T));
  if (threadIdx.x == 0) {
    for (int s = 0; s < CL_RING; ++s) {
      cl_mbar_init(&full[s], 1u);
      cl_mbar_init(&empty[s], 1u);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const bool fx = a.ox[n0] >= 0.0, fy = a.oy[n0] >= 0.0, fz = a.oz[n0] >= 0.0;
  const int r0 = rank * ROWS;
  const int64_t N = ncells_dev(g);
  const int64_t n2 = (int64_t)nx * ny;
  const int slot_bits = (int)((a.down_slots >> (4 * oct)) & 15u);
  const int slot = slot_bits == 15 ? -1 : slot_bits * a.groups + grp;
  T* Go = Goct + (int64_t)part * N;
  const int64_t wstride = (int64_t)nz * nx;
  T* wrap0 = wrap + (int64_t)n0 * wstride;
  const bool periodic = a.periodic != 0;
  const uint64_t keep = l2_policy_evict_last();
  const int j = fy ? jp : ny - 1 - jp;  // the column's y index (compute lanes with has)
  // the inputs of hyperplane d for the lane's cells: (kappa, kappa*B), the
  // ground intensity under the first row of the first CTA, the y-inflow of
  // the first column
  auto prefetch = [&](int d) {
    if (has) {
      const int sl = d % CL_AHEAD;
#pragma unroll
      for (int kl = 0; kl < ROWS; ++kl) {
        const int kp = r0 + kl;
        const int ip = d - jp - kp;
        if (kp < nz && ip >= 0 && ip < nx) {
          const int i = fx ? ip : nx - 1 - ip;
          const int k = fz ? kp : nz - 1 - kp;
          cp_async_kb(&kab_ring[(size_t)(sl * ROWS + kl) * NWL + jp],
                      &kb[((int64_t)k * ny + j) * nx + i], keep);
          if (fz && kp == 0) cp_async8(&ig_ring[(size_t)sl * NWL + jp], &a.Ig[(int64_t)j * nx + i]);
          if (jp == 0) {
            T* dst = yin + (size_t)(sl * ROWS + kl) * MO;
            const T* src = wrap0 + (int64_t)k * nx + i;
#pragma unroll
            for (int m = 0; m < MO; ++m) {
              if (periodic)
                cp_async_val(&dst[m], src + m * wstride);
              else
                dst[m] = I_amb;
            }
          }
        }
      }
    }
    cp_async_commit();
  };
  for (int d = 0; d < CL_AHEAD - 1; ++d) prefetch(d);
  __syncthreads();
  if (helper && lane == 0 && rank > 0)
    for (int s = 0; s < CL_RING; ++s) cl_arrive_expect(smem_u32(&full[s]), fill_bytes);
  cluster_arrive_release();
  cluster_wait_acquire();
  constexpr uint32_t TS = (uint32_t)sizeof(T);
  constexpr uint32_t PS = (uint32_t)MP * TS;
  const uint32_t a_ring = smem_u32(ring);
  const uint32_t a_dring = rank < C - 1 ? cl_mapa(a_ring, (unsigned)(rank + 1)) : 0u;
  const uint32_t full_dn = rank < C - 1 ? cl_mapa(smem_u32(full), (unsigned)(rank + 1)) : 0u;
  const uint32_t empty_up = rank > 0 ? cl_mapa(smem_u32(empty), (unsigned)(rank - 1)) : 0u;
  const bool pusher = has && rank < C - 1;  // the last row feeds the next CTA
  // the column of ring slots this lane reads and writes (idle lanes: column 0)
  const int jr = has ? jp : 0;
  bool failed = false;
  T st[ROWS][MO];
#pragma unroll
  for (int kl = 0; kl < ROWS; ++kl)
#pragma unroll
    for (int m = 0; m < MO; ++m) st[kl][m] = I_amb;
  for (int d = 0; d < nplanes; ++d) {
    prefetch(d + CL_AHEAD - 1);  // an empty group past the last plane
    cp_async_wait<CL_AHEAD - 1>();
    if (helper && lane == 0 && rank > 0 && d > 0)
      cl_wait(smem_u32(&full[(d - 1) % CL_RING]), (uint32_t)(((d - 1) / CL_RING) & 1), failed,
              a.err);
    __syncthreads();  // hyperplane d-1 complete in this CTA
    if (helper) {
      if (lane == 0 && rank > 0 && d >= 2 && !failed) {
        cl_arrive_expect(smem_u32(&full[(d - 2) % CL_RING]), fill_bytes);
        cl_arrive_remote(empty_up + 8u * ((d - 2) % CL_RING));
      }
      continue;
    }
    const int sl = d % CL_AHEAD;
    const int zslot = (d + CL_RING - 1) % CL_RING;
    const int pslot = d % CL_RING;
    const int par = d & 1;
    const bool hold = rank == 0 && d == a.withhold;
    // this thread's own acquire of the ring slot the first row reads
    if (rank > 0 && d > 0)
      cl_wait(smem_u32(&full[zslot]), (uint32_t)(((d - 1) / CL_RING) & 1), failed, a.err);
    // the downstream CTA has finished with the slot this hyperplane fills
    if (pusher && d >= CL_RING)
      cl_wait(smem_u32(&empty[pslot]), (uint32_t)((d / CL_RING - 1) & 1), failed, a.err);
    const bool push = pusher && !failed && !hold;
    const uint32_t apush = a_dring + (uint32_t)(pslot * ny + jr) * PS;
    const uint32_t pbar = full_dn + 8u * pslot;
    // rows from the top down: row kl's z-inflow is row kl-1's value of d-1
#pragma unroll
    for (int kl = ROWS - 1; kl >= 0; --kl) {
      const int kp = r0 + kl;
      const int ip = d - jp - kp;
      const bool act = has && kp < nz && ip >= 0 && ip < nx;
      const int k = kp < nz ? (fz ? kp : nz - 1 - kp) : 0;
      T Iy[MO], Iz[MO], v[MO];
#pragma unroll
      for (int m = 0; m < MO; ++m) Iy[m] = __shfl_up_sync(0xffffffffu, st[kl][m], 1);
      if (lane == 0) {
        const T* src = jp == 0 ? yin + (size_t)(sl * ROWS + kl) * MO
                               : xb + (size_t)(((par ^ 1) * nw + (wid - 1)) * ROWS + kl) * MO;
#pragma unroll
        for (int m = 0; m < MO; ++m) Iy[m] = src[m];
      }
      if (kl > 0) {
#pragma unroll
        for (int m = 0; m < MO; ++m) Iz[m] = st[kl > 0 ? kl - 1 : 0][m];
      } else if (rank == 0) {
        const T z = fz ? (T)ig_ring[(size_t)sl * NWL + jp] : I_amb;
#pragma unroll
        for (int m = 0; m < MO; ++m) Iz[m] = z;
      } else {
        const T* zr = ring + (size_t)(zslot * ny + jr) * MP;
#pragma unroll
        for (int m = 0; m < MO; ++m) Iz[m] = zr[m];
      }
      const T2 kab = kab_ring[(size_t)(sl * ROWS + kl) * NWL + jp];
      const T2* kzr = kz + k * MO;
#pragma unroll
      for (int m = 0; m < MO; ++m) {
        const T2 zc = kzr[m];
        const T2 xy = cxy[m];
        const T num = fmat(zc.x, Iz[m], fmat(xy.y, Iy[m], fmat(xy.x, st[kl][m], kab.y)));
        v[m] = sweep_quot(num, kab.x + zc.y);
      }
      T gs = (T)0;
#pragma unroll
      for (int m = 0; m < MO; ++m) gs = fmat(cwq[m].x, v[m], gs);
#pragma unroll
      for (int m = 0; m < MO; ++m) st[kl][m] = act ? v[m] : st[kl][m];
      if (kl == ROWS - 1 && push) {
#pragma unroll
        for (int m = 0; m < MO; ++m) cl_st_async(apush + (uint32_t)m * TS, act ? v[m] : I_amb, pbar);
      }
      if (lane == 31 && wid < nw - 1) {
        T* xo = xb + (size_t)((par * nw + wid) * ROWS + kl) * MO;
#pragma unroll
        for (int m = 0; m < MO; ++m) xo[m] = st[kl][m];
      }
      if (act) {
        const int i = fx ? ip : nx - 1 - ip;
        st_cs(Go + ((int64_t)k * ny + j) * nx + i, gs);
        if (!fz && k == 0 && slot >= 0) {
          T qs = (T)0;
#pragma unroll
          for (int m = 0; m < MO; ++m) qs = fmat(cwq[m].y, v[m], qs);
          Qoct[(int64_t)slot * n2 + (int64_t)j * nx + i] = qs;
        }
        if (jp == ny - 1 && periodic) {
          // the y-outflow, read by the next sweep at the row's other end
          T* wo = wrap0 + (int64_t)k * nx + i;
#pragma unroll
          for (int m = 0; m < MO; ++m) wo[m * wstride] = v[m];
        }
      }
    }
  }
  cp_async_wait<0>();
  if (helper && lane == 0 && rank > 0)
    cl_wait(smem_u32(&full[(nplanes - 1) % CL_RING]), (uint32_t)(((nplanes - 1) / CL_RING) & 1),
            failed, a.err);
  cluster_arrive_release();
  cluster_wait_acquire();
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

// The lane-column kernels built: ten ordinates per cluster (the S8 octant),
// 4 to 8 k' rows per CTA.
static const void* octant_lc_ptr(bool fp32, int Mo, int rows) {
#define LCP(T, R) (const void*)k_dom_octant_lc<T, 10, R>
  if (Mo != 10) return nullptr;
  switch (rows) {
    case 4: return fp32 ? LCP(float, 4) : LCP(double, 4);
    case 5: return fp32 ? LCP(float, 5) : LCP(double, 5);
    case 6: return fp32 ? LCP(float, 6) : LCP(double, 6);
    case 7: return fp32 ? LCP(float, 7) : LCP(double, 7);
    case 8: return fp32 ? LCP(float, 8) : LCP(double, 8);
  }
#undef LCP
  return nullptr;
}

// G (FP64) = sum over the octant partials (octant order, FP64 or FP32
// partials); max G and max |G - G_prev|
template <typename T>
__global__ void k_dom_G_oct(int64_t N, int nparts, const T* __restrict__ Goct, double* G,
                            const double* __restrict__ Gp, unsigned long long* keys,
                            const int* done) {
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

// q_in at the ground from the downward octants' partial fluxes; ground
// intensity relaxation
template <typename T>
__global__ void k_dom_ground_oct(int n2, int nslots, const T* __restrict__ Qoct,
                                 const double* __restrict__ Isoil, double refl, double relax,
                                 double* Ig, double* qin, const int* done) {
  if (done && *done) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n2) return;
  double s = 0.0;
  for (int o = 0; o < nslots; ++o) s += (double)Qoct[(int64_t)o * n2 + q];
  qin[q] = s;
  double Inew = Isoil[q] + refl * s;
  Ig[q] = relax * Inew + (1.0 - relax) * Ig[q];
}

template <typename A, typename B>
__global__ void k_convert(int64_t n, const A* __restrict__ a, B* b) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) b[t] = (B)a[t];
}

// wrap rows from a full intensity field: wrap[n][k][i] = I[n][k][j_far][i]
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

// ---- host side ---------------------------------------------------------------
void* dom_create(const GridDev& g, int M, const double* ox, const double* oy, const double* oz,
                 const double* w, double kgmax) {
  DomCtx* D = new DomCtx();
  D->g = g;
  D->M = M;
  D->hox.assign(ox, ox + M); D->hoy.assign(oy, oy + M); D->hoz.assign(oz, oz + M);
  D->hw.assign(w, w + M);
  int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  SetupStream ss;
  cudaMalloc(&D->ox, sizeof(double) * M); cudaMalloc(&D->oy, sizeof(double) * M);
  cudaMalloc(&D->oz, sizeof(double) * M); cudaMalloc(&D->w, sizeof(double) * M);
  cudaMemcpyAsync(D->ox, ox, sizeof(double) * M, cudaMemcpyHostToDevice, ss.s);
  cudaMemcpyAsync(D->oy, oy, sizeof(double) * M, cudaMemcpyHostToDevice, ss.s);
  cudaMemcpyAsync(D->oz, oz, sizeof(double) * M, cudaMemcpyHostToDevice, ss.s);
  cudaMemcpyAsync(D->w, w, sizeof(double) * M, cudaMemcpyHostToDevice, ss.s);
  D->I = nullptr; D->kb = nullptr; D->Goct = nullptr; D->Qoct = nullptr; D->wrap = nullptr;
  D->mode = 0; D->mode_req = 0; D->force_C = 0; D->groups = 1; D->force_groups = 0;
  D->withhold_plane = -1;
  D->fp32 = 0; D->cl_ppt = 1; D->cl_waves = 0; D->begun = 0; D->pend_I_amb = 0.0;
  D->sweep_kernel = 0; D->cl_lane = 0;
  cudaMalloc(&D->G, sizeof(double) * N); cudaMalloc(&D->Gp, sizeof(double) * N);
  cudaMemsetAsync(D->G, 0, sizeof(double) * N, ss.s);
  cudaMemsetAsync(D->Gp, 0, sizeof(double) * N, ss.s);
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
  // the copies and the clearing above are complete before any solve is queued
  if (!ss.sync() || cudaGetLastError() != cudaSuccess) {
    dom_destroy(D);
    return nullptr;
  }
  return D;
}

void dom_destroy(void* h) {
  DomCtx* D = (DomCtx*)h;
  if (!D) return;
  cudaFree(D->ox); cudaFree(D->oy); cudaFree(D->oz); cudaFree(D->w); cudaFree(D->I);
  cudaFree(D->kb); cudaFree(D->Goct); cudaFree(D->Qoct); cudaFree(D->wrap);
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

// Octant grouping required by path 8: M = 8*Mo, ordinates octant-major, every
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

// Launch shape of path 8: ordinate groups per octant (1, or 2 when the
// octant's ordinates split evenly), cluster size C (k' rows per CTA), pencils
// per thread (1 or 2), one CTA per SM.  The configuration with the fewest
// waves of resident clusters times work per CTA per hyperplane (pencils x
// ordinates) wins; on a tie the one with fewer waves.  One cluster per octant
// is kept whenever all eight clusters are resident at once: two clusters per
// octant take more SMs for about the same sweep time, and the SMs left free
// are the ones the concurrent projection and k-epsilon run on (measured: 23.4
// against 22.8 ms per step).  force_C / D->force_groups pin C / the grouping
// (0: free).
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
  int best_waves = 1 << 30;
  bool found = false;
  for (int groups = 1; groups <= 2; ++groups) {
    if (force_groups > 0 && groups != force_groups) continue;
    if (MoAll % groups != 0) continue;
    if (found && best_waves == 1 && force_groups == 0) break;  // one cluster per octant, all resident
    const int Mo = MoAll / groups;
    for (int C = 16; C >= 1; --C) {
      if (force_C > 0 && C != force_C) continue;
      const int rows = (g.nz + C - 1) / C;
      if ((g.nz + rows - 1) / rows != C) continue;
      const int pencils = rows * g.ny;
      // pencil threads in whole warps, then the helper warp
      const int t1 = (pencils + 31) / 32 * 32 + 32;
      const int t2 = ((pencils + 1) / 2 + 31) / 32 * 32 + 32;
      const int ppt = t1 <= CL_MAX_THREADS_1 ? 1 : (t2 <= CL_MAX_THREADS_2 ? 2 : 0);
      if (ppt == 0) continue;
      const int threads = ppt == 1 ? t1 : t2;
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
      if (cost < best || (cost == best && waves < best_waves)) {
        best = cost; best_waves = waves; found = true;
        D->cl_C = C; D->cl_rows = rows; D->cl_threads = threads; D->cl_smem = smem;
        D->cl_ppt = ppt; D->groups = groups; D->cl_waves = waves;
      }
    }
  }
  return found;
}

// The first call (at the first solve or intensity access) picks the sweep path,
// allocates its buffers and clears the y-inflow rows on the caller's stream,
// so the clearing is ordered before that stream's first sweep (a plain
// cudaMemset runs on the legacy default stream, which does not order work on
// streams created non-blocking, such as torch's side streams).
// The lane-column kernel for the planned shape (same clusters, rows and
// ordinate groups), when it is requested, built for the shape, and all
// clusters stay resident at once as with the pencil-per-thread kernel.
static bool plan_lc(DomCtx* D) {
  const GridDev& g = D->g;
  const int Mo = D->M / 8 / D->groups;
  const int nw = (g.ny + 31) / 32;
  const void* fn = octant_lc_ptr(D->fp32 != 0, Mo, D->cl_rows);
  if (!fn || nw > LC_MAX_WARPS || D->cl_rows * D->cl_C < g.nz) return false;
  int dev = 0, optin = 0, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  const int tsize = D->fp32 ? (int)sizeof(float) : (int)sizeof(double);
  const size_t need = lc_layout(tsize, Mo, D->cl_rows, nw, g.ny, g.nz).total;
  const size_t pad = (size_t)smem_sm / 2 + 1024;  // no two CTAs on one SM
  const size_t smem = need > pad ? need : pad;
  if (smem > (size_t)optin) return false;
  cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  const int threads = 32 * (nw + 1);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = D->cl_C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(8 * D->groups * D->cl_C); cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem; cfg.attrs = at; cfg.numAttrs = 1;
  int active = 0;
  if (cudaOccupancyMaxActiveClusters(&active, fn, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (active < 1 || (8 * D->groups + active - 1) / active > D->cl_waves) return false;
  D->cl_lane = 1;
  D->cl_threads = threads;
  D->cl_smem = smem;
  return true;
}

static int dom_prepare(DomCtx* D, cudaStream_t st) {
  if (D->mode != 0) return FS_OK;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const int want = D->mode_req;
  const bool oct = (want == 0 || want == 8) && octant_grouping(D) && plan_cl(D, D->force_C);
  if (oct && D->sweep_kernel == 2 && !plan_lc(D)) {
    fs_set_error("the lane-column sweep kernel is not built for this shape (ten ordinates per "
                 "cluster, 4 to 8 k' rows per CTA, ny <= %d)", 32 * LC_MAX_WARPS);
    return FS_EARG;
  }
  if (oct) {
    D->mode = 8;
    D->Mo = D->M / 8;
    int slot = 0;
    for (int o = 0; o < 8; ++o) D->down_slot[o] = D->hoz[o * D->Mo] < 0.0 ? slot++ : -1;
    const size_t ts = D->fp32 ? sizeof(float) : sizeof(double);
    cudaMalloc(&D->kb, 2 * ts * N);
    cudaMalloc(&D->Goct, ts * 8 * D->groups * N);
    cudaMalloc(&D->Qoct, ts * 8 * D->groups * n2);
    cudaMalloc(&D->wrap, ts * D->M * g.nz * g.nx);
    cudaMemsetAsync(D->wrap, 0, ts * D->M * g.nz * g.nx, st);
    return cuda_status();
  }
  if (D->fp32) {
    fs_set_error("the single-precision sweep needs octant-grouped ordinates and a cluster "
                 "shape that fits this grid (path 8)");
    return FS_EARG;
  }
  if (want == 8) {
    fs_set_error("octant-cluster sweep not possible for this grid or quadrature");
    return FS_EARG;
  }
  D->mode = 3;
  cudaMalloc(&D->I, sizeof(double) * N * D->M);
  cudaMemsetAsync(D->I, 0, sizeof(double) * N * D->M, st);
  return cuda_status();
}

int dom_set_mode(void* h, int mode, int cluster_ctas) {
  DomCtx* D = (DomCtx*)h;
  if ((mode != 0 && mode != 3 && mode != 8) || cluster_ctas < 0 || cluster_ctas > 16) {
    fs_set_error("sweep mode %d / cluster size %d: the paths are 0 (automatic), 3 (one launch "
                 "per hyperplane) and 8 (octant clusters of at most 16 CTAs)", mode, cluster_ctas);
    return FS_EARG;
  }
  if (D->mode != 0) {
    fs_set_error("sweep mode must be set before the first solve or intensity load");
    return FS_EARG;
  }
  D->mode_req = mode;
  D->force_C = cluster_ctas;
  return FS_OK;
}

int dom_set_sweep_kernel(void* h, int kernel) {
  DomCtx* D = (DomCtx*)h;
  if (kernel < 0 || kernel > 2) {
    fs_set_error("sweep kernel %d: 0 (automatic), 1 (pencil per thread), 2 (lane column)", kernel);
    return FS_EARG;
  }
  if (D->mode != 0) {
    fs_set_error("the sweep kernel must be set before the first solve or intensity load");
    return FS_EARG;
  }
  D->sweep_kernel = kernel;
  return FS_OK;
}
int dom_sweep_kernel(void* h) {
  const DomCtx* D = (const DomCtx*)h;
  return D->mode != 8 ? 0 : (D->cl_lane ? 2 : 1);
}

int dom_mode(void* h) { return ((DomCtx*)h)->mode; }
int dom_set_wait_test(void* h, int plane) {
  ((DomCtx*)h)->withhold_plane = plane < 0 ? -1 : plane;
  return FS_OK;
}
int dom_launch_shape(void* h, int* out5) {
  const DomCtx* D = (const DomCtx*)h;
  if (D->mode != 8) {
    fs_set_error("fs_dom_launch_shape: path 8 is not in use (path %d)", D->mode);
    return FS_EARG;
  }
  out5[0] = D->cl_C;
  out5[1] = D->cl_rows;
  out5[2] = D->cl_threads;
  out5[3] = (int)D->cl_smem;
  out5[4] = D->groups;
  return FS_OK;
}

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
  const int64_t tot = (int64_t)D->M * g.nz * g.nx;
  if (D->mode == 8) {
    if (D->fp32)
      k_dom_extract_wrap<float><<<blocks_for(tot, 256), 256, 0, st>>>(g, D->M, D->oy, I_full,
                                                                     (float*)D->wrap);
    else
      k_dom_extract_wrap<double><<<blocks_for(tot, 256), 256, 0, st>>>(g, D->M, D->oy, I_full,
                                                                      (double*)D->wrap);
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
  if (D->mode == 8 && D->fp32) {
    k_convert<float, double><<<blocks_for(tot, 256), 256, 0, st>>>(tot, (const float*)D->wrap,
                                                                   dst);
    fs_count_launch();
  } else if (D->mode == 8) {
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
  if (D->mode == 8 && D->fp32) {
    k_convert<double, float><<<blocks_for(tot, 256), 256, 0, st>>>(tot, src, (float*)D->wrap);
    fs_count_launch();
  } else if (D->mode == 8) {
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
  if (D->cl_lane) {
#define LCL(T, R) e = cudaLaunchKernelEx(&cfg, k_dom_octant_lc<T, 10, R>, D->g, a)
    switch (D->cl_rows) {
      case 4: if (f) LCL(float, 4); else LCL(double, 4); break;
      case 5: if (f) LCL(float, 5); else LCL(double, 5); break;
      case 6: if (f) LCL(float, 6); else LCL(double, 6); break;
      case 7: if (f) LCL(float, 7); else LCL(double, 7); break;
      case 8: if (f) LCL(float, 8); else LCL(double, 8); break;
    }
#undef LCL
    fs_count_launch();
    return e == cudaSuccess ? FS_OK : FS_ECUDA;
  }
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

int dom_begin(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH,
              const double* rho, const double* Mloc, cudaStream_t st) {
  DomCtx* D = (DomCtx*)h;
  int rc = dom_prepare(D, st);
  if (rc != FS_OK) return rc;
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const double Tamb4 = pow(T_amb, 4.0);
  double2* kb = (D->mode == 8 && !D->fp32) ? (double2*)D->kb : nullptr;
  float2* kb32 = (D->mode == 8 && D->fp32) ? (float2*)D->kb : nullptr;
  k_dom_setup<<<blocks_for(N, 256), 256, 0, st>>>(g, Ts, Tg, as, om, YH, rho, Mloc, sigma, Tamb4,
                                                  D->kgmax, D->ks, D->kg, D->ksafe, D->B, kb,
                                                  kb32);
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

// End of queued source iteration q: the host loop's test on the device.
// st: [0] done, [1] iterations run, [2] error (2 non-finite G).  A non-finite
// G ends the solve on every iteration, the first included; the convergence
// ratio, as the reference's (dom_3d.py:450-460), from the second.
__global__ void k_dom_check(const unsigned long long* __restrict__ keys, double tol, int q,
                            int* st) {
  if (st[0]) return;
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
  const int nparts = 8 * D->groups;
  while (true) {
    for (int q = 0; q < batch && queued < D->max_iter; ++q, ++queued) {
      std::swap(D->G, D->Gp);
      if (D->timing) cudaEventRecord(D->ev0[queued], st);
      ClArgs ca = base;
      ca.done = D->dstate;
      ca.err = D->dstate + 3;
      int rc = launch_cl_sweep(D, ca, st);
      if (rc != FS_OK) return rc;
      if (D->timing) cudaEventRecord(D->ev1[queued], st);
      cudaMemsetAsync(D->keys, 0, sizeof(unsigned long long) * 2, st);
      if (D->fp32) {
        k_dom_G_oct<float><<<nb, 256, 0, st>>>(N, nparts, (const float*)D->Goct, D->G, D->Gp,
                                               D->keys, D->dstate);
        k_dom_ground_oct<float><<<blocks_for(n2, 128), 128, 0, st>>>(
            (int)n2, nslots, (const float*)D->Qoct, D->Isoil, refl, D->relax, D->Ig_out, D->qin,
            D->dstate);
      } else {
        k_dom_G_oct<double><<<nb, 256, 0, st>>>(N, nparts, (const double*)D->Goct, D->G, D->Gp,
                                                D->keys, D->dstate);
        k_dom_ground_oct<double><<<blocks_for(n2, 128), 128, 0, st>>>(
            (int)n2, nslots, (const double*)D->Qoct, D->Isoil, refl, D->relax, D->Ig_out, D->qin,
            D->dstate);
      }
      k_dom_check<<<1, 1, 0, st>>>(D->keys, D->tol, queued, D->dstate);
      fs_count_launch(); fs_count_launch(); fs_count_launch();
    }
    cudaMemcpyAsync(D->h_dstate, D->dstate, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
    if (D->h_dstate[3]) {
      fs_set_error("DOM sweep: a bounded wait for the row hand-off between the cluster's CTAs "
                   "gave up");
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

// Path 3's source iterations: the host reads G's maxima after every
// iteration (the non-finite check on every one, the convergence test from
// the second, as the reference's).
static int dom_iterate_planes(DomCtx* D, double refl, cudaStream_t st, int* iters_out) {
  const GridDev& g = D->g;
  const int64_t N = ncells(g), n2 = (int64_t)g.nx * g.ny;
  const int M = D->M;
  SweepArgs a{};
  a.ox = D->ox; a.oy = D->oy; a.oz = D->oz; a.I = D->I; a.ksafe = D->ksafe; a.B = D->B;
  a.Ig = D->Ig_out; a.I_amb = D->pend_I_amb; a.M = M; a.periodic = 1;
  const int nplanes = g.nx + g.ny + g.nz - 2;
  const int64_t nthr = (int64_t)g.ny * g.nz * M;
  unsigned nb = blocks_for(N, 256);
  if (nb > 1184) nb = 1184;
  int it = 0;
  for (it = 0; it < D->max_iter; ++it) {
    std::swap(D->G, D->Gp);
    if (D->timing) cudaEventRecord(D->ev0[it], st);
    for (int d = 0; d < nplanes; ++d) {
      a.plane = d;
      k_dom_plane<<<blocks_for(nthr, 256), 256, 0, st>>>(g, a);
      fs_count_launch();
    }
    if (D->timing) cudaEventRecord(D->ev1[it], st);
    cudaMemsetAsync(D->keys, 0, sizeof(unsigned long long) * 2, st);
    k_dom_G<<<nb, 256, 0, st>>>(N, M, D->w, D->I, D->G, D->Gp, D->keys);
    k_dom_ground<<<blocks_for(n2, 128), 128, 0, st>>>((int)n2, M, D->oz, D->w, D->I, N, D->Isoil,
                                                      refl, D->relax, D->Ig_out, D->qin);
    fs_count_launch(); fs_count_launch();
    cudaMemcpyAsync(D->h_keys, D->keys, sizeof(unsigned long long) * 2, cudaMemcpyDeviceToHost,
                    st);
    if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
    double Gmax = key_to_double(D->h_keys[0]);
    const double dmax = key_to_double(D->h_keys[1]);
    if (Gmax != Gmax || dmax != dmax) return FS_ENONFINITE;
    if (Gmax < 1e-12) Gmax = 1e-12;
    if (it > 0 && dmax / Gmax < D->tol) { ++it; break; }
  }
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
  const double refl = (1.0 - D->eps_w) / PI_D;
  int it = 0;
  if (D->mode == 8) {
    ClArgs ca{};
    ca.kb = D->kb; ca.Goct = D->Goct; ca.Qoct = D->Qoct; ca.wrap = D->wrap;
    ca.I_amb = D->pend_I_amb;
    ca.ox = D->ox; ca.oy = D->oy; ca.oz = D->oz; ca.w = D->w; ca.Ig = D->Ig_out;
    ca.C = D->cl_C; ca.rows = D->cl_rows; ca.periodic = 1; ca.groups = D->groups;
    ca.down_slots = 0;
    ca.withhold = D->withhold_plane;
    int nslots = 0;
    for (int o = 0; o < 8; ++o) {
      ca.down_slots |= (unsigned)(D->down_slot[o] >= 0 ? D->down_slot[o] : 15) << (4 * o);
      nslots += D->down_slot[o] >= 0 ? D->groups : 0;
    }
    rc = dom_iterate_dev(D, ca, nslots, refl, st, &it);
  } else {
    rc = dom_iterate_planes(D, refl, st, &it);
  }
  if (rc != FS_OK) return rc;
  D->last_iters = it;
  if (D->timing && it > 0) {
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
