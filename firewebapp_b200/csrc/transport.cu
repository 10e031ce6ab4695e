// Explicit transport stencils of the Tier-3 step (FP64, one thread per cell).
//
// Each kernel restates one reference operator; the comment above it names
// the reference function and lines.  All kernels are out-of-place (read the
// old field, write a new one), which is what the reference's double buffers
// (dY, du/dv/dw, k_turb_new, T_s_new) amount to.
#include <mutex>
#include "common.cuh"
#include "kernels.h"
#include "tma.cuh"

// ---------------------------------------------------------------------------
// Species transport, up to 3 species in one pass
// (species_3d.py:41-175 step_species_transport, called x3 at spread_3d.py:3015-3038)
// ---------------------------------------------------------------------------
struct SpeciesArgs {
  const double* Y[3];
  double* Yo[3];
  const double* S[3];
  double Y_inlet[3];
  int nspec;
  // fused form (fuel, O2, H2O in that order): the sources from S_pyro and
  // S_drying as k_species_sources forms them, and O2 clipped to [0, o2_cap]
  // after the update as k_clip does
  const double* Sp;
  const double* Sd;
  double o2_cap;
};

// One thread per cell; a block is a 32 (x) by 8 (y) tile of one z-level, so
// that the y-neighbours of the MUSCL and diffusion stencils (rows j-2..j+2)
// are mostly rows of the same block and come from L1 (6 % faster than blocks
// of 256 consecutive cells on the 400x120x60 grid, cold L2; with 3 blocks per
// SM and no spills it was 18 % slower: the kernel waits on loads, and the
// fourth block hides more of them).  The species loop is
// unrolled so the loads of all species are in flight together.  The level's
// reciprocals of the z spacings are computed once per block, and the
// divisions by the centred z spacing and by rho are multiplications by one
// reciprocal per cell, shared by the three species.
#define SP_TX 32
#define SP_TY 8
template <int NS, bool FUSED>
__global__ void __launch_bounds__(SP_TX * SP_TY, 4)
k_species(GridDev g, SpeciesArgs a, const double* __restrict__ rho,
          const double* __restrict__ u, const double* __restrict__ v,
          const double* __restrict__ w, double dt, double D, double inv_dx, double inv_dy,
          double inv_dx2, double inv_dy2) {
  __shared__ double rk[4];  // 1/da, 1/db, 1/dz, 1/hz of the block's level
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int k = blockIdx.z;
  const int tid = threadIdx.y * SP_TX + threadIdx.x;
  if (tid == 0) {
    const double da = g.da[k], db = g.db[k];
    rk[0] = 1.0 / da;
    rk[1] = 1.0 / db;
    rk[2] = 1.0 / g.dz[k];
    rk[3] = 1.0 / (0.5 * (da + db));
  }
  __syncthreads();
  const int i = blockIdx.x * SP_TX + threadIdx.x;
  const int j = blockIdx.y * SP_TY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int64_t crow = (int64_t)k * sz + i;
  const int64_t c = crow + (int64_t)j * sy;
  const int jm2 = wrapj(j - 2, ny), jm1 = wrapj(j - 1, ny);
  const int jp1 = wrapj(j + 1, ny), jp2 = wrapj(j + 2, ny);
  const double ui = u[c], vi = v[c], wi = w[c];
  const double inv_rho = 1.0 / rho[c];
  const double inv_d_above = rk[0], inv_d_below = rk[1], inv_dz_k = rk[2], inv_hz = rk[3];
  double sp = 0.0, sd = 0.0, stot = 0.0;
  if (FUSED) {
    sp = a.Sp[c];
    sd = a.Sd[c];
    stot = sp + sd;
  }
  const bool mx = (i >= 2 && i <= nx - 3);
  const bool mz = (k >= 2 && k <= nz - 3);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double* __restrict__ Y = a.Y[s];
    const double Yi = Y[c];
    const double YL_x = (i == 0) ? a.Y_inlet[s] : Y[c - 1];
    const double YR_x = (i == nx - 1) ? Yi : Y[c + 1];
    const double YL_z = (k == 0) ? Yi : Y[c - sz];
    const double YR_z = (k == nz - 1) ? Yi : Y[c + sz];
    double flux_x, flux_z;
    if (mx) {
      double fxp = muscl_face(Y[c - 1], Yi, Y[c + 1], Y[c + 2], ui);
      double fxm = muscl_face(Y[c - 2], Y[c - 1], Yi, Y[c + 1], ui);
      flux_x = ui * (fxp - fxm) * inv_dx;
    } else {
      flux_x = (ui >= 0.0) ? ui * (Yi - YL_x) * inv_dx : ui * (YR_x - Yi) * inv_dx;
    }
    const double Yjm2 = Y[crow + jm2 * sy], Yjm1 = Y[crow + jm1 * sy];
    const double Yjp1 = Y[crow + jp1 * sy], Yjp2 = Y[crow + jp2 * sy];
    double fyp = muscl_face(Yjm1, Yi, Yjp1, Yjp2, vi);
    double fym = muscl_face(Yjm2, Yjm1, Yi, Yjp1, vi);
    double flux_y = vi * (fyp - fym) * inv_dy;
    if (mz) {
      double fzp = muscl_face(Y[c - sz], Yi, Y[c + sz], Y[c + 2 * sz], wi);
      double fzm = muscl_face(Y[c - 2 * sz], Y[c - sz], Yi, Y[c + sz], wi);
      flux_z = wi * (fzp - fzm) * inv_hz;
    } else {
      flux_z = (wi >= 0.0) ? wi * (Yi - YL_z) * inv_d_below : wi * (YR_z - Yi) * inv_d_above;
    }
    double adv = -(flux_x + flux_y + flux_z);
    double d2x = (YR_x - 2.0 * Yi + YL_x) * inv_dx2;
    double d2y = (Yjp1 - 2.0 * Yi + Yjm1) * inv_dy2;
    double d2z = ((YR_z - Yi) * inv_d_above - (Yi - YL_z) * inv_d_below) * inv_dz_k;
    double diff = D * (d2x + d2y + d2z);
    double S;
    if (FUSED) S = (s == 0) ? sp - Yi * stot : ((s == 1) ? -(Yi * stot) : sd - Yi * stot);
    else S = a.S[s][c];
    double src = S * inv_rho;
    double dY = (adv + diff + src) * dt;
    double nw = Yi + dY;
    if (nw < 0.0) nw = 0.0;
    else if (nw > 1.0) nw = 1.0;
    if (FUSED && s == 1) {
      if (nw > a.o2_cap) nw = a.o2_cap;
      if (nw < 0.0) nw = 0.0;
    }
    a.Yo[s][c] = nw;
  }
}

int launch_species(const GridDev& g, int nspec, const double* const* Y, double* const* Yo,
                   const double* const* S, const double* Y_inlet, const double* rho,
                   const double* u, const double* v, const double* w, double dt, double D,
                   cudaStream_t st) {
  if (nspec < 1 || nspec > 3) return FS_EARG;
  SpeciesArgs a{};
  a.nspec = nspec;
  for (int s = 0; s < nspec; ++s) {
    a.Y[s] = Y[s]; a.Yo[s] = Yo[s]; a.S[s] = S[s]; a.Y_inlet[s] = Y_inlet[s];
  }
  double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  const dim3 nb((g.nx + SP_TX - 1) / SP_TX, (g.ny + SP_TY - 1) / SP_TY, g.nz);
  const dim3 tb(SP_TX, SP_TY);
  switch (nspec) {
    case 1: k_species<1, false><<<nb, tb, 0, st>>>(g, a, rho, u, v, w, dt, D, inv_dx, inv_dy,
                                                   inv_dx * inv_dx, inv_dy * inv_dy); break;
    case 2: k_species<2, false><<<nb, tb, 0, st>>>(g, a, rho, u, v, w, dt, D, inv_dx, inv_dy,
                                                   inv_dx * inv_dx, inv_dy * inv_dy); break;
    default: k_species<3, false><<<nb, tb, 0, st>>>(g, a, rho, u, v, w, dt, D, inv_dx, inv_dy,
                                                    inv_dx * inv_dx, inv_dy * inv_dy); break;
  }
  fs_count_launch();
  return cuda_status();
}

// The sub-step's species work in one pass: the sources with dilution
// (k_species_sources), the transport of fuel, O2 and H2O, and the O2 clip
// that follows it (spread_3d.py:2996-3004, 3015-3038, 3059); the results equal
// those three launches'.
struct SpeciesArgs;
static bool launch_species_step_tma(const GridDev& g, const SpeciesArgs& a, const double* rho,
                                    const double* u, const double* v, const double* w, double dt,
                                    double D, cudaStream_t st);

int launch_species_step(const GridDev& g, const double* const* Y, double* const* Yo,
                        const double* Sp, const double* Sd, const double* Y_inlet,
                        const double* rho, const double* u, const double* v, const double* w,
                        double dt, double D, double o2_cap, cudaStream_t st) {
  SpeciesArgs a{};
  a.nspec = 3;
  for (int s = 0; s < 3; ++s) {
    a.Y[s] = Y[s]; a.Yo[s] = Yo[s]; a.S[s] = nullptr; a.Y_inlet[s] = Y_inlet[s];
  }
  a.Sp = Sp;
  a.Sd = Sd;
  a.o2_cap = o2_cap;
  if (launch_species_step_tma(g, a, rho, u, v, w, dt, D, st)) return cuda_status();
  double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  const dim3 nb((g.nx + SP_TX - 1) / SP_TX, (g.ny + SP_TY - 1) / SP_TY, g.nz);
  const dim3 tb(SP_TX, SP_TY);
  k_species<3, true><<<nb, tb, 0, st>>>(g, a, rho, u, v, w, dt, D, inv_dx, inv_dy,
                                        inv_dx * inv_dx, inv_dy * inv_dy);
  fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// The fused species step with its stencil inputs staged by TMA.
//
// A block owns a 32 (x) by 8 (y) tile and marches up a chunk of z-levels.
// Each z-plane of the three mass fractions arrives as one TMA box of
// 36 x 12 doubles (the tile with the two-cell x and y halos the MUSCL faces
// read) in a ring of six shared-memory slots: the five planes k-2..k+2 the
// stencil reads and one in flight, so every value is fetched from L2/HBM once
// per block instead of once per neighbour.  Tiles whose halo crosses the
// periodic y boundary have those rows replaced by the wrapped rows after the
// box lands (TMA fills rows outside the tensor with zeros).  Cell-centred
// inputs (u, v, w, rho, the bed sources) are read directly.  The arithmetic
// is k_species<3, true>'s, expression for expression (same results).
// ---------------------------------------------------------------------------
#define TS_HX (SP_TX + 4)
#define TS_HY (SP_TY + 4)
#define TS_PLANE (TS_HX * TS_HY)
#define TS_SLOTS 6
#define TS_MAXKZ 64

struct SpeciesMaps {
  CUtensorMap Y[3];
};

__device__ int g_stencil_err;  // set when a bounded TMA wait gave up

__host__ __device__ inline size_t species_tma_smem() {
  return (size_t)TS_SLOTS * 3 * TS_PLANE * sizeof(double) + TS_SLOTS * sizeof(uint64_t) +
         4 * TS_MAXKZ * sizeof(double);
}

__global__ void __launch_bounds__(SP_TX * SP_TY, 3)
k_species_tma(GridDev g, SpeciesArgs a, const __grid_constant__ SpeciesMaps tm,
              const double* __restrict__ rho, const double* __restrict__ u,
              const double* __restrict__ v, const double* __restrict__ w, double dt, double D,
              double inv_dx, double inv_dy, double inv_dx2, double inv_dy2, int kz) {
  extern __shared__ __align__(128) unsigned char ts_raw[];
  double* ring = (double*)ts_raw;
  uint64_t* bars = (uint64_t*)(ts_raw + (size_t)TS_SLOTS * 3 * TS_PLANE * sizeof(double));
  double* rkz = (double*)(bars + TS_SLOTS);  // per level: 1/da, 1/db, 1/dz, 1/hz
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SP_TX + tx;
  const int i0 = blockIdx.x * SP_TX, j0 = blockIdx.y * SP_TY;
  const int k0 = blockIdx.z * kz;
  const int k1 = min(nz, k0 + kz);
  const int pfirst = k0 - 2, plast = k1 + 1;  // planes the chunk's stencil reads
  const bool ywrap = (j0 - 2 < 0) || (j0 + SP_TY + 2 > ny);
  if (tid == 0) {
    for (int q = 0; q < TS_SLOTS; ++q) tma_mbar_init(&bars[q], 1);
    tma_fence_init();
  }
  for (int q = tid; q < k1 - k0; q += SP_TX * SP_TY) {
    const int k = k0 + q;
    const double da = g.da[k], db = g.db[k];
    rkz[4 * q + 0] = 1.0 / da;
    rkz[4 * q + 1] = 1.0 / db;
    rkz[4 * q + 2] = 1.0 / g.dz[k];
    rkz[4 * q + 3] = 1.0 / (0.5 * (da + db));
  }
  __syncthreads();
  auto slot_of = [&](int p) { return (p - pfirst) % TS_SLOTS; };
  auto issue = [&](int p) {
    const int sl = slot_of(p);
    tma_arrive_expect(&bars[sl], 3 * TS_PLANE * sizeof(double));
#pragma unroll
    for (int s = 0; s < 3; ++s)
      tma_load_3d(ring + ((size_t)sl * 3 + s) * TS_PLANE, &tm.Y[s], i0 - 2, j0 - 2, p, &bars[sl]);
  };
  if (tid == 0) {
    tma_fence_proxy();
    for (int p = pfirst; p <= min(pfirst + TS_SLOTS - 1, plast); ++p) issue(p);
  }
  const int i = i0 + tx, j = j0 + ty;
  const bool inside = i < nx && j < ny;
  const int ii = tx + 2, jj = ty + 2;
  const int cix = jj * TS_HX + ii;
  // the cell-centred inputs of the next level are loaded while this level
  // computes (registers, one level ahead)
  double nu_ = 0.0, nv_ = 0.0, nw_ = 0.0, nr_ = 1.0, nsp = 0.0, nsd = 0.0;
  auto load_centre = [&](int k) {
    if (inside && k < k1) {
      const int64_t c = (int64_t)k * sz + (int64_t)j * sy + i;
      nu_ = u[c]; nv_ = v[c]; nw_ = w[c]; nr_ = rho[c]; nsp = a.Sp[c]; nsd = a.Sd[c];
    }
  };
  load_centre(k0);
  int waited = pfirst - 1;  // planes up to here have landed (and been patched)
  for (int k = k0; k < k1; ++k) {
    const double ui = nu_, vi = nv_, wi = nw_, rho_c = nr_, sp = nsp, sd = nsd;
    load_centre(k + 1);
    // the planes this level reads that have not been waited for yet
    const int need = min(k + 2, plast);
    for (int p = waited + 1; p <= need; ++p) {
      const int sl = slot_of(p);
      tma_wait(&bars[sl], (uint32_t)(((p - pfirst) / TS_SLOTS) & 1), &g_stencil_err);
      if (ywrap && p >= 0 && p < nz) {
        // rows of the box outside [0, ny) hold zeros: put the periodic rows there
        for (int e = tid; e < 3 * TS_PLANE; e += SP_TX * SP_TY) {
          const int s = e / TS_PLANE, r = (e % TS_PLANE) / TS_HX, col = e % TS_HX;
          const int jg = j0 - 2 + r, ig = i0 - 2 + col;
          if ((jg < 0 || jg >= ny) && ig >= 0 && ig < nx) {
            const double* Ys = s == 0 ? a.Y[0] : (s == 1 ? a.Y[1] : a.Y[2]);
            ring[((size_t)sl * 3 + s) * TS_PLANE + r * TS_HX + col] =
                Ys[(int64_t)p * sz + (int64_t)wrapj(jg, ny) * sy + ig];
          }
        }
      }
    }
    if (ywrap && need > waited) __syncthreads();
    waited = need > waited ? need : waited;
    if (inside) {
      const double* const pl0 = ring + (size_t)slot_of(k) * 3 * TS_PLANE;
      const double* const plm1 = ring + (size_t)slot_of(k - 1) * 3 * TS_PLANE;
      const double* const plp1 = ring + (size_t)slot_of(k + 1) * 3 * TS_PLANE;
      const double* const plm2 = ring + (size_t)slot_of(k - 2) * 3 * TS_PLANE;
      const double* const plp2 = ring + (size_t)slot_of(k + 2) * 3 * TS_PLANE;
      const int64_t c = (int64_t)k * sz + (int64_t)j * sy + i;
      const double inv_rho = 1.0 / rho_c;
      const double* rk = rkz + 4 * (k - k0);
      const double inv_d_above = rk[0], inv_d_below = rk[1], inv_dz_k = rk[2], inv_hz = rk[3];
      const double stot = sp + sd;
      const bool mx = (i >= 2 && i <= nx - 3);
      const bool mz = (k >= 2 && k <= nz - 3);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double* P0 = pl0 + s * TS_PLANE;
        const double Yi = P0[cix];
        const double Yxm1 = P0[cix - 1], Yxp1 = P0[cix + 1];
        const double YL_x = (i == 0) ? a.Y_inlet[s] : Yxm1;
        const double YR_x = (i == nx - 1) ? Yi : Yxp1;
        const double Yzm1 = plm1[s * TS_PLANE + cix], Yzp1 = plp1[s * TS_PLANE + cix];
        const double YL_z = (k == 0) ? Yi : Yzm1;
        const double YR_z = (k == nz - 1) ? Yi : Yzp1;
        double flux_x, flux_z;
        if (mx) {
          double fxp = muscl_face(Yxm1, Yi, Yxp1, P0[cix + 2], ui);
          double fxm = muscl_face(P0[cix - 2], Yxm1, Yi, Yxp1, ui);
          flux_x = ui * (fxp - fxm) * inv_dx;
        } else {
          flux_x = (ui >= 0.0) ? ui * (Yi - YL_x) * inv_dx : ui * (YR_x - Yi) * inv_dx;
        }
        const double Yjm2 = P0[cix - 2 * TS_HX], Yjm1 = P0[cix - TS_HX];
        const double Yjp1 = P0[cix + TS_HX], Yjp2 = P0[cix + 2 * TS_HX];
        double fyp = muscl_face(Yjm1, Yi, Yjp1, Yjp2, vi);
        double fym = muscl_face(Yjm2, Yjm1, Yi, Yjp1, vi);
        double flux_y = vi * (fyp - fym) * inv_dy;
        if (mz) {
          double fzp = muscl_face(Yzm1, Yi, Yzp1, plp2[s * TS_PLANE + cix], wi);
          double fzm = muscl_face(plm2[s * TS_PLANE + cix], Yzm1, Yi, Yzp1, wi);
          flux_z = wi * (fzp - fzm) * inv_hz;
        } else {
          flux_z = (wi >= 0.0) ? wi * (Yi - YL_z) * inv_d_below : wi * (YR_z - Yi) * inv_d_above;
        }
        double adv = -(flux_x + flux_y + flux_z);
        double d2x = (YR_x - 2.0 * Yi + YL_x) * inv_dx2;
        double d2y = (Yjp1 - 2.0 * Yi + Yjm1) * inv_dy2;
        double d2z = ((YR_z - Yi) * inv_d_above - (Yi - YL_z) * inv_d_below) * inv_dz_k;
        double diff = D * (d2x + d2y + d2z);
        double S = (s == 0) ? sp - Yi * stot : ((s == 1) ? -(Yi * stot) : sd - Yi * stot);
        double src = S * inv_rho;
        double dY = (adv + diff + src) * dt;
        double nw = Yi + dY;
        if (nw < 0.0) nw = 0.0;
        else if (nw > 1.0) nw = 1.0;
        if (s == 1) {
          if (nw > a.o2_cap) nw = a.o2_cap;
          if (nw < 0.0) nw = 0.0;
        }
        a.Yo[s][c] = nw;
      }
    }
    // every thread is done with plane k-2's slot: plane k+4 may land there
    if (ywrap) tma_fence_proxy();
    __syncthreads();
    if (tid == 0 && k + 4 <= plast && k + 4 > pfirst + TS_SLOTS - 1) {
      tma_fence_proxy();
      issue(k + 4);
    }
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;
static bool g_tma_on = true;

bool tma_enabled() { return g_tma_on; }

bool tma_map_field(CUtensorMap* map, const double* base, int nx, int ny, int nz, int bx, int by) {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    else
      cudaGetLastError();
  });
  if (!g_encode || !base || (nx & 1) || ((uintptr_t)base & 15) || bx > 256 || by > 256 ||
      (bx * (int)sizeof(double)) % 16)
    return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(double),
                                 (cuuint64_t)nx * ny * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the TMA form of the fused species step; false when it cannot run here
static bool launch_species_step_tma(const GridDev& g, const SpeciesArgs& a, const double* rho,
                                    const double* u, const double* v, const double* w, double dt,
                                    double D, cudaStream_t st) {
  if (!tma_enabled()) return false;
  SpeciesMaps tm;
  for (int s = 0; s < 3; ++s)
    if (!tma_map_field(&tm.Y[s], a.Y[s], g.nx, g.ny, g.nz, TS_HX, TS_HY)) return false;
  const int tiles = ((g.nx + SP_TX - 1) / SP_TX) * ((g.ny + SP_TY - 1) / SP_TY);
  // enough blocks for about six per SM of the 148, in z-chunks of at most
  // TS_MAXKZ levels
  int chunks = (6 * 148 + tiles - 1) / tiles;
  if (chunks > g.nz) chunks = g.nz;
  if (chunks < 1) chunks = 1;
  int kz = (g.nz + chunks - 1) / chunks;
  if (kz < 4) kz = g.nz < 4 ? g.nz : 4;  // at least four levels per chunk (halo overhead)
  if (kz > TS_MAXKZ) kz = TS_MAXKZ;
  chunks = (g.nz + kz - 1) / kz;
  static bool attr = false;
  const size_t smem = species_tma_smem();
  if (!attr) {
    if (cudaFuncSetAttribute(k_species_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    attr = true;
  }
  const dim3 nb((g.nx + SP_TX - 1) / SP_TX, (g.ny + SP_TY - 1) / SP_TY, chunks);
  const dim3 tb(SP_TX, SP_TY);
  const double inv_dx = 1.0 / g.dx, inv_dy = 1.0 / g.dy;
  k_species_tma<<<nb, tb, smem, st>>>(g, a, tm, rho, u, v, w, dt, D, inv_dx, inv_dy,
                                      inv_dx * inv_dx, inv_dy * inv_dy, kz);
  fs_count_launch();
  return true;
}

int stencil_status(int clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_stencil_err, sizeof(int)) != cudaSuccess) return -1;
  if (clear && v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_stencil_err, &z, sizeof(int));
  }
  return v;
}

void set_tma(int on) { g_tma_on = on != 0; }

// ---------------------------------------------------------------------------
// Species source terms with dilution (spread_3d.py:2996-3004, Lagrangian branch)
//   S_F = Sp - Y_F (Sp + Sd); S_O2 = -Y_O2 (Sp + Sd); S_H2O = Sd - Y_H2O (Sp + Sd)
// ---------------------------------------------------------------------------
__global__ void k_species_sources(int64_t n, const double* __restrict__ Sp,
                                  const double* __restrict__ Sd, const double* __restrict__ YF,
                                  const double* __restrict__ YO, const double* __restrict__ YH,
                                  double* SF, double* SO, double* SH) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double sp = Sp[c], sd = Sd[c];
  double st = sp + sd;
  SF[c] = sp - YF[c] * st;
  SO[c] = -(YO[c] * st);
  SH[c] = sd - YH[c] * st;
}

int launch_species_sources(int64_t n, const double* Sp, const double* Sd, const double* YF,
                           const double* YO, const double* YH, double* SF, double* SO,
                           double* SH, cudaStream_t st) {
  k_species_sources<<<blocks_for(n, 256), 256, 0, st>>>(n, Sp, Sd, YF, YO, YH, SF, SO, SH); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Scalar MUSCL advection accumulator (muscl_3d.py:67-171):  rhs -= u . grad(phi)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double advect_flux_sum(const GridDev& g, const double* __restrict__ phi,
                                                  int k, int j, int i, int64_t c, double uc,
                                                  double vc, double wc, double phi_inlet) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const double pc = phi[c];
  const double xL = (i == 0) ? phi_inlet : phi[c - 1];
  const double xR = (i == nx - 1) ? pc : phi[c + 1];
  const double zL = (k == 0) ? pc : phi[c - sz];
  const double zR = (k == nz - 1) ? pc : phi[c + sz];
  double fx, fz;
  if (i >= 2 && i <= nx - 3) {
    double fp = muscl_face(phi[c - 1], pc, phi[c + 1], phi[c + 2], uc);
    double fm = muscl_face(phi[c - 2], phi[c - 1], pc, phi[c + 1], uc);
    fx = uc * (fp - fm) / g.dx;
  } else {
    fx = (uc >= 0.0) ? uc * (pc - xL) / g.dx : uc * (xR - pc) / g.dx;
  }
  const int64_t crow = c - (int64_t)j * sy;
  const int jm2 = wrapj(j - 2, ny), jm1 = wrapj(j - 1, ny);
  const int jp1 = wrapj(j + 1, ny), jp2 = wrapj(j + 2, ny);
  double fyp = muscl_face(phi[crow + jm1 * sy], pc, phi[crow + jp1 * sy], phi[crow + jp2 * sy], vc);
  double fym = muscl_face(phi[crow + jm2 * sy], phi[crow + jm1 * sy], pc, phi[crow + jp1 * sy], vc);
  double fy = vc * (fyp - fym) / g.dy;
  if (k >= 2 && k <= nz - 3) {
    double fp = muscl_face(phi[c - sz], pc, phi[c + sz], phi[c + 2 * sz], wc);
    double fm = muscl_face(phi[c - 2 * sz], phi[c - sz], pc, phi[c + sz], wc);
    fz = wc * (fp - fm) / (0.5 * (g.da[k] + g.db[k]));
  } else {
    double inv_db = 1.0 / g.db[k], inv_da = 1.0 / g.da[k];
    fz = (wc >= 0.0) ? wc * (pc - zL) * inv_db : wc * (zR - pc) * inv_da;
  }
  return fx + fy + fz;
}

__global__ void k_advect_scalar(GridDev g, const double* __restrict__ phi,
                                const double* __restrict__ u, const double* __restrict__ v,
                                const double* __restrict__ w, double* rhs, double phi_inlet) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  int64_t c = cidx(g, k, j, i);
  rhs[c] -= advect_flux_sum(g, phi, k, j, i, c, u[c], v[c], w[c], phi_inlet);
}

int launch_advect_scalar(const GridDev& g, const double* phi, const double* u, const double* v,
                         const double* w, double* rhs, double phi_inlet, cudaStream_t st) {
  Launch3 L = launch_cells(g);
  k_advect_scalar<<<L.grid, L.block, 0, st>>>(g, phi, u, v, w, rhs, phi_inlet); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Gas-temperature advection + molecular diffusion (spread_3d.py:3827-3897 _adv_gas_energy)
// ---------------------------------------------------------------------------
__global__ void k_gas_energy_adv(GridDev g, const double* __restrict__ T,
                                 const double* __restrict__ u, const double* __restrict__ v,
                                 const double* __restrict__ w, double* __restrict__ To, double dt,
                                 double alpha, double T_amb, double inv_dx2, double dy2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int64_t c = cidx(g, k, j, i);
  const double Tc = T[c];
  double dT = 0.0 - advect_flux_sum(g, T, k, j, i, c, u[c], v[c], w[c], T_amb);
  // x diffusion: interior central, inlet ghost T_amb, outlet zero-gradient
  if (i >= 1 && i <= nx - 2) {
    dT += alpha * (T[c + 1] - 2.0 * Tc + T[c - 1]) * inv_dx2;
  } else if (i == 0) {
    dT += alpha * (T[c + 1] - 2.0 * Tc + T_amb) * inv_dx2;
  }
  if (i == nx - 1) {
    dT += alpha * (T[c - 1] - Tc) * inv_dx2;
  }
  // y diffusion (periodic)
  {
    const int64_t crow = c - (int64_t)j * sy;
    const double Tp = T[crow + wrapj(j + 1, ny) * sy];
    const double Tm = T[crow + wrapj(j - 1, ny) * sy];
    dT += alpha * (Tp - 2.0 * Tc + Tm) / dy2;
  }
  // z diffusion (finite-volume, zero-flux wall and top)
  if (k >= 1 && k <= nz - 2) {
    double ida = 1.0 / g.da[k], idb = 1.0 / g.db[k], idz = 1.0 / g.dz[k];
    dT += alpha * ((T[c + sz] - Tc) * ida - (Tc - T[c - sz]) * idb) * idz;
  } else if (k == 0) {
    dT += alpha * ((T[c + sz] - Tc) / g.da[0]) / g.dz[0];
  }
  if (k == nz - 1) {
    dT += alpha * (-(Tc - T[c - sz]) / g.db[nz - 1]) / g.dz[nz - 1];
  }
  double Tn = Tc + dT * dt;
  if (Tn < T_amb) Tn = T_amb;
  if (Tn > 10000.0) Tn = 10000.0;
  To[c] = Tn;
}

int launch_gas_energy_adv(const GridDev& g, const double* T, const double* u, const double* v,
                          const double* w, double* To, double dt, double alpha, double T_amb,
                          cudaStream_t st) {
  if (g.nx < 3 || g.nz < 3) return FS_EARG;
  Launch3 L = launch_cells(g);
  k_gas_energy_adv<<<L.grid, L.block, 0, st>>>(g, T, u, v, w, To, dt, alpha, T_amb,
                                               1.0 / (g.dx * g.dx), g.dy * g.dy); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Turbulent diffusion sub-iteration for up to 4 fields sharing nu_t and sc_t
// (turbulence_3d.py:862-949 apply_turbulent_diffusion, inner prange pair)
// Optional clip [lo, hi] after the LAST sub-iteration is applied by the caller.
// ---------------------------------------------------------------------------
struct DiffArgs {
  const double* f[4];
  double* fo[4];
  double lo[4], hi[4];
  int nfield;
  int clip;
};

// A block owns a 32 x 8 (x, y) tile and marches up a chunk of z-levels: each
// thread keeps its column's values at k-1, k and k+1 of every field in
// registers (the z-neighbours cost no loads) and requests level k+2 (and the
// next level's nu_t) while level k computes, so a column always has a level
// of loads in flight; x- and y-neighbours come from L1.  The chunk's
// reciprocal spacings are computed once per block.  The arithmetic of each
// cell is the one-thread-per-cell form's, expression for expression.
#define TD_MAXKZ 64
template <int NF>
__global__ void __launch_bounds__(SP_TX * SP_TY, 4)
k_turb_diff(GridDev g, DiffArgs a, const double* __restrict__ nu_t, double sc_t, double dt_sub,
            double inv_dx2, double inv_dy2, int kz) {
  __shared__ double rk[TD_MAXKZ][3];  // 1/dz, 1/da, 1/db of the chunk's levels
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int k0 = blockIdx.z * kz;
  const int k1 = min(nz, k0 + kz);
  const int tid = threadIdx.y * SP_TX + threadIdx.x;
  for (int q = tid; q < k1 - k0; q += SP_TX * SP_TY) {
    rk[q][0] = 1.0 / g.dz[k0 + q];
    rk[q][1] = 1.0 / g.da[k0 + q];
    rk[q][2] = 1.0 / g.db[k0 + q];
  }
  __syncthreads();
  const int i = blockIdx.x * SP_TX + threadIdx.x;
  const int j = blockIdx.y * SP_TY + threadIdx.y;
  if (i >= nx || j >= ny || k0 >= nz) return;
  const int64_t col = (int64_t)j * sy + i;
  const int64_t cjp0 = (int64_t)wrapj(j + 1, ny) * sy + i, cjm0 = (int64_t)wrapj(j - 1, ny) * sy + i;
  // fL, fC, fN: the column at k-1, k and k+1 (k+1 clamped to k at the top)
  double fL[NF], fC[NF], fN[NF];
#pragma unroll
  for (int s = 0; s < NF; ++s) {
    fC[s] = a.f[s][(int64_t)k0 * sz + col];
    fL[s] = (k0 == 0) ? fC[s] : a.f[s][(int64_t)(k0 - 1) * sz + col];
    fN[s] = (k0 == nz - 1) ? fC[s] : a.f[s][(int64_t)(k0 + 1) * sz + col];
  }
  double nu_c = nu_t[(int64_t)k0 * sz + col];
  for (int k = k0; k < k1; ++k) {
    const int64_t ks = (int64_t)k * sz;
    const int64_t c = ks + col;
    // the next level's loads: nu_t at k+1 and the fields at k+2
    const bool more = k + 1 < k1;
    double nu_n = 0.0, fNN[NF];
    if (more) nu_n = nu_t[c + sz];
#pragma unroll
    for (int s = 0; s < NF; ++s)
      fNN[s] = (more && k + 2 < nz) ? a.f[s][c + 2 * sz] : fN[s];
    const double inv_dz_k = rk[k - k0][0];
    const double inv_d_above = rk[k - k0][1];
    const double inv_d_below = rk[k - k0][2];
    const double D_t = nu_c / sc_t;
#pragma unroll
    for (int s = 0; s < NF; ++s) {
      const double* __restrict__ f = a.f[s];
      const double fc = fC[s];
      const double fxL = (i == 0) ? fc : f[c - 1];
      const double fxR = (i == nx - 1) ? fc : f[c + 1];
      const double fzL = fL[s];
      const double fzR = fN[s];
      double d2x = (fxR - 2.0 * fc + fxL) * inv_dx2;
      double d2y = (f[ks + cjp0] - 2.0 * fc + f[ks + cjm0]) * inv_dy2;
      double d2z = ((fzR - fc) * inv_d_above - (fc - fzL) * inv_d_below) * inv_dz_k;
      double df = D_t * (d2x + d2y + d2z) * dt_sub;
      double nv = fc + df;
      if (a.clip) {
        if (nv < a.lo[s]) nv = a.lo[s];
        if (nv > a.hi[s]) nv = a.hi[s];
      }
      a.fo[s][c] = nv;
      fL[s] = fc;
      fC[s] = fzR;
      fN[s] = fNN[s];
    }
    nu_c = nu_n;
  }
}

int launch_turb_diff(const GridDev& g, int nfield, const double* const* f, double* const* fo,
                     const double* nu_t, double sc_t, double dt_sub, int clip, const double* lo,
                     const double* hi, cudaStream_t st) {
  if (nfield < 1 || nfield > 4) return FS_EARG;
  DiffArgs a{};
  a.nfield = nfield;
  a.clip = clip;
  for (int s = 0; s < nfield; ++s) {
    a.f[s] = f[s]; a.fo[s] = fo[s];
    a.lo[s] = clip ? lo[s] : 0.0;
    a.hi[s] = clip ? hi[s] : 0.0;
  }
  // z-chunks: about six blocks per SM of the 148, at least four levels each
  const int tiles = ((g.nx + SP_TX - 1) / SP_TX) * ((g.ny + SP_TY - 1) / SP_TY);
  int chunks = (6 * 148 + tiles - 1) / tiles;
  if (chunks > g.nz) chunks = g.nz;
  if (chunks < 1) chunks = 1;
  int kz = (g.nz + chunks - 1) / chunks;
  if (kz < 4) kz = g.nz < 4 ? g.nz : 4;
  if (kz > TD_MAXKZ) kz = TD_MAXKZ;
  chunks = (g.nz + kz - 1) / kz;
  const dim3 nb((g.nx + SP_TX - 1) / SP_TX, (g.ny + SP_TY - 1) / SP_TY, chunks);
  const dim3 tb(SP_TX, SP_TY);
  const double ix2 = 1.0 / (g.dx * g.dx), iy2 = 1.0 / (g.dy * g.dy);
  switch (nfield) {
    case 1: k_turb_diff<1><<<nb, tb, 0, st>>>(g, a, nu_t, sc_t, dt_sub, ix2, iy2, kz); break;
    case 2: k_turb_diff<2><<<nb, tb, 0, st>>>(g, a, nu_t, sc_t, dt_sub, ix2, iy2, kz); break;
    case 3: k_turb_diff<3><<<nb, tb, 0, st>>>(g, a, nu_t, sc_t, dt_sub, ix2, iy2, kz); break;
    default: k_turb_diff<4><<<nb, tb, 0, st>>>(g, a, nu_t, sc_t, dt_sub, ix2, iy2, kz); break;
  }
  fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Porous drag (drag_3d.py:100-144 step_drag_force)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double drag_coeff(double ui, double vi, double wi, double rho,
                                             double a, double sigma, double sigma2, double C_D) {
  double speed = sqrt(ui * ui + vi * vi + wi * wi);
  double om = 1.0 - a;
  double K_visc = 50.0 * 3.0e-5 * sigma2 * a * a / (om * om * om);
  double K_quad = C_D * sigma * a * 0.5 * rho * speed;
  return -(K_visc + K_quad);
}

__global__ void k_drag(int64_t n, const double* __restrict__ u, const double* __restrict__ v,
                       const double* __restrict__ w, const double* __restrict__ rho,
                       const double* __restrict__ as, double sigma, double sigma2, double C_D,
                       double* Fx, double* Fy, double* Fz) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double a = as[c];
  if (a <= 0.0) {
    Fx[c] = 0.0; Fy[c] = 0.0; Fz[c] = 0.0;
    return;
  }
  double ui = u[c], vi = v[c], wi = w[c];
  double co = drag_coeff(ui, vi, wi, rho[c], a, sigma, sigma2, C_D);
  Fx[c] = co * ui; Fy[c] = co * vi; Fz[c] = co * wi;
}

int launch_drag(int64_t n, const double* u, const double* v, const double* w, const double* rho,
                const double* as, double sigma, double C_D, double* Fx, double* Fy, double* Fz,
                cudaStream_t st) {
  k_drag<<<blocks_for(n, 256), 256, 0, st>>>(n, u, v, w, rho, as, sigma, sigma * sigma, C_D, Fx,
                                             Fy, Fz); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Tentative velocity (momentum_3d.py:42-276), optionally with the porous drag
// force evaluated in-kernel (drag_3d.py:128-144) instead of read from Fx/Fy/Fz.
// ---------------------------------------------------------------------------
struct MomArgs {
  const double *u, *v, *w, *rho, *T;
  const double *Fx, *Fy, *Fz;           // null when drag is fused
  const double *alpha_s;                // used when drag is fused
  const double *u_in, *v_in, *w_in;     // (Nz, Ny) inlet ghosts; v_in/w_in may be null
  double *uo, *vo, *wo;
  double sigma, sigma2, C_D;
  double dt, T_amb;
  double inv_dx, inv_dy, inv_dx2, inv_dy2;
};

__global__ void k_momentum(GridDev g, MomArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int64_t c = cidx(g, k, j, i);
  const double* u = a.u; const double* v = a.v; const double* w = a.w;
  const double ui = u[c], vi = v[c], wi = w[c];
  const double rho_i = a.rho[c];
  const double nu_i = 1.8e-5 / rho_i;
  double uLx, vLx, wLx, uRx, vRx, wRx, uLz, vLz, wLz, uRz, vRz, wRz;
  if (i == 0) {
    int64_t q = (int64_t)k * ny + j;
    uLx = a.u_in[q];
    vLx = a.v_in ? a.v_in[q] : 0.0;
    wLx = a.w_in ? a.w_in[q] : 0.0;
  } else {
    uLx = u[c - 1]; vLx = v[c - 1]; wLx = w[c - 1];
  }
  if (i == nx - 1) { uRx = ui; vRx = vi; wRx = wi; }
  else { uRx = u[c + 1]; vRx = v[c + 1]; wRx = w[c + 1]; }
  if (k == 0) { uLz = 0.0; vLz = 0.0; wLz = 0.0; }
  else { uLz = u[c - sz]; vLz = v[c - sz]; wLz = w[c - sz]; }
  if (k == nz - 1) { uRz = ui; vRz = vi; wRz = wi; }
  else { uRz = u[c + sz]; vRz = v[c + sz]; wRz = w[c + sz]; }

  double dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz;
  if (i >= 2 && i <= nx - 3) {
    double uxp = muscl_face(u[c - 1], ui, u[c + 1], u[c + 2], ui);
    double uxm = muscl_face(u[c - 2], u[c - 1], ui, u[c + 1], ui);
    double vxp = muscl_face(v[c - 1], vi, v[c + 1], v[c + 2], ui);
    double vxm = muscl_face(v[c - 2], v[c - 1], vi, v[c + 1], ui);
    double wxp = muscl_face(w[c - 1], wi, w[c + 1], w[c + 2], ui);
    double wxm = muscl_face(w[c - 2], w[c - 1], wi, w[c + 1], ui);
    dudx = (uxp - uxm) * a.inv_dx;
    dvdx = (vxp - vxm) * a.inv_dx;
    dwdx = (wxp - wxm) * a.inv_dx;
  } else if (ui >= 0.0) {
    dudx = (ui - uLx) * a.inv_dx; dvdx = (vi - vLx) * a.inv_dx; dwdx = (wi - wLx) * a.inv_dx;
  } else {
    dudx = (uRx - ui) * a.inv_dx; dvdx = (vRx - vi) * a.inv_dx; dwdx = (wRx - wi) * a.inv_dx;
  }
  const int64_t crow = c - (int64_t)j * sy;
  const int64_t cm2 = crow + wrapj(j - 2, ny) * sy, cm1 = crow + wrapj(j - 1, ny) * sy;
  const int64_t cp1 = crow + wrapj(j + 1, ny) * sy, cp2 = crow + wrapj(j + 2, ny) * sy;
  {
    double uyp = muscl_face(u[cm1], ui, u[cp1], u[cp2], vi);
    double uym = muscl_face(u[cm2], u[cm1], ui, u[cp1], vi);
    double vyp = muscl_face(v[cm1], vi, v[cp1], v[cp2], vi);
    double vym = muscl_face(v[cm2], v[cm1], vi, v[cp1], vi);
    double wyp = muscl_face(w[cm1], wi, w[cp1], w[cp2], vi);
    double wym = muscl_face(w[cm2], w[cm1], wi, w[cp1], vi);
    dudy = (uyp - uym) * a.inv_dy;
    dvdy = (vyp - vym) * a.inv_dy;
    dwdy = (wyp - wym) * a.inv_dy;
  }
  if (k >= 2 && k <= nz - 3) {
    double inv_dz_eff = 1.0 / (0.5 * (g.da[k] + g.db[k]));
    double uzp = muscl_face(u[c - sz], ui, u[c + sz], u[c + 2 * sz], wi);
    double uzm = muscl_face(u[c - 2 * sz], u[c - sz], ui, u[c + sz], wi);
    double vzp = muscl_face(v[c - sz], vi, v[c + sz], v[c + 2 * sz], wi);
    double vzm = muscl_face(v[c - 2 * sz], v[c - sz], vi, v[c + sz], wi);
    double wzp = muscl_face(w[c - sz], wi, w[c + sz], w[c + 2 * sz], wi);
    double wzm = muscl_face(w[c - 2 * sz], w[c - sz], wi, w[c + sz], wi);
    dudz = (uzp - uzm) * inv_dz_eff;
    dvdz = (vzp - vzm) * inv_dz_eff;
    dwdz = (wzp - wzm) * inv_dz_eff;
  } else if (wi >= 0.0) {
    double idb = 1.0 / g.db[k];
    dudz = (ui - uLz) * idb; dvdz = (vi - vLz) * idb; dwdz = (wi - wLz) * idb;
  } else {
    double ida = 1.0 / g.da[k];
    dudz = (uRz - ui) * ida; dvdz = (vRz - vi) * ida; dwdz = (wRz - wi) * ida;
  }
  double adv_u = -(ui * dudx + vi * dudy + wi * dudz);
  double adv_v = -(ui * dvdx + vi * dvdy + wi * dvdz);
  double adv_w = -(ui * dwdx + vi * dwdy + wi * dwdz);

  const double inv_dz_k = 1.0 / g.dz[k];
  const double inv_d_above = 1.0 / g.da[k];
  const double inv_d_below = 1.0 / g.db[k];
  double d2u_dx2 = (uRx - 2.0 * ui + uLx) * a.inv_dx2;
  double d2u_dy2 = (u[cp1] - 2.0 * ui + u[cm1]) * a.inv_dy2;
  double d2u_dz2 = ((uRz - ui) * inv_d_above - (ui - uLz) * inv_d_below) * inv_dz_k;
  double d2v_dx2 = (vRx - 2.0 * vi + vLx) * a.inv_dx2;
  double d2v_dy2 = (v[cp1] - 2.0 * vi + v[cm1]) * a.inv_dy2;
  double d2v_dz2 = ((vRz - vi) * inv_d_above - (vi - vLz) * inv_d_below) * inv_dz_k;
  double d2w_dx2 = (wRx - 2.0 * wi + wLx) * a.inv_dx2;
  double d2w_dy2 = (w[cp1] - 2.0 * wi + w[cm1]) * a.inv_dy2;
  double d2w_dz2 = ((wRz - wi) * inv_d_above - (wi - wLz) * inv_d_below) * inv_dz_k;
  double visc_u = nu_i * (d2u_dx2 + d2u_dy2 + d2u_dz2);
  double visc_v = nu_i * (d2v_dx2 + d2v_dy2 + d2v_dz2);
  double visc_w = nu_i * (d2w_dx2 + d2w_dy2 + d2w_dz2);
  double buoy_w = 9.81 * (a.T[c] - a.T_amb) / a.T_amb;
  double Fx, Fy, Fz;
  if (a.Fx) {
    Fx = a.Fx[c]; Fy = a.Fy[c]; Fz = a.Fz[c];
  } else {
    double as = a.alpha_s[c];
    if (as <= 0.0) {
      Fx = 0.0; Fy = 0.0; Fz = 0.0;
    } else {
      double co = drag_coeff(ui, vi, wi, rho_i, as, a.sigma, a.sigma2, a.C_D);
      Fx = co * ui; Fy = co * vi; Fz = co * wi;
    }
  }
  double ext_u = Fx / rho_i, ext_v = Fy / rho_i, ext_w = Fz / rho_i;
  double du = (adv_u + visc_u + ext_u) * a.dt;
  double dv = (adv_v + visc_v + ext_v) * a.dt;
  double dw = (adv_w + visc_w + buoy_w + ext_w) * a.dt;
  a.uo[c] = ui + du;
  a.vo[c] = vi + dv;
  a.wo[c] = wi + dw;
}

int launch_momentum(const GridDev& g, const double* u, const double* v, const double* w,
                    const double* rho, const double* T, const double* Fx, const double* Fy,
                    const double* Fz, const double* alpha_s, double sigma, double C_D,
                    const double* u_in, const double* v_in, const double* w_in, double* uo,
                    double* vo, double* wo, double dt, double T_amb, cudaStream_t st) {
  MomArgs a{};
  a.u = u; a.v = v; a.w = w; a.rho = rho; a.T = T;
  a.Fx = Fx; a.Fy = Fy; a.Fz = Fz; a.alpha_s = alpha_s;
  if (!Fx && !alpha_s) return FS_EARG;
  a.u_in = u_in; a.v_in = v_in; a.w_in = w_in;
  a.uo = uo; a.vo = vo; a.wo = wo;
  a.sigma = sigma; a.sigma2 = sigma * sigma; a.C_D = C_D;
  a.dt = dt; a.T_amb = T_amb;
  a.inv_dx = 1.0 / g.dx; a.inv_dy = 1.0 / g.dy;
  a.inv_dx2 = a.inv_dx * a.inv_dx; a.inv_dy2 = a.inv_dy * a.inv_dy;
  Launch3 L = launch_cells(g);
  k_momentum<<<L.grid, L.block, 0, st>>>(g, a); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Outflow sponge (momentum_3d.py:293-317), in place
// ---------------------------------------------------------------------------
__global__ void k_sponge(GridDev g, double* u, const double* __restrict__ u_t,
                         const double* __restrict__ sig_x, const double* __restrict__ YF,
                         double skip, double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  double s = sig_x[i];
  int64_t c = cidx(g, k, j, i);
  if (s > 0.0 && YF[c] < skip) {
    double ut = u_t[(int64_t)k * g.ny + j];
    u[c] += s * dt * (ut - u[c]);
  }
}

int launch_sponge(const GridDev& g, double* u, const double* u_t, const double* sig_x,
                  const double* YF, double skip, double dt, cudaStream_t st) {
  Launch3 L = launch_cells(g);
  k_sponge<<<L.grid, L.block, 0, st>>>(g, u, u_t, sig_x, YF, skip, dt); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Realizable k-epsilon with in-kernel strain/vorticity invariants
// (turbulence_3d.py:392-478 _strain_and_vorticity_squared and :482-858
//  step_k_epsilon; buoyancy gradient with the one-sided boundary form of the
//  upstream fix, docs/js/physics/kepsilon.js:182-185,233-236)
// ---------------------------------------------------------------------------
struct KepsArgs {
  const double *k, *e, *u, *v, *w, *T, *alpha_s, *u_in, *kwall, *ewall;
  double *ko, *eo, *nuo;
  double *S2o, *O2o;  // optional outputs of the invariants (may be null)
  double sigma, dt, T_amb, beta_p, beta_d;
  double inv_dx, inv_dy, inv_dx2, inv_dy2;
};

__device__ __forceinline__ void strain_invariants(const GridDev& g, const KepsArgs& a, int k,
                                                  int j, int i, int64_t c, double& S2,
                                                  double& O2) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  double idzc;
  if (k == 0) idzc = 1.0 / g.da[0];
  else if (k == nz - 1) idzc = 1.0 / g.db[nz - 1];
  else idzc = 1.0 / (g.db[k] + g.da[k]);
  const double ui = a.u[c], vi = a.v[c], wi = a.w[c];
  double uxL, vxL, wxL, uxR, vxR, wxR, uzL, vzL, wzL, uzR, vzR, wzR;
  if (i == 0) { uxL = a.u_in[(int64_t)k * ny + j]; vxL = 0.0; wxL = 0.0; }
  else { uxL = a.u[c - 1]; vxL = a.v[c - 1]; wxL = a.w[c - 1]; }
  if (i == nx - 1) { uxR = ui; vxR = vi; wxR = wi; }
  else { uxR = a.u[c + 1]; vxR = a.v[c + 1]; wxR = a.w[c + 1]; }
  if (k == 0) { uzL = 0.0; vzL = 0.0; wzL = 0.0; }
  else { uzL = a.u[c - sz]; vzL = a.v[c - sz]; wzL = a.w[c - sz]; }
  if (k == nz - 1) { uzR = ui; vzR = vi; wzR = wi; }
  else { uzR = a.u[c + sz]; vzR = a.v[c + sz]; wzR = a.w[c + sz]; }
  const int64_t crow = c - (int64_t)j * sy;
  const int64_t cp = crow + wrapj(j + 1, ny) * sy, cm = crow + wrapj(j - 1, ny) * sy;
  double dudx = (uxR - uxL) * 0.5 * a.inv_dx;
  double dudy = (a.u[cp] - a.u[cm]) * 0.5 * a.inv_dy;
  double dudz = (uzR - uzL) * idzc;
  double dvdx = (vxR - vxL) * 0.5 * a.inv_dx;
  double dvdy = (a.v[cp] - a.v[cm]) * 0.5 * a.inv_dy;
  double dvdz = (vzR - vzL) * idzc;
  double dwdx = (wxR - wxL) * 0.5 * a.inv_dx;
  double dwdy = (a.w[cp] - a.w[cm]) * 0.5 * a.inv_dy;
  double dwdz = (wzR - wzL) * idzc;
  double S12 = 0.5 * (dudy + dvdx), S13 = 0.5 * (dudz + dwdx), S23 = 0.5 * (dvdz + dwdy);
  S2 = 2.0 * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + 4.0 * (S12 * S12 + S13 * S13 + S23 * S23);
  double O12 = 0.5 * (dudy - dvdx), O13 = 0.5 * (dudz - dwdx), O23 = 0.5 * (dvdz - dwdy);
  O2 = 4.0 * (O12 * O12 + O13 * O13 + O23 * O23);
}

#define K_MIN 1.0e-8
#define EPS_MIN 1.0e-8

__global__ void k_keps(GridDev g, KepsArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int64_t c = cidx(g, k, j, i);
  const double* KT = a.k;
  const double* ET = a.e;
  double S2, O2;
  strain_invariants(g, a, k, j, i, c, S2, O2);
  if (a.S2o) { a.S2o[c] = S2; a.O2o[c] = O2; }

  const double inv_dz_k = 1.0 / g.dz[k];
  const double inv_d_above = 1.0 / g.da[k];
  const double inv_d_below = 1.0 / g.db[k];
  const double hz = 0.5 * (g.da[k] + g.db[k]);
  double k_loc = KT[c], e_loc = ET[c];
  if (k_loc < K_MIN) k_loc = K_MIN;
  if (e_loc < EPS_MIN) e_loc = EPS_MIN;
  const int64_t q2 = (int64_t)j * nx + i;
  const double kxL = (i == 0) ? K_MIN : KT[c - 1];
  const double exL = (i == 0) ? EPS_MIN : ET[c - 1];
  const double kxR = (i == nx - 1) ? k_loc : KT[c + 1];
  const double exR = (i == nx - 1) ? e_loc : ET[c + 1];
  const double kzL = (k == 0) ? a.kwall[q2] : KT[c - sz];
  const double ezL = (k == 0) ? a.ewall[q2] : ET[c - sz];
  const double kzR = (k == nz - 1) ? k_loc : KT[c + sz];
  const double ezR = (k == nz - 1) ? e_loc : ET[c + sz];

  const double U_star = sqrt(0.5 * (S2 + O2));
  const double C_mu = 1.0 / (4.04 + 4.5 * U_star * k_loc / e_loc);
  double nu_t = C_mu * k_loc * k_loc / e_loc;
  if (nu_t < 0.0) nu_t = 0.0;
  const double P_k = nu_t * S2;
  double P_k_lim = P_k;
  if (P_k_lim > 10.0 * e_loc) P_k_lim = 10.0 * e_loc;
  double dTdz;
  if (k == 0) dTdz = (a.T[c + sz] - a.T[c]) * (1.0 / g.da[0]);
  else if (k == nz - 1) dTdz = (a.T[c] - a.T[c - sz]) * (1.0 / g.db[nz - 1]);
  else dTdz = (a.T[c + sz] - a.T[c - sz]) * (1.0 / (g.da[k] + g.db[k]));
  double Tfb = a.T[c];
  if (Tfb < a.T_amb) Tfb = a.T_amb;
  double G_k = (nu_t / 0.85) * (9.81 / Tfb) * dTdz;
  if (G_k < 0.0) G_k = 0.0;
  double G_kk = G_k;
  if (G_kk > P_k_lim) G_kk = P_k_lim;
  const double ui = a.u[c], vi = a.v[c], wi = a.w[c];
  double u_h = sqrt(ui * ui + vi * vi);
  if (u_h < 0.01) u_h = 0.01;
  const double C3 = tanh(fabs(wi) / u_h);
  double Pc = 0.0, Dc = 0.0;
  const double as = a.alpha_s[c];
  if (as > 0.0) {
    double a_v = a.sigma * as;
    double speed = sqrt(ui * ui + vi * vi + wi * wi);
    double cds = 1.0 * a_v * speed;
    Pc = a.beta_p * cds * speed * speed;
    Dc = a.beta_d * cds * k_loc;
  }
  const double G_B = 0.0;  // BVG term: bvg_factor = 0 at the production call site

  const int64_t crow = c - (int64_t)j * sy;
  const int64_t cm2 = crow + wrapj(j - 2, ny) * sy, cm1 = crow + wrapj(j - 1, ny) * sy;
  const int64_t cp1 = crow + wrapj(j + 1, ny) * sy, cp2 = crow + wrapj(j + 2, ny) * sy;
  const bool mx = (i >= 2 && i <= nx - 3), mz = (k >= 2 && k <= nz - 3);
  // ---- k
  double ax, ay, az;
  if (mx) {
    double fp = muscl_face(KT[c - 1], k_loc, KT[c + 1], KT[c + 2], ui);
    double fm = muscl_face(KT[c - 2], KT[c - 1], k_loc, KT[c + 1], ui);
    ax = ui * (fp - fm) * a.inv_dx;
  } else {
    ax = (ui >= 0.0) ? ui * (k_loc - kxL) * a.inv_dx : ui * (kxR - k_loc) * a.inv_dx;
  }
  {
    double fp = muscl_face(KT[cm1], k_loc, KT[cp1], KT[cp2], vi);
    double fm = muscl_face(KT[cm2], KT[cm1], k_loc, KT[cp1], vi);
    ay = vi * (fp - fm) * a.inv_dy;
  }
  if (mz) {
    double fp = muscl_face(KT[c - sz], k_loc, KT[c + sz], KT[c + 2 * sz], wi);
    double fm = muscl_face(KT[c - 2 * sz], KT[c - sz], k_loc, KT[c + sz], wi);
    az = wi * (fp - fm) / hz;
  } else {
    az = (wi >= 0.0) ? wi * (k_loc - kzL) * inv_d_below : wi * (kzR - k_loc) * inv_d_above;
  }
  double adv_k = ax + ay + az;
  double alpha_k = 1.5e-5 + nu_t / 1.0;
  double d2k = (kxR - 2.0 * k_loc + kxL) * a.inv_dx2 +
               (KT[cp1] - 2.0 * k_loc + KT[cm1]) * a.inv_dy2 +
               ((kzR - k_loc) * inv_d_above - (k_loc - kzL) * inv_d_below) * inv_dz_k;
  double diff_k = alpha_k * d2k;
  double S_pos_k = P_k_lim + G_kk + Pc + G_B;
  double S_neg_k = e_loc + Dc;
  double k_new = (k_loc + (-adv_k + diff_k + S_pos_k) * a.dt) / (1.0 + S_neg_k * a.dt / k_loc);
  if (k_new < K_MIN) k_new = K_MIN;
  // ---- epsilon
  if (mx) {
    double fp = muscl_face(ET[c - 1], e_loc, ET[c + 1], ET[c + 2], ui);
    double fm = muscl_face(ET[c - 2], ET[c - 1], e_loc, ET[c + 1], ui);
    ax = ui * (fp - fm) * a.inv_dx;
  } else {
    ax = (ui >= 0.0) ? ui * (e_loc - exL) * a.inv_dx : ui * (exR - e_loc) * a.inv_dx;
  }
  {
    double fp = muscl_face(ET[cm1], e_loc, ET[cp1], ET[cp2], vi);
    double fm = muscl_face(ET[cm2], ET[cm1], e_loc, ET[cp1], vi);
    ay = vi * (fp - fm) * a.inv_dy;
  }
  if (mz) {
    double fp = muscl_face(ET[c - sz], e_loc, ET[c + sz], ET[c + 2 * sz], wi);
    double fm = muscl_face(ET[c - 2 * sz], ET[c - sz], e_loc, ET[c + sz], wi);
    az = wi * (fp - fm) / hz;
  } else {
    az = (wi >= 0.0) ? wi * (e_loc - ezL) * inv_d_below : wi * (ezR - e_loc) * inv_d_above;
  }
  double adv_e = ax + ay + az;
  double alpha_e = 1.5e-5 + nu_t / 1.3;
  double d2e = (exR - 2.0 * e_loc + exL) * a.inv_dx2 +
               (ET[cp1] - 2.0 * e_loc + ET[cm1]) * a.inv_dy2 +
               ((ezR - e_loc) * inv_d_above - (e_loc - ezL) * inv_d_below) * inv_dz_k;
  double diff_e = alpha_e * d2e;
  double S_mag = sqrt(S2);
  double eta = S_mag * k_loc / e_loc;
  double eta3 = eta * (eta * eta);
  double rng = 0.09 * eta3 * (1.0 - eta / 4.38) / (1.0 + 0.012 * eta3);
  if (rng < 0.0) rng = 0.0;
  double C2 = 1.92 + rng;
  double ek = e_loc / k_loc;
  double S_pos_e = 1.44 * (P_k_lim + C3 * G_k) * ek + 0.9 * Pc * ek;
  double S_neg_e = C2 * e_loc * ek + 0.9 * Dc * ek;
  double e_new = (e_loc + (-adv_e + diff_e + S_pos_e) * a.dt) / (1.0 + S_neg_e * a.dt / e_loc);
  if (e_new < EPS_MIN) e_new = EPS_MIN;
  a.ko[c] = k_new;
  a.eo[c] = e_new;
  double C_mu_new = 1.0 / (4.04 + 4.5 * U_star * k_new / e_new);
  double nu_new = C_mu_new * k_new * k_new / e_new;
  if (nu_new < 0.0) nu_new = 0.0;
  a.nuo[c] = nu_new;
}

int launch_keps(const GridDev& g, const double* k, const double* e, const double* u,
                const double* v, const double* w, const double* T, const double* alpha_s,
                const double* u_in, const double* kwall, const double* ewall, double* ko,
                double* eo, double* nuo, double* S2o, double* O2o, double sigma, double dt,
                double T_amb, double beta_p, double beta_d, cudaStream_t st) {
  KepsArgs a{};
  a.k = k; a.e = e; a.u = u; a.v = v; a.w = w; a.T = T; a.alpha_s = alpha_s; a.u_in = u_in;
  a.kwall = kwall; a.ewall = ewall; a.ko = ko; a.eo = eo; a.nuo = nuo; a.S2o = S2o; a.O2o = O2o;
  a.sigma = sigma; a.dt = dt; a.T_amb = T_amb; a.beta_p = beta_p; a.beta_d = beta_d;
  a.inv_dx = 1.0 / g.dx; a.inv_dy = 1.0 / g.dy;
  a.inv_dx2 = 1.0 / (g.dx * g.dx); a.inv_dy2 = 1.0 / (g.dy * g.dy);
  if (g.nz < 2) return FS_EARG;
  Launch3 L = launch_cells(g);
  k_keps<<<L.grid, L.block, 0, st>>>(g, a); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Vertical solid conduction on the bed T_s grid (solid_conduction_3d.py:56-127)
// ---------------------------------------------------------------------------
// cap = 1: the result is then clipped to [lo, hi] as k_clip does (the T_s
// cap that follows the conduction, spread_3d.py:3193-3196)
__global__ void k_solid_cond(GridDev g, const double* __restrict__ Ts,
                             const double* __restrict__ as, double* __restrict__ To,
                             double k_solid, double inv_rho_cp, double dt, int cap, double lo,
                             double hi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int64_t c = cidx(g, k, j, i);
  To[c] = solid_cond_cell(g, Ts, as, k, c, Ts[c], k_solid, inv_rho_cp, dt, cap, lo, hi);
}

int launch_solid_cond(const GridDev& g, const double* Ts, const double* as, double* To,
                      double k_solid, double rho_s, double cp_s, double dt, int nz_active,
                      cudaStream_t st, int cap, double lo, double hi) {
  GridDev gg = g;
  Launch3 L = launch_cells(g);
  (void)nz_active;
  k_solid_cond<<<L.grid, L.block, 0, st>>>(gg, Ts, as, To, k_solid, 1.0 / (rho_s * cp_s), dt,
                                           cap, lo, hi); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Soil columns (soil_3d.py:106-153): sequential in k per column (in-place
// Gauss-Seidel order: cell k sees the already-updated cell k-1).
// ---------------------------------------------------------------------------
__global__ void k_soil(int nsoil, int ny, int nx, double* T, const double* __restrict__ qin,
                       double dt, const double* __restrict__ sdz, const double* __restrict__ sda,
                       const double* __restrict__ sdb, double k_s, double rho_cp_inv,
                       double eps_s, double T_amb) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t n2 = (int64_t)ny * nx;
  if (q >= n2) return;
  for (int k = 0; k < nsoil; ++k) {
    double Tk = T[k * n2 + q];
    double qtop, qbot;
    if (k == 0) {
      double T2 = Tk * Tk;
      qtop = qin[q] - eps_s * 5.67e-8 * (T2 * T2);
    } else {
      qtop = k_s * (T[(k - 1) * n2 + q] - Tk) * (1.0 / sda[k]);
    }
    if (k == nsoil - 1) qbot = k_s * (Tk - T_amb) * (1.0 / sdb[k]);
    else qbot = k_s * (Tk - T[(k + 1) * n2 + q]) * (1.0 / sdb[k]);
    T[k * n2 + q] = Tk + dt * (qtop - qbot) * rho_cp_inv / sdz[k];
  }
}

int launch_soil(int nsoil, int ny, int nx, double* T, const double* qin, double dt,
                const double* sdz, const double* sda, const double* sdb, double k_s,
                double rho_s, double cp_s, double eps_s, double T_amb, cudaStream_t st) {
  int64_t n2 = (int64_t)ny * nx;
  k_soil<<<blocks_for(n2, 128), 128, 0, st>>>(nsoil, ny, nx, T, qin, dt, sdz, sda, sdb, k_s,
                                             1.0 / (rho_s * cp_s), eps_s, T_amb); fs_count_launch();
  return cuda_status();
}
