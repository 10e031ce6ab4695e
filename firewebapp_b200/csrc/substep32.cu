// Single-precision forms of the chemistry/transport sub-step kernels, for the
// mixed-precision solver (no counterpart in the reference, which is FP64
// throughout).  The ten sub-steps of an outer step (spread_3d.py:2678-3196)
// run on FP32 copies of the fields they update (T_g, Y_F, Y_O2, Y_H2O) and of
// the fields they only read (rho, u, v, w, k, eps, nu_t, the bed sources);
// the copies are made once before the first sub-step and T_g, the mass
// fractions, omega and Q_comb are widened back to FP64 after the last.  The
// solid conduction and every other operator of the step stay FP64.
//
// Each kernel restates its FP64 counterpart (transport.cu, pointwise.cu)
// expression for expression in float arithmetic: the EDC closure
// (edc.py:134-335, the same flat-order H2O-quench flag scan), the fused
// species step (species_3d.py:41-175 with the dilution sources and the O2
// clip), the turbulent diffusion sub-iteration (turbulence_3d.py:862-949)
// and the Lagrangian-branch gas-energy update (spread_3d.py:3088-3146).
#include "common.cuh"
#include "kernels.h"

// ---- conversions -------------------------------------------------------------
#define CV_MAX 16
struct CvArgs {
  const void* src[CV_MAX];
  void* dst[CV_MAX];
  int nf;
};

__global__ void k_to_f32(int64_t n, CvArgs a) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    for (int f = 0; f < a.nf; ++f) ((float*)a.dst[f])[c] = (float)((const double*)a.src[f])[c];
}

__global__ void k_to_f64(int64_t n, CvArgs a) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    for (int f = 0; f < a.nf; ++f) ((double*)a.dst[f])[c] = (double)((const float*)a.src[f])[c];
}

int launch_convert(int64_t n, int nf, const void* const* src, void* const* dst, int to_f32,
                   cudaStream_t st) {
  if (nf < 1 || nf > CV_MAX || n < 0) return FS_EARG;
  if (n == 0) return FS_OK;
  CvArgs a{};
  a.nf = nf;
  for (int f = 0; f < nf; ++f) {
    a.src[f] = src[f];
    a.dst[f] = dst[f];
  }
  unsigned nb = blocks_for(n, 256);
  if (nb > 148 * 16) nb = 148 * 16;
  if (to_f32) k_to_f32<<<nb, 256, 0, st>>>(n, a);
  else k_to_f64<<<nb, 256, 0, st>>>(n, a);
  fs_count_launch();
  return cuda_status();
}

// ---- EDC -----------------------------------------------------------------------
// The FP64 kernels' tiling: EDC_TPB threads own EDC_TILE consecutive cells,
// EDC_CPT (four) per thread, one 16-byte load per field and thread.
#define E32_BLK EDC_TILE

__device__ __forceinline__ int edc_flag_code32(float Yf, float YO2, float YH, int t) {
  if (Yf <= 1e-9f || YO2 <= 1e-9f) return -1;
  int f = 0;
  if (YH > 0.0f) {
    float fac = 1.0f - YH / 0.18f;
    if (fac < 0.0f) fac = 0.0f;
    if (fac < 0.5f) f = 1;
  }
  return (t << 1) | f;
}

__device__ __forceinline__ void e32_ld4(const float* p, int64_t c0, int64_t n, bool vec, float* v) {
  if (vec) {
    const float4 x = *reinterpret_cast<const float4*>(p + c0);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
#pragma unroll
    for (int q = 0; q < EDC_CPT; ++q) v[q] = (c0 + q < n) ? p[c0 + q] : 0.0f;
  }
}

__device__ __forceinline__ void e32_st4(float* p, int64_t c0, int64_t n, bool vec, const float* v) {
  if (vec) {
    *reinterpret_cast<float4*>(p + c0) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int q = 0; q < EDC_CPT; ++q)
      if (c0 + q < n) p[c0 + q] = v[q];
  }
}

__global__ void __launch_bounds__(EDC_TPB)
k_edc_agg32(int64_t n, const float* Yf, const float* YO, const float* YH, int vec_ok,
            signed char* agg) {
  __shared__ int sh[EDC_TPB / 32];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * E32_BLK + EDC_CPT * t;
  const bool vec = vec_ok && c0 + EDC_CPT <= n;
  float yf[EDC_CPT], yo[EDC_CPT], yh[EDC_CPT];
  e32_ld4(Yf, c0, n, vec, yf);
  e32_ld4(YO, c0, n, vec, yo);
  e32_ld4(YH, c0, n, vec, yh);
  int v = -1;
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q)
    if (c0 + q < n) v = max(v, edc_flag_code32(yf[q], yo[q], yh[q], EDC_CPT * t + q));
  const int lane = t & 31, wid = t >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (t == 0) {
    for (int w = 1; w < EDC_TPB / 32; ++w) v = max(v, sh[w]);
    agg[blockIdx.x] = (signed char)(v < 0 ? -1 : (v & 1));
  }
}

struct Edc32Args {
  const float* rho;
  float *Tg, *Yf, *YO;
  const float *kt, *et, *YH;
  float* omega;
  const signed char* carry;
  float cp_g, dt, s_stoich, HoC_eff, relax, inv_s, inv_dt;
  int extinction, nsub;
  int vec_ok;  // every array 16-byte aligned
};

// One cell's EDC update in float arithmetic (edc_cell's steps); Yf, YO2, Tg
// in place, the mean reaction rate returned.
__device__ __forceinline__ float edc_cell32(const Edc32Args& a, bool flag, float& Yf, float& YO2,
                                            float YH, float& Tg, float rho_i, float k_t,
                                            float e_t) {
  if (k_t < 1.0e-4f) k_t = 1.0e-4f;
  if (e_t < 1.0e-6f) e_t = 1.0e-6f;
  float ratio = 1.5e-5f * e_t / (k_t * k_t);
  if (ratio < 1e-30f) ratio = 1e-30f;
  const float gx = 2.1377f * sqrtf(sqrtf(ratio));
  float gamma_star = gx * (gx * gx);
  if (gamma_star > 1.0f) gamma_star = 1.0f;
  const float tau_star = 0.4083f * sqrtf(1.5e-5f / e_t);
  const float inv_tau = 1.0f / tau_star;
  const float inv_rho = 1.0f / rho_i;
  const float h = a.dt / (float)a.nsub;
  float acc = 0.0f;
  for (int sub = 0; sub < a.nsub; ++sub) {
    float omega;
    if (Yf <= 1e-9f || YO2 <= 1e-9f) {
      omega = 0.0f;
    } else {
      const float lim = YO2 * a.inv_s;
      const float Y_lim = Yf < lim ? Yf : lim;
      omega = gamma_star * (rho_i * Y_lim * inv_tau);
      if (YH > 0.0f) {
        float fac = 1.0f - YH * (1.0f / 0.18f);
        if (fac < 0.0f) fac = 0.0f;
        omega = omega * fac;
      }
    }
    bool fired = false;
    if (a.extinction && omega > 0.0f) {
      const float Yib = 1.0f - Yf - YO2;
      if (Yib > 0.88f) {
        float rs = (1.0f - Yib) * (1.0f / (1.0f - 0.88f));
        if (rs < 0.0f) rs = 0.0f;
        omega = omega * rs;
        if (rs < 0.5f) fired = true;
      }
      if (omega > 0.0f && Tg < 1200.0f) { omega = 0.0f; fired = true; }
      if (omega > 0.0f && omega * a.HoC_eff < 75000.0f) { omega = 0.0f; fired = true; }
    }
    if ((fired || flag) && Tg > 373.15f && YH > 0.0f) {
      float wb = YH * (1.0f / 0.10f);
      if (wb > 1.0f) wb = 1.0f;
      Tg = Tg - (Tg - 373.15f) * a.relax * wb;
    }
    const float dY = -omega * h * inv_rho;
    Yf = Yf + dY;
    if (Yf < 0.0f) Yf = 0.0f;
    YO2 = YO2 + a.s_stoich * dY;
    if (YO2 < 0.0f) YO2 = 0.0f;
    const float cp_mix = (1.0f - YH) * a.cp_g + YH * 2000.0f;
    Tg = Tg + omega * a.HoC_eff * h * inv_rho / cp_mix;
    if (Tg > 2400.0f) Tg = 2400.0f;
    acc += omega * h;
  }
  return a.dt > 0.0f ? acc * a.inv_dt : 0.0f;
}

__global__ void __launch_bounds__(EDC_TPB)
k_edc_main32(int64_t n, Edc32Args a) {
  __shared__ int sh[EDC_TPB / 32];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * E32_BLK + EDC_CPT * t;
  const bool vec = a.vec_ok && c0 + EDC_CPT <= n;
  float yf[EDC_CPT], yo[EDC_CPT], yh[EDC_CPT], tg[EDC_CPT], rh[EDC_CPT], kt[EDC_CPT],
      et[EDC_CPT];
  e32_ld4(a.Yf, c0, n, vec, yf);
  e32_ld4(a.YO, c0, n, vec, yo);
  e32_ld4(a.YH, c0, n, vec, yh);
  e32_ld4(a.Tg, c0, n, vec, tg);
  e32_ld4(a.rho, c0, n, vec, rh);
  e32_ld4(a.kt, c0, n, vec, kt);
  e32_ld4(a.et, c0, n, vec, et);
  const bool carry_in = a.carry[blockIdx.x] > 0;
  int code[EDC_CPT];
  int last = -1;
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q) {
    code[q] = (c0 + q < n) ? edc_flag_code32(yf[q], yo[q], yh[q], EDC_CPT * t + q) : -1;
    last = max(last, code[q]);
  }
  int run = edc_block_exclusive_max(last, sh);
  if (c0 >= n) return;
  float om[EDC_CPT];
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q) {
    run = max(run, code[q]);
    const bool flag = (run >= 0) ? (run & 1) : carry_in;
    om[q] = edc_cell32(a, flag, yf[q], yo[q], yh[q], tg[q], rh[q], kt[q], et[q]);
  }
  e32_st4(a.Yf, c0, n, vec, yf);
  e32_st4(a.YO, c0, n, vec, yo);
  e32_st4(a.Tg, c0, n, vec, tg);
  e32_st4(a.omega, c0, n, vec, om);
}

int64_t edc32_scratch_bytes(int64_t n) { return 2 * ((n + E32_BLK - 1) / E32_BLK) + 16; }

static bool al16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int launch_edc32(int64_t n, const float* rho, float* Tg, float* Yf, float* YO, const float* kt,
                 const float* et, const float* YH, float* omega, double chi_rad, double cp_g,
                 double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
                 void* scratch, cudaStream_t st) {
  if (n == 0) return FS_OK;
  const int64_t nb = (n + E32_BLK - 1) / E32_BLK;
  signed char* agg = (signed char*)scratch;
  signed char* carry = agg + nb;
  const int vec_ok = al16(rho) && al16(Tg) && al16(Yf) && al16(YO) && al16(kt) && al16(et) &&
                     al16(YH) && al16(omega);
  k_edc_agg32<<<(unsigned)nb, EDC_TPB, 0, st>>>(n, Yf, YO, YH, vec_ok, agg);
  fs_count_launch();
  int rc = launch_edc_carry((int)nb, agg, carry, st);
  if (rc != FS_OK) return rc;
  Edc32Args a{};
  a.rho = rho; a.Tg = Tg; a.Yf = Yf; a.YO = YO; a.kt = kt; a.et = et; a.YH = YH;
  a.omega = omega; a.carry = carry;
  a.cp_g = (float)cp_g; a.dt = (float)dt; a.s_stoich = (float)s_stoich;
  a.inv_s = (float)(1.0 / s_stoich);
  a.inv_dt = dt > 0.0 ? (float)(1.0 / dt) : 0.0f;
  a.HoC_eff = (float)(hoc_J * (1.0 - chi_rad));
  a.nsub = n_substeps > 1 ? n_substeps : 1;
  a.relax = (float)(1.0 - exp(-(dt / (double)a.nsub) / 0.5));
  a.extinction = extinction;
  a.vec_ok = vec_ok;
  k_edc_main32<<<(unsigned)nb, EDC_TPB, 0, st>>>(n, a);
  fs_count_launch();
  return cuda_status();
}

// ---- species step ------------------------------------------------------------
// minmod and the MUSCL face value in float (the FP64 helpers' forms)
__device__ __forceinline__ float minmod32(float a, float b) {
  const float m = copysignf(fminf(fabsf(a), fabsf(b)), a);
  return (a * b <= 0.0f) ? 0.0f : m;
}

__device__ __forceinline__ float muscl_face32(float pim1, float pi, float pip1, float pip2,
                                              float uf) {
  const bool up = uf >= 0.0f;
  const float m = minmod32(pip1 - pi, up ? pi - pim1 : pip2 - pip1);
  const float base = up ? pi : pip1;
  const float half = up ? 0.5f : -0.5f;
  return base + half * m;
}

#define S32_TX 32
#define S32_TY 8
struct Species32Args {
  const float* Y[3];
  float* Yo[3];
  float Y_inlet[3];
  const float *Sp, *Sd, *rho, *u, *v, *w;
  float dt, D, inv_dx, inv_dy, inv_dx2, inv_dy2, o2_cap;
};

__global__ void __launch_bounds__(S32_TX * S32_TY, 4) k_species32(GridDev g, Species32Args a) {
  __shared__ float rk[4];  // 1/da, 1/db, 1/dz, 1/hz of the block's level
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int k = blockIdx.z;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const double da = g.da[k], db = g.db[k];
    rk[0] = (float)(1.0 / da);
    rk[1] = (float)(1.0 / db);
    rk[2] = (float)(1.0 / g.dz[k]);
    rk[3] = (float)(1.0 / (0.5 * (da + db)));
  }
  __syncthreads();
  const int i = blockIdx.x * S32_TX + threadIdx.x;
  const int j = blockIdx.y * S32_TY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int64_t crow = (int64_t)k * sz + i;
  const int64_t c = crow + (int64_t)j * sy;
  const int jm2 = wrapj(j - 2, ny), jm1 = wrapj(j - 1, ny);
  const int jp1 = wrapj(j + 1, ny), jp2 = wrapj(j + 2, ny);
  const float ui = a.u[c], vi = a.v[c], wi = a.w[c];
  const float inv_rho = 1.0f / a.rho[c];
  const float inv_d_above = rk[0], inv_d_below = rk[1], inv_dz_k = rk[2], inv_hz = rk[3];
  const float sp = a.Sp[c], sd = a.Sd[c];
  const float stot = sp + sd;
  const bool mx = (i >= 2 && i <= nx - 3);
  const bool mz = (k >= 2 && k <= nz - 3);
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const float* __restrict__ Y = a.Y[s];
    const float Yi = Y[c];
    const float YL_x = (i == 0) ? a.Y_inlet[s] : Y[c - 1];
    const float YR_x = (i == nx - 1) ? Yi : Y[c + 1];
    const float YL_z = (k == 0) ? Yi : Y[c - sz];
    const float YR_z = (k == nz - 1) ? Yi : Y[c + sz];
    float flux_x, flux_z;
    if (mx) {
      const float fxp = muscl_face32(Y[c - 1], Yi, Y[c + 1], Y[c + 2], ui);
      const float fxm = muscl_face32(Y[c - 2], Y[c - 1], Yi, Y[c + 1], ui);
      flux_x = ui * (fxp - fxm) * a.inv_dx;
    } else {
      flux_x = (ui >= 0.0f) ? ui * (Yi - YL_x) * a.inv_dx : ui * (YR_x - Yi) * a.inv_dx;
    }
    const float Yjm2 = Y[crow + jm2 * sy], Yjm1 = Y[crow + jm1 * sy];
    const float Yjp1 = Y[crow + jp1 * sy], Yjp2 = Y[crow + jp2 * sy];
    const float fyp = muscl_face32(Yjm1, Yi, Yjp1, Yjp2, vi);
    const float fym = muscl_face32(Yjm2, Yjm1, Yi, Yjp1, vi);
    const float flux_y = vi * (fyp - fym) * a.inv_dy;
    if (mz) {
      const float fzp = muscl_face32(Y[c - sz], Yi, Y[c + sz], Y[c + 2 * sz], wi);
      const float fzm = muscl_face32(Y[c - 2 * sz], Y[c - sz], Yi, Y[c + sz], wi);
      flux_z = wi * (fzp - fzm) * inv_hz;
    } else {
      flux_z = (wi >= 0.0f) ? wi * (Yi - YL_z) * inv_d_below : wi * (YR_z - Yi) * inv_d_above;
    }
    const float adv = -(flux_x + flux_y + flux_z);
    const float d2x = (YR_x - 2.0f * Yi + YL_x) * a.inv_dx2;
    const float d2y = (Yjp1 - 2.0f * Yi + Yjm1) * a.inv_dy2;
    const float d2z = ((YR_z - Yi) * inv_d_above - (Yi - YL_z) * inv_d_below) * inv_dz_k;
    const float diff = a.D * (d2x + d2y + d2z);
    const float S = (s == 0) ? sp - Yi * stot : ((s == 1) ? -(Yi * stot) : sd - Yi * stot);
    float nw = Yi + (adv + diff + S * inv_rho) * a.dt;
    if (nw < 0.0f) nw = 0.0f;
    else if (nw > 1.0f) nw = 1.0f;
    if (s == 1) {
      if (nw > a.o2_cap) nw = a.o2_cap;
      if (nw < 0.0f) nw = 0.0f;
    }
    a.Yo[s][c] = nw;
  }
}

int launch_species_step32(const GridDev& g, const float* const* Y, float* const* Yo,
                          const float* Sp, const float* Sd, const double* Y_inlet,
                          const float* rho, const float* u, const float* v, const float* w,
                          double dt, double D, double o2_cap, cudaStream_t st) {
  Species32Args a{};
  for (int s = 0; s < 3; ++s) {
    a.Y[s] = Y[s];
    a.Yo[s] = Yo[s];
    a.Y_inlet[s] = (float)Y_inlet[s];
  }
  a.Sp = Sp; a.Sd = Sd; a.rho = rho; a.u = u; a.v = v; a.w = w;
  a.dt = (float)dt; a.D = (float)D; a.o2_cap = (float)o2_cap;
  a.inv_dx = (float)(1.0 / g.dx); a.inv_dy = (float)(1.0 / g.dy);
  a.inv_dx2 = (float)(1.0 / (g.dx * g.dx)); a.inv_dy2 = (float)(1.0 / (g.dy * g.dy));
  const dim3 nb((g.nx + S32_TX - 1) / S32_TX, (g.ny + S32_TY - 1) / S32_TY, g.nz);
  k_species32<<<nb, dim3(S32_TX, S32_TY), 0, st>>>(g, a);
  fs_count_launch();
  return cuda_status();
}

// ---- turbulent diffusion -----------------------------------------------------
struct Diff32Args {
  const float* f[4];
  float* fo[4];
  float lo[4], hi[4];
  int clip;
};

// A block owns a 32 x 8 tile and marches up a chunk of z-levels (the FP64
// kernel's scheme): the column's k-1, k, k+1 values stay in registers and
// level k+2 is requested while level k computes.
#define TD32_MAXKZ 64
template <int NF>
__global__ void __launch_bounds__(S32_TX * S32_TY, 4)
    k_turb_diff32(GridDev g, Diff32Args a, const float* __restrict__ nu_t, float inv_sc,
                  float dt_sub, float inv_dx2, float inv_dy2, int kz) {
  __shared__ float rk[TD32_MAXKZ][3];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  const int k0 = blockIdx.z * kz;
  const int k1 = min(nz, k0 + kz);
  const int tid = threadIdx.y * S32_TX + threadIdx.x;
  for (int q = tid; q < k1 - k0; q += S32_TX * S32_TY) {
    rk[q][0] = (float)(1.0 / g.dz[k0 + q]);
    rk[q][1] = (float)(1.0 / g.da[k0 + q]);
    rk[q][2] = (float)(1.0 / g.db[k0 + q]);
  }
  __syncthreads();
  const int i = blockIdx.x * S32_TX + threadIdx.x;
  const int j = blockIdx.y * S32_TY + threadIdx.y;
  if (i >= nx || j >= ny || k0 >= nz) return;
  const int64_t col = (int64_t)j * sy + i;
  const int64_t cjp0 = (int64_t)wrapj(j + 1, ny) * sy + i, cjm0 = (int64_t)wrapj(j - 1, ny) * sy + i;
  float fL[NF], fC[NF], fN[NF];
#pragma unroll
  for (int s = 0; s < NF; ++s) {
    fC[s] = a.f[s][(int64_t)k0 * sz + col];
    fL[s] = (k0 == 0) ? fC[s] : a.f[s][(int64_t)(k0 - 1) * sz + col];
    fN[s] = (k0 == nz - 1) ? fC[s] : a.f[s][(int64_t)(k0 + 1) * sz + col];
  }
  float nu_c = nu_t[(int64_t)k0 * sz + col];
  for (int k = k0; k < k1; ++k) {
    const int64_t ks = (int64_t)k * sz;
    const int64_t c = ks + col;
    const bool more = k + 1 < k1;
    float nu_n = 0.0f, fNN[NF];
    if (more) nu_n = nu_t[c + sz];
#pragma unroll
    for (int s = 0; s < NF; ++s)
      fNN[s] = (more && k + 2 < nz) ? a.f[s][c + 2 * sz] : fN[s];
    const float D_t = nu_c * inv_sc;
    const float r0 = rk[k - k0][0], r1 = rk[k - k0][1], r2 = rk[k - k0][2];
#pragma unroll
    for (int s = 0; s < NF; ++s) {
      const float* __restrict__ f = a.f[s];
      const float fc = fC[s];
      const float fxL = (i == 0) ? fc : f[c - 1];
      const float fxR = (i == nx - 1) ? fc : f[c + 1];
      const float fzL = fL[s];
      const float fzR = fN[s];
      const float d2x = (fxR - 2.0f * fc + fxL) * inv_dx2;
      const float d2y = (f[ks + cjp0] - 2.0f * fc + f[ks + cjm0]) * inv_dy2;
      const float d2z = ((fzR - fc) * r1 - (fc - fzL) * r2) * r0;
      float nv = fc + D_t * (d2x + d2y + d2z) * dt_sub;
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

int launch_turb_diff32(const GridDev& g, int nfield, const float* const* f, float* const* fo,
                       const float* nu_t, double sc_t, double dt_sub, int clip, const double* lo,
                       const double* hi, cudaStream_t st) {
  if (nfield != 1 && nfield != 3) return FS_EARG;
  Diff32Args a{};
  a.clip = clip;
  for (int s = 0; s < nfield; ++s) {
    a.f[s] = f[s];
    a.fo[s] = fo[s];
    a.lo[s] = clip ? (float)lo[s] : 0.0f;
    a.hi[s] = clip ? (float)hi[s] : 0.0f;
  }
  // z-chunks: about six blocks per SM of the 148, at least four levels each
  const int tiles = ((g.nx + S32_TX - 1) / S32_TX) * ((g.ny + S32_TY - 1) / S32_TY);
  int chunks = (6 * 148 + tiles - 1) / tiles;
  if (chunks > g.nz) chunks = g.nz;
  if (chunks < 1) chunks = 1;
  int kz = (g.nz + chunks - 1) / chunks;
  if (kz < 4) kz = g.nz < 4 ? g.nz : 4;
  if (kz > TD32_MAXKZ) kz = TD32_MAXKZ;
  chunks = (g.nz + kz - 1) / kz;
  const dim3 nb((g.nx + S32_TX - 1) / S32_TX, (g.ny + S32_TY - 1) / S32_TY, chunks);
  const dim3 tb(S32_TX, S32_TY);
  const float ix2 = (float)(1.0 / (g.dx * g.dx)), iy2 = (float)(1.0 / (g.dy * g.dy));
  if (nfield == 1)
    k_turb_diff32<1><<<nb, tb, 0, st>>>(g, a, nu_t, (float)(1.0 / sc_t), (float)dt_sub, ix2, iy2,
                                        kz);
  else
    k_turb_diff32<3><<<nb, tb, 0, st>>>(g, a, nu_t, (float)(1.0 / sc_t), (float)dt_sub, ix2, iy2,
                                        kz);
  fs_count_launch();
  return cuda_status();
}

// ---- gas-energy update -------------------------------------------------------
struct Gas32Args {
  float* Tg;
  const float *rho, *YH, *Sp, *Sd, *Qgc;
  const double *Ts, *qrg;  // T_s (FP64 solid state) and the DOM's gas source
  float* Qcomb_out;
  float dt_sub, T_amb, q_drip_gas;
  int drip_on, n_z_bed, i_src0, i_src1;
};

__global__ void k_gas_update32(GridDev g, Gas32Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const int64_t c = cidx(g, k, j, i);
  float qc = 0.0f;
  if (a.drip_on && k < a.n_z_bed && i >= a.i_src0 && i < a.i_src1) qc = qc + a.q_drip_gas;
  qc = qc + (float)(a.qrg[c] / g.dz[k]);
  const float T = a.Tg[c];
  const float YH = a.YH[c];
  const float cp = (1.0f - YH) * 1100.0f + YH * 2000.0f;
  float d1 = T - (float)a.Ts[c];
  if (!(d1 >= 0.0f)) d1 = (d1 != d1) ? d1 : 0.0f;
  float d2 = T - 373.15f;
  if (!(d2 >= 0.0f)) d2 = (d2 != d2) ? d2 : 0.0f;
  const float debit = (a.Sp[c] * d1 + a.Sd[c] * d2) * 2000.0f;
  const float r = a.rho[c];
  const float rm = (r >= 1.0e-3f || r != r) ? r : 1.0e-3f;
  float Tn = T + (qc - a.Qgc[c] - debit) * (a.dt_sub / (rm * cp));
  if (Tn < a.T_amb) Tn = a.T_amb;
  a.Tg[c] = Tn;
  if (a.Qcomb_out) a.Qcomb_out[c] = qc;
}

int launch_gas_update32(const GridDev& g, float* Tg, const float* rho, const float* YH,
                        const double* Ts, const float* Sp, const float* Sd, const float* Qgc,
                        const double* qrg, float* Qcomb_out, double dt_sub, double T_amb,
                        double h_bed, int drip_on, int n_z_bed, int i_src0, int i_src1,
                        cudaStream_t st) {
  Gas32Args a{};
  a.Tg = Tg; a.rho = rho; a.YH = YH; a.Ts = Ts; a.Sp = Sp; a.Sd = Sd; a.Qgc = Qgc; a.qrg = qrg;
  a.Qcomb_out = Qcomb_out;
  a.dt_sub = (float)dt_sub; a.T_amb = (float)T_amb;
  const double q_drip = 30000.0 / (h_bed > 1e-3 ? h_bed : 1e-3);
  a.q_drip_gas = (float)((1.0 - 0.80) * q_drip);
  a.drip_on = drip_on; a.n_z_bed = n_z_bed; a.i_src0 = i_src0; a.i_src1 = i_src1;
  Launch3 L = launch_cells(g);
  k_gas_update32<<<L.grid, L.block, 0, st>>>(g, a);
  fs_count_launch();
  return cuda_status();
}

// ---- clip ------------------------------------------------------------------------
__global__ void k_clip32(int64_t n, float* f, float lo, float hi) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  float x = f[c];
  if (x > hi) x = hi;
  if (x < lo) x = lo;
  f[c] = x;
}

int launch_clip32(int64_t n, float* f, double lo, double hi, cudaStream_t st) {
  if (n == 0) return FS_OK;
  k_clip32<<<blocks_for(n, 256), 256, 0, st>>>(n, f, (float)lo, (float)hi);
  fs_count_launch();
  return cuda_status();
}
