// Pointwise kernels of the Tier-3 step: EDC chemistry, the Lagrangian-branch
// gas-energy update, EoS, caps and the step's max reductions.
#include "common.cuh"
#include "kernels.h"

// ---------------------------------------------------------------------------
// EDC (chemistry_closures/edc.py:134-335 step_chemistry_ode_edc, n_substeps=1)
//
// The reference assigns the H2O-quench flag `_h2o_quench_substantial` only in
// the branch taken when Y_F > 1e-9 and Y_O2 > 1e-9 (edc.py:223).  Cells that
// skip that branch reuse the value left by the previously visited cell, which
// with one thread is the previous cell in flat k-j-i order (initially False).
// The flag gates the wet-bulb relaxation of T_g.  To reproduce that order on
// the GPU the flag is resolved by a flat-order "last assigned value" scan over
// tiles of EDC_TILE cells:
//   pass 1: per tile, the last assigned flag (or none);
//   pass 2: one block carries the flag across tiles;
//   pass 3: in-tile scan + carry, then the EDC update itself.
// Passes 1 and 3 give each thread EDC_CPT consecutive cells and issue all of
// a thread's loads before the scan's barrier, so the block's memory requests
// are in flight together instead of after it.
// ---------------------------------------------------------------------------
#define EDC_BLK EDC_TILE

__device__ __forceinline__ int edc_flag_code(double Yf, double YO2, double YH, int t) {
  // -1: flag not assigned in this cell; else (t << 1) | flag
  if (Yf <= 1e-9 || YO2 <= 1e-9) return -1;
  int f = 0;
  if (YH > 0.0) {
    double fac = 1.0 - YH / 0.18;
    if (fac < 0.0) fac = 0.0;
    if (fac < 0.5) f = 1;
  }
  return (t << 1) | f;
}

// EDC_CPT consecutive values from p + c0: two 16-byte loads when `vec` (the
// four cells are all inside the array and p is 16-byte aligned), else
// element by element with 0 past n.
__device__ __forceinline__ void edc_ld4(const double* p, int64_t c0, int64_t n, bool vec,
                                        double* v) {
  if (vec) {
    const double2 x = *reinterpret_cast<const double2*>(p + c0);
    const double2 y = *reinterpret_cast<const double2*>(p + c0 + 2);
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
  } else {
#pragma unroll
    for (int q = 0; q < EDC_CPT; ++q) v[q] = (c0 + q < n) ? p[c0 + q] : 0.0;
  }
}

__device__ __forceinline__ void edc_st4(double* p, int64_t c0, int64_t n, bool vec,
                                        const double* v) {
  if (vec) {
    *reinterpret_cast<double2*>(p + c0) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(p + c0 + 2) = make_double2(v[2], v[3]);
  } else {
#pragma unroll
    for (int q = 0; q < EDC_CPT; ++q)
      if (c0 + q < n) p[c0 + q] = v[q];
  }
}

__global__ void __launch_bounds__(EDC_TPB)
k_edc_agg(int64_t n, const double* Yf, const double* YO, const double* YH, int vec_ok,
          signed char* agg) {
  __shared__ int sh[EDC_TPB / 32];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * EDC_TILE + EDC_CPT * t;
  const bool vec = vec_ok && c0 + EDC_CPT <= n;
  double yf[EDC_CPT], yo[EDC_CPT], yh[EDC_CPT];
  edc_ld4(Yf, c0, n, vec, yf);
  edc_ld4(YO, c0, n, vec, yo);
  edc_ld4(YH, c0, n, vec, yh);
  int v = -1;
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q)
    if (c0 + q < n) v = max(v, edc_flag_code(yf[q], yo[q], yh[q], EDC_CPT * t + q));
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

// Carry of the last assigned flag into every block: each thread folds a
// contiguous run of blocks, a block-wide max-scan of (block << 1 | flag)
// gives every run its incoming flag, then each thread writes its run.
#define EDC_CARRY_THREADS 1024
__global__ void __launch_bounds__(EDC_CARRY_THREADS)
k_edc_carry(int nb, const signed char* agg, signed char* carry, const signed char* carry_in) {
  __shared__ int incl[EDC_CARRY_THREADS];
  __shared__ int wsum[32];
  const int t = threadIdx.x;
  const int per = (nb + EDC_CARRY_THREADS - 1) / EDC_CARRY_THREADS;
  const int b0 = t * per;
  const int b1 = min(nb, b0 + per);
  int last = -1;
  for (int b = b0; b < b1; ++b)
    if (agg[b] >= 0) last = (b << 1) | agg[b];
  const int lane = t & 31, wid = t >> 5;
  int v = last;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, y);
  }
  if (lane == 31) wsum[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w = max(w, y);
    }
    wsum[lane] = w;
  }
  __syncthreads();
  if (wid > 0) v = max(v, wsum[wid - 1]);
  incl[t] = v;
  __syncthreads();
  const int before = t > 0 ? incl[t - 1] : -1;
  signed char cur = before >= 0 ? (signed char)(before & 1) : (carry_in ? carry_in[0] : 0);
  for (int b = b0; b < b1; ++b) {
    carry[b] = cur;
    if (agg[b] >= 0) cur = agg[b];
  }
}

int launch_edc_carry(int nb, const signed char* agg, signed char* carry, cudaStream_t st) {
  k_edc_carry<<<1, EDC_CARRY_THREADS, 0, st>>>(nb, agg, carry, nullptr);
  fs_count_launch();
  return cuda_status();
}

struct EdcArgs {
  const double* rho;
  double *Tg, *Yf, *YO;
  const double *kt, *et, *YH;
  double* omega;
  const signed char* carry;
  double chi_rad, cp_g, dt, s_stoich, HoC_eff, relax;
  // reciprocals of the constant divisors (1/s_stoich, 1/dt); the divisions
  // by them, by rho and by tau* are multiplications
  double inv_s, inv_dt;
  int extinction, nsub;
  int vec_ok;  // every array 16-byte aligned
};

// One cell's EDC update (edc.py:180-330 for one cell, `flag` the quench flag
// it sees on entry); Yf, YO2, Tg updated in place, the mean reaction rate
// returned.
__device__ __forceinline__ double edc_cell(const EdcArgs& a, bool flag, double& Yf, double& YO2,
                                           double YH, double& Tg, double rho_i, double k_t,
                                           double e_t) {
  if (k_t < 1.0e-4) k_t = 1.0e-4;
  if (e_t < 1.0e-6) e_t = 1.0e-6;
  double ratio = 1.5e-5 * e_t / (k_t * k_t);
  if (ratio < 1e-30) ratio = 1e-30;
  // ratio**0.25 as two square roots: each is correctly rounded, so the
  // fourth root is within about one ulp of the correctly rounded power, the
  // accuracy of a libm pow, at a fraction of pow's cost
  double gx = 2.1377 * sqrt(sqrt(ratio));
  double gamma_star = gx * (gx * gx);
  if (gamma_star > 1.0) gamma_star = 1.0;
  double tau_star = 0.4083 * sqrt(1.5e-5 / e_t);
  // Division costs a Newton sequence here, so the constant and per-cell
  // divisors become one reciprocal each: every quotient below is then within
  // an ulp or two of the reference's (the kernel is instruction-bound).
  const double inv_tau = 1.0 / tau_star;
  const double inv_rho = 1.0 / rho_i;
  const double h = a.dt / (double)a.nsub;
  double acc = 0.0;
  for (int sub = 0; sub < a.nsub; ++sub) {
    double omega;
    if (Yf <= 1e-9 || YO2 <= 1e-9) {
      omega = 0.0;
    } else {
      double lim = YO2 * a.inv_s;
      double Y_lim = Yf < lim ? Yf : lim;
      double omega_fine = rho_i * Y_lim * inv_tau;
      omega = gamma_star * omega_fine;
      if (YH > 0.0) {
        double fac = 1.0 - YH * (1.0 / 0.18);
        if (fac < 0.0) fac = 0.0;
        omega = omega * fac;
      }
    }
    bool fired = false;
    if (a.extinction && omega > 0.0) {
      double Yib = 1.0 - Yf - YO2;
      if (Yib > 0.88) {
        double rs = (1.0 - Yib) * (1.0 / (1.0 - 0.88));
        if (rs < 0.0) rs = 0.0;
        omega = omega * rs;
        if (rs < 0.5) fired = true;
      }
      if (omega > 0.0 && Tg < 1200.0) { omega = 0.0; fired = true; }
      if (omega > 0.0) {
        double Q_rate = omega * a.HoC_eff;
        if (Q_rate < 75000.0) { omega = 0.0; fired = true; }
      }
    }
    if ((fired || flag) && Tg > 373.15) {
      if (YH > 0.0) {
        double wb = YH * (1.0 / 0.10);
        if (wb > 1.0) wb = 1.0;
        double dT_wb = (Tg - 373.15) * a.relax * wb;
        Tg = Tg - dT_wb;
      }
    }
    double dY = -omega * h * inv_rho;
    Yf = Yf + dY;
    if (Yf < 0.0) Yf = 0.0;
    YO2 = YO2 + a.s_stoich * dY;
    if (YO2 < 0.0) YO2 = 0.0;
    double cp_mix = (1.0 - YH) * a.cp_g + YH * 2000.0;
    Tg = Tg + omega * a.HoC_eff * h * inv_rho / cp_mix;
    if (Tg > 2400.0) Tg = 2400.0;
    acc += omega * h;
  }
  return a.dt > 0.0 ? acc * a.inv_dt : 0.0;
}

__global__ void __launch_bounds__(EDC_TPB)
k_edc_main(int64_t n, EdcArgs a) {
  __shared__ int sh[EDC_TPB / 32];
  const int t = threadIdx.x;
  const int64_t c0 = (int64_t)blockIdx.x * EDC_TILE + EDC_CPT * t;
  const bool vec = a.vec_ok && c0 + EDC_CPT <= n;
  // every input of the thread's cells is requested before the scan's barrier
  double yf[EDC_CPT], yo[EDC_CPT], yh[EDC_CPT], tg[EDC_CPT], rh[EDC_CPT], kt[EDC_CPT],
      et[EDC_CPT];
  edc_ld4(a.Yf, c0, n, vec, yf);
  edc_ld4(a.YO, c0, n, vec, yo);
  edc_ld4(a.YH, c0, n, vec, yh);
  edc_ld4(a.Tg, c0, n, vec, tg);
  edc_ld4(a.rho, c0, n, vec, rh);
  edc_ld4(a.kt, c0, n, vec, kt);
  edc_ld4(a.et, c0, n, vec, et);
  const bool carry_in = a.carry[blockIdx.x] > 0;
  int code[EDC_CPT];
  int last = -1;
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q) {
    code[q] = (c0 + q < n) ? edc_flag_code(yf[q], yo[q], yh[q], EDC_CPT * t + q) : -1;
    last = max(last, code[q]);
  }
  int run = edc_block_exclusive_max(last, sh);
  if (c0 >= n) return;
  double om[EDC_CPT];
#pragma unroll
  for (int q = 0; q < EDC_CPT; ++q) {
    run = max(run, code[q]);
    const bool flag = (run >= 0) ? (run & 1) : carry_in;
    om[q] = edc_cell(a, flag, yf[q], yo[q], yh[q], tg[q], rh[q], kt[q], et[q]);
  }
  edc_st4(a.Yf, c0, n, vec, yf);
  edc_st4(a.YO, c0, n, vec, yo);
  edc_st4(a.Tg, c0, n, vec, tg);
  edc_st4(a.omega, c0, n, vec, om);
}

int edc_scratch_bytes(int64_t n) {
  int64_t nb = (n + EDC_BLK - 1) / EDC_BLK;
  return (int)(2 * nb + 16);
}

static bool al16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int launch_edc(int64_t n, const double* rho, double* Tg, double* Yf, double* YO, const double* kt,
               const double* et, const double* YH, double* omega, double chi_rad, double cp_g,
               double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
               void* scratch, cudaStream_t st) {
  int64_t nb = (n + EDC_BLK - 1) / EDC_BLK;
  signed char* agg = (signed char*)scratch;
  signed char* carry = agg + nb;
  const int vec_ok = al16(rho) && al16(Tg) && al16(Yf) && al16(YO) && al16(kt) && al16(et) &&
                     al16(YH) && al16(omega);
  k_edc_agg<<<(unsigned)nb, EDC_TPB, 0, st>>>(n, Yf, YO, YH, vec_ok, agg); fs_count_launch();
  k_edc_carry<<<1, EDC_CARRY_THREADS, 0, st>>>((int)nb, agg, carry, nullptr); fs_count_launch();
  EdcArgs a{};
  a.rho = rho; a.Tg = Tg; a.Yf = Yf; a.YO = YO; a.kt = kt; a.et = et; a.YH = YH;
  a.omega = omega; a.carry = carry;
  a.chi_rad = chi_rad; a.cp_g = cp_g; a.dt = dt; a.s_stoich = s_stoich;
  a.inv_s = 1.0 / s_stoich;
  a.inv_dt = dt > 0.0 ? 1.0 / dt : 0.0;
  a.HoC_eff = hoc_J * (1.0 - chi_rad);
  a.nsub = n_substeps > 1 ? n_substeps : 1;
  a.relax = 1.0 - exp(-(dt / (double)a.nsub) / 0.5);
  a.extinction = extinction;
  a.vec_ok = vec_ok;
  k_edc_main<<<(unsigned)nb, EDC_TPB, 0, st>>>(n, a); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Lagrangian-branch gas-energy update (spread_3d.py:3088-3146):
//   Q_comb = drip (20 % of 30 kW/m^2 / h_bed in source bed cells during the
//   ignition window, spread_3d.py:2916-2957) + q_rad_gas / dz
//   T_g += (Q_comb - Q_g_conv - vapour debit) dt_sub / (max(rho,1e-3) cp_mix)
//   T_g = max(T_g, T_amb)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long dkey(double x) {
  long long b = __double_as_longlong(x);
  return b >= 0 ? ((unsigned long long)b ^ 0x8000000000000000ull) : ~(unsigned long long)b;
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  long long b = (k & 0x8000000000000000ull) ? (long long)(k ^ 0x8000000000000000ull)
                                            : (long long)(~k);
  return __longlong_as_double(b);
}

struct GasArgs {
  double* Tg;
  const double *rho, *YH, *Ts, *Sp, *Sd, *Qgc, *qrg;
  double* Qcomb_out;           // optional
  unsigned long long* qc_max;  // optional
  double dt_sub, T_amb, q_drip_gas;
  int drip_on, n_z_bed, i_src0, i_src1;
};

// One cell of the update; T_s = Ts[c].  Returns the new T_g and the cell's
// Q_comb in *qc (the caller stores both, after every load of the cell).
__device__ __forceinline__ double gas_update_cell(const GridDev& g, const GasArgs& a, int k, int i,
                                                  int64_t c, double T_s, double* qc_out) {
  double qc = 0.0;
  if (a.drip_on && k < a.n_z_bed && i >= a.i_src0 && i < a.i_src1) qc = qc + a.q_drip_gas;
  qc = qc + a.qrg[c] / g.dz[k];
  double T = a.Tg[c];
  double YH = a.YH[c];
  double cp = (1.0 - YH) * 1100.0 + YH * 2000.0;
  double d1 = T - T_s;
  if (!(d1 >= 0.0)) d1 = (d1 != d1) ? d1 : 0.0;
  double d2 = T - 373.15;
  if (!(d2 >= 0.0)) d2 = (d2 != d2) ? d2 : 0.0;
  double debit = (a.Sp[c] * d1 + a.Sd[c] * d2) * 2000.0;
  double r = a.rho[c];
  double rm = (r >= 1.0e-3 || r != r) ? r : 1.0e-3;
  double ginv = a.dt_sub / (rm * cp);
  double Tn = T + (qc - a.Qgc[c] - debit) * ginv;
  if (Tn < a.T_amb) Tn = a.T_amb;
  *qc_out = qc;
  return Tn;
}

__global__ void k_gas_update(GridDev g, GasArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  int64_t c = cidx(g, k, j, i);
  double qc;
  const double Tn = gas_update_cell(g, a, k, i, c, a.Ts[c], &qc);
  a.Tg[c] = Tn;
  if (a.Qcomb_out) a.Qcomb_out[c] = qc;
  if (a.qc_max) atomicMax(a.qc_max, dkey(qc));
}

// The gas-energy update and the capped solid conduction of the same
// sub-step in one pass (both read the old T_s; neither reads what the other
// writes): T_s is read once per cell, one launch replaces two, and every
// load of a cell is issued before its stores.
struct SolidArgs {
  const double* as;
  double* To;
  double k_solid, inv_rho_cp, lo, hi;
};

__global__ void k_gas_solid(GridDev g, GasArgs a, SolidArgs b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  int64_t c = cidx(g, k, j, i);
  const double T_s = a.Ts[c];
  double qc;
  const double Tn = gas_update_cell(g, a, k, i, c, T_s, &qc);
  const double To = solid_cond_cell(g, a.Ts, b.as, k, c, T_s, b.k_solid, b.inv_rho_cp, a.dt_sub,
                                    1, b.lo, b.hi);
  a.Tg[c] = Tn;
  if (a.Qcomb_out) a.Qcomb_out[c] = qc;
  b.To[c] = To;
}

int launch_gas_solid(const GridDev& g, double* Tg, const double* rho, const double* YH,
                     const double* Ts, const double* Sp, const double* Sd, const double* Qgc,
                     const double* qrg, double* Qcomb_out, double dt_sub, double T_amb,
                     double h_bed, int drip_on, int n_z_bed, int i_src0, int i_src1,
                     const double* as, double* Ts_out, double k_solid, double rho_s, double cp_s,
                     double lo, double hi, cudaStream_t st) {
  GasArgs a{};
  a.Tg = Tg; a.rho = rho; a.YH = YH; a.Ts = Ts; a.Sp = Sp; a.Sd = Sd; a.Qgc = Qgc; a.qrg = qrg;
  a.Qcomb_out = Qcomb_out; a.qc_max = nullptr;
  a.dt_sub = dt_sub; a.T_amb = T_amb;
  double q_drip = 30000.0 / (h_bed > 1e-3 ? h_bed : 1e-3);
  a.q_drip_gas = (1.0 - 0.80) * q_drip;
  a.drip_on = drip_on; a.n_z_bed = n_z_bed; a.i_src0 = i_src0; a.i_src1 = i_src1;
  SolidArgs b{as, Ts_out, k_solid, 1.0 / (rho_s * cp_s), lo, hi};
  Launch3 L = launch_cells(g);
  k_gas_solid<<<L.grid, L.block, 0, st>>>(g, a, b); fs_count_launch();
  return cuda_status();
}

int launch_gas_update(const GridDev& g, double* Tg, const double* rho, const double* YH,
                      const double* Ts, const double* Sp, const double* Sd, const double* Qgc,
                      const double* qrg, double* Qcomb_out, unsigned long long* qc_max,
                      double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                      int i_src0, int i_src1, cudaStream_t st) {
  GasArgs a{};
  a.Tg = Tg; a.rho = rho; a.YH = YH; a.Ts = Ts; a.Sp = Sp; a.Sd = Sd; a.Qgc = Qgc; a.qrg = qrg;
  a.Qcomb_out = Qcomb_out; a.qc_max = qc_max;
  a.dt_sub = dt_sub; a.T_amb = T_amb;
  double q_drip = 30000.0 / (h_bed > 1e-3 ? h_bed : 1e-3);
  a.q_drip_gas = (1.0 - 0.80) * q_drip;
  a.drip_on = drip_on; a.n_z_bed = n_z_bed; a.i_src0 = i_src0; a.i_src1 = i_src1;
  Launch3 L = launch_cells(g);
  k_gas_update<<<L.grid, L.block, 0, st>>>(g, a); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Start-of-step bookkeeping (spread_3d.py:1984-2050):
//   rho_prev = rho; rho = P0 / (R_air max(T_g, T_amb)); Y_O2[:, :, 0] = 0.232
// and the closing EoS (spread_3d.py:3440) with prev == null.
// ---------------------------------------------------------------------------
__global__ void k_eos(GridDev g, double* rho, double* rho_prev, const double* __restrict__ Tg,
                      double* YO, double P0, double R_air, double T_amb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  int64_t c = cidx(g, k, j, i);
  if (rho_prev) rho_prev[c] = rho[c];
  double T = Tg[c];
  double Tm = (T >= T_amb || T != T) ? T : T_amb;
  rho[c] = P0 / (R_air * Tm);
  if (YO && i == 0) YO[c] = 0.232;
}

int launch_eos(const GridDev& g, double* rho, double* rho_prev, const double* Tg, double* YO,
               double P0, double R_air, double T_amb, cudaStream_t st) {
  Launch3 L = launch_cells(g);
  k_eos<<<L.grid, L.block, 0, st>>>(g, rho, rho_prev, Tg, YO, P0, R_air, T_amb); fs_count_launch();
  return cuda_status();
}

// Divergence target of the pressure projection (spread_3d.py:2300-2317, the
// unweighted form): ((S_pyro + S_drying) - (rho - rho_prev)/dt) / max(rho, 0.1),
// with S_pyro = copy of the bed's pyrolysis source plus its drying source
// (spread_3d.py:2147-2148).  np.maximum keeps a NaN rho.
__global__ void k_div_target(int64_t n, const double* __restrict__ rho,
                             const double* __restrict__ rho_prev, const double* __restrict__ Sp,
                             const double* __restrict__ Sd, double dt, double* __restrict__ out) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double r = rho[c];
  const double s = Sp[c] + Sd[c];
  const double drho = (r - rho_prev[c]) / dt;
  const double rs = (r != r) ? r : (r > 0.1 ? r : 0.1);
  out[c] = (s - drho) / rs;
}

int launch_div_target(int64_t n, const double* rho, const double* rho_prev, const double* Sp,
                      const double* Sd, double dt, double* out, cudaStream_t st) {
  if (n == 0) return FS_OK;
  k_div_target<<<blocks_for(n, 256), 256, 0, st>>>(n, rho, rho_prev, Sp, Sd, dt, out);
  fs_count_launch();
  return cuda_status();
}

// External ignition pulse (spread_3d.py:2528-2532): q_rad[k, :, i0:i1] += q_add.
__global__ void k_ignition_pulse(GridDev g, double* q, int k, int i0, int w, double q_add) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w * g.ny) return;
  const int j = t / w, i = i0 + (t - j * w);
  q[cidx(g, k, j, i)] += q_add;
}

int launch_ignition_pulse(const GridDev& g, double* q, int k, int i0, int i1, double q_add,
                          cudaStream_t st) {
  const int w = i1 - i0;
  if (w <= 0 || g.ny <= 0) return FS_OK;
  k_ignition_pulse<<<blocks_for((int64_t)w * g.ny, 128), 128, 0, st>>>(g, q, k, i0, w, q_add);
  fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Per-step front and heat-release diagnostics over x columns, in two passes:
//   hrr_x[i] = scale * sum_{k,j} omega[k,j,i] * dz[k]   (HRRPUA(x) with
//              scale = HOC * dy / Ly)
//   lead     = largest i whose column holds a T_s >= T_front, T_s rounded to
//              float32 first (the snapshot worker's ROS_Ts test,
//              _cheney_phase16_worker.py:208-231, reads float32 snapshots)
//   n_ign    = number of cells with T_s >= T_ign (spread_3d.py:3509)
//   sp_max   = max(S_pyro + S_drying) (spread_3d.py:3506)
//   hrr_max  = max_i hrr_x[i]
// Pass 1: a block holds 32 columns and one of S slices of the (k, j) rows;
// partial column sums are added per slice in a fixed order, so the result
// does not depend on scheduling.  Pass 2 adds the slices in slice order.
// ---------------------------------------------------------------------------
#define COLDIAG_X 32
#define COLDIAG_Y 8

__global__ void __launch_bounds__(COLDIAG_X * COLDIAG_Y)
    k_coldiag_partial(GridDev g, const double* __restrict__ Ts, const double* __restrict__ om,
                      const double* __restrict__ Sp, const double* __restrict__ Sd, double T_ign,
                      float T_front, int S, double* __restrict__ part, int* __restrict__ hot,
                      unsigned long long* keys) {
  __shared__ double s_sum[COLDIAG_Y][COLDIAG_X];
  __shared__ int s_hot[COLDIAG_Y][COLDIAG_X];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * COLDIAG_X + tx;
  const int rows = g.nz * g.ny;
  double acc = 0.0;
  int h = 0;
  unsigned long long cnt = 0, spk = 0;
  if (i < g.nx) {
    for (int r = blockIdx.y * COLDIAG_Y + ty; r < rows; r += COLDIAG_Y * S) {
      const int k = r / g.ny;
      const int64_t c = (int64_t)r * g.nx + i;
      const double t = Ts[c];
      acc += om[c] * g.dz[k];
      h |= ((float)t >= T_front) ? 1 : 0;
      cnt += (t >= T_ign) ? 1ull : 0ull;
      const unsigned long long kk = dkey(Sp[c] + Sd[c]);
      spk = kk > spk ? kk : spk;
    }
  }
  s_sum[ty][tx] = acc;
  s_hot[ty][tx] = h;
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, spk, o);
    spk = y > spk ? y : spk;
  }
  if (tx == 0) {
    if (cnt) atomicAdd(keys + 0, cnt);
    if (spk) atomicMax(keys + 1, spk);
  }
  __syncthreads();
  if (ty == 0 && i < g.nx) {
    double sum = s_sum[0][tx];
    int hh = s_hot[0][tx];
    for (int y = 1; y < COLDIAG_Y; ++y) {
      sum += s_sum[y][tx];
      hh |= s_hot[y][tx];
    }
    part[(int64_t)blockIdx.y * g.nx + i] = sum;
    hot[(int64_t)blockIdx.y * g.nx + i] = hh;
  }
}

__global__ void k_coldiag_final(int nx, int S, const double* __restrict__ part,
                                const int* __restrict__ hot, double scale, double* hrr_x,
                                unsigned long long* keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    int h = 0;
    for (int b = 0; b < S; ++b) {
      s += part[(int64_t)b * nx + i];
      h |= hot[(int64_t)b * nx + i];
    }
    const double v = s * scale;
    if (hrr_x) hrr_x[i] = v;
    atomicMax(keys + 2, dkey(v));
    if (h) atomicMax(keys + 3, (unsigned long long)(i + 1));
  }
}

int coldiag_slices(const GridDev& g) {
  const int bx = (g.nx + COLDIAG_X - 1) / COLDIAG_X;
  int S = (2 * 148 + bx - 1) / bx;
  const int rows = g.nz * g.ny;
  const int smax = (rows + COLDIAG_Y - 1) / COLDIAG_Y;
  if (S > smax) S = smax;
  if (S > 64) S = 64;
  return S < 1 ? 1 : S;
}

int64_t coldiag_scratch_bytes(const GridDev& g) {
  const int S = coldiag_slices(g);
  return 32 + (int64_t)S * g.nx * (int64_t)(sizeof(double) + sizeof(int)) + 256;
}

int launch_coldiag(const GridDev& g, const double* Ts, const double* om, const double* Sp,
                   const double* Sd, double T_ign, double T_front, double scale, double* hrr_x,
                   void* scratch, cudaStream_t st) {
  const int S = coldiag_slices(g);
  unsigned long long* keys = (unsigned long long*)scratch;
  double* part = (double*)((char*)scratch + 32);
  int* hot = (int*)(part + (int64_t)S * g.nx);
  cudaMemsetAsync(keys, 0, 32, st);
  dim3 grid((g.nx + COLDIAG_X - 1) / COLDIAG_X, S);
  k_coldiag_partial<<<grid, dim3(COLDIAG_X, COLDIAG_Y), 0, st>>>(
      g, Ts, om, Sp, Sd, T_ign, (float)T_front, S, part, hot, keys);
  fs_count_launch();
  k_coldiag_final<<<blocks_for(g.nx, 128), 128, 0, st>>>(g.nx, S, part, hot, scale, hrr_x,
                                                         keys);
  fs_count_launch();
  return cuda_status();
}

__global__ void k_coldiag_keys(const unsigned long long* keys, double* out) {
  if (threadIdx.x == 0) {
    out[0] = (double)keys[0];
    out[1] = keys[1] ? dkey_inv(keys[1]) : 0.0;
    out[2] = keys[2] ? dkey_inv(keys[2]) : 0.0;
    out[3] = (double)keys[3] - 1.0;
  }
}

int launch_coldiag_keys(const void* scratch, double* out4, cudaStream_t st) {
  k_coldiag_keys<<<1, 32, 0, st>>>((const unsigned long long*)scratch, out4);
  fs_count_launch();
  return cuda_status();
}

// clip a field to [lo, hi] (numpy minimum/maximum semantics: NaN stays NaN)
__global__ void k_clip(int64_t n, double* f, double lo, double hi) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double x = f[c];
  if (x > hi) x = hi;
  if (x < lo) x = lo;
  f[c] = x;
}

int launch_clip(int64_t n, double* f, double lo, double hi, cudaStream_t st) {
  k_clip<<<blocks_for(n, 256), 256, 0, st>>>(n, f, lo, hi); fs_count_launch();
  return cuda_status();
}

// ---------------------------------------------------------------------------
// Max reductions.  Slots written as order-preserving uint64 keys.
//   mode 0: max |f| (NaN propagates)      mode 1: max f (NaN propagates)
//   mode 2: max f over k in [1,Nz-2], i in [1,Nx-2], starting at 0, NaN ignored
//           (turbulence_3d.py:894-900)
// ---------------------------------------------------------------------------
__global__ void k_max(GridDev g, const double* __restrict__ f, int mode,
                      unsigned long long* out) {
  int64_t n = ncells_dev(g);
  unsigned long long best = dkey(mode == 2 ? 0.0 : -INFINITY);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    double x = f[c];
    if (mode == 0) x = fabs(x);
    if (mode == 2) {
      int i = (int)(c % g.nx);
      int k = (int)(c / ((int64_t)g.nx * g.ny));
      if (k < 1 || k > g.nz - 2 || i < 1 || i > g.nx - 2) continue;
      if (x != x) continue;
    }
    if (x != x) x = __longlong_as_double(0x7ff8000000000000ll);
    unsigned long long kk = dkey(x);
    if (kk > best) best = kk;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_xor_sync(0xffffffffu, best, o);
    if (y > best) best = y;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void k_init_keys(unsigned long long* out, int n, int mode2_mask) {
  int t = threadIdx.x;
  if (t < n) out[t] = ((mode2_mask >> t) & 1) ? dkey(0.0) : dkey(-INFINITY);
}

int launch_max(const GridDev& g, const double* f, int mode, unsigned long long* out_key,
               cudaStream_t st) {
  int64_t n = ncells(g);
  unsigned nb = blocks_for(n, 256);
  if (nb > 148 * 8) nb = 148 * 8;
  k_max<<<nb, 256, 0, st>>>(g, f, mode, out_key); fs_count_launch();
  return cuda_status();
}

int launch_init_keys(unsigned long long* out, int n, int mode2_mask, cudaStream_t st) {
  k_init_keys<<<1, 64, 0, st>>>(out, n, mode2_mask); fs_count_launch();
  return cuda_status();
}

__global__ void k_keys_to_double(const unsigned long long* in, double* out, int n) {
  int t = threadIdx.x;
  if (t < n) out[t] = dkey_inv(in[t]);
}

int launch_keys_to_double(const unsigned long long* in, double* out, int n, cudaStream_t st) {
  k_keys_to_double<<<1, 64, 0, st>>>(in, out, n); fs_count_launch();
  return cuda_status();
}
