// Lagrangian bed particles (lagrangian_bed_3d.py).
//
// Bed particles are stationary, so the cell of every slot is fixed at set-up
// (locate_cell, lagrangian_particles_3d.py:112-140).  The host builds a
// segment table: the slots of each occupied cell in increasing slot order.
// One thread walks one segment, so every per-cell sum is accumulated in the
// same order as the reference's serial slot loop (bit-identical `+=` order,
// no atomics), and every particle's own update is independent.
#include "common.cuh"
#include "kernels.h"

struct BedPart {
  double *x, *y, *z;
  signed char* alive;
  double *m_solid, *m_water, *m_char, *T_s, *m_water_0, *sav, *m_char_max;
};

struct BedSeg {
  int nseg;
  const int* seg_start;  // [nseg+1] into perm
  const int* seg_cell;   // [nseg] flat cell index
  const int* perm;       // slot indices grouped by cell, slot order within a cell
};

struct BedOut {
  double *S_pyro, *S_dry, *Q_pyro, *Q_dry, *YF_src, *Q_char, *Q_smold, *Q_gconv;
};

struct BedParams {
  double dt, inv_dt, h_conv, rho_true, cp_solid, eps_solid, T_amb, view, h_bed, kappa_bed;
  double char_cap, ash_exp, dxdy, eta, q_drip_solid, qrad_max;
  int do_dry, do_pyro, do_char, do_smold, mode, geometric, n_split, n_z_bed, i_src0, i_src1;
  int drip_on;
  const double* q_rad;  // for Q_solid_ext (null: Q_solid_ext given)
  const double* Qsx;
};

// pyrolysis_3d.py constants used by the particle kernel
#define R_GAS 8.314
#define A_DRY 4.29e3
#define E_DRY 43800.0
#define A_DRY_GRASS 4.29e3
#define E_DRY_GRASS 30000.0
#define L_VAP 2.26e6
#define A_MD 36280.0
#define E_MD 58600.0
#define A_OP 7.26e4
#define E_OP 55000.0
#define Y_O2_MIN_OP 1.0e-3
#define CHAR_YIELD 0.15
#define HEAT_OF_PYRO 4.0e5
#define HOR_OP (-1.0e6)
#define A_CHAR 7.09e5
#define E_CHAR 94000.0
#define HOC_CHAR 32000000.0
#define T_CHAR_ONSET 600.0
#define Y_O2_MIN_CHAR 1.0e-3
#define A_SMOLD 1.0e6
#define E_SMOLD 80000.0
#define HOC_SMOLD 28000000.0
#define T_SMOLD_ONSET 473.0
#define Y_O2_MIN_SMOLD 1.0e-3
#define SIGMA_SB 5.67e-8
#define T_BOIL 373.15

__global__ void k_bed_step(GridDev g, BedPart P, BedSeg S, BedOut O, BedParams B,
                           const double* __restrict__ Tg, const double* __restrict__ YO2) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.nseg) return;
  const int c = S.seg_cell[s];
  const int nxy = g.nx * g.ny;
  const int k = c / nxy;
  const int i = c % g.nx;
  const double V_cell = B.dxdy * g.dz[k];
  const double T_g = Tg[c];
  const double Y_O2 = YO2[c];
  double Qsx;
  if (B.Qsx) {
    Qsx = B.Qsx[c];
  } else {
    Qsx = 0.0;
    if (B.drip_on && k < B.n_z_bed && i >= B.i_src0 && i < B.i_src1) Qsx = Qsx + B.q_drip_solid;
    if (k < B.n_z_bed) {
      double vq = B.q_rad[c] / g.dz[k];
      if (vq < -B.qrad_max) vq = -B.qrad_max;
      if (vq > B.qrad_max) vq = B.qrad_max;
      Qsx = Qsx + vq;
    }
  }
  double aS_pyro = 0.0, aS_dry = 0.0, aQ_pyro = 0.0, aQ_dry = 0.0, aYF = 0.0, aQ_char = 0.0,
         aQ_smold = 0.0, aQ_gconv = 0.0;
  const double inv_V = 1.0 / V_cell;
  for (int q = S.seg_start[s]; q < S.seg_start[s + 1]; ++q) {
    const int p = S.perm[q];
    if (P.alive[p] == 0) continue;
    double T_s = P.T_s[p];
    double m_solid = P.m_solid[p], m_water = P.m_water[p], m_char = P.m_char[p];
    const double m_water_0 = P.m_water_0[p], sav = P.sav[p];
    double dm_evap = 0.0;
    if (B.do_dry && m_water > 0.0 && T_s > 0.0) {
      if (B.mode == 0 || B.mode == 2) {
        double A = B.mode == 0 ? A_DRY : A_DRY_GRASS;
        double E = B.mode == 0 ? E_DRY : E_DRY_GRASS;
        double k_dry = A * exp(-E / (R_GAS * T_s));
        double mw_new = m_water * exp(-k_dry * B.dt);
        dm_evap = m_water - mw_new;
        m_water = mw_new;
      }
    }
    double rate_pyro = 0.0, f_thermal = 1.0, f_op = 0.0;
    if (B.do_pyro && m_solid > 0.0 && T_s > 0.0) {
      double moist_gate;
      if (m_water_0 > 0.0) {
        double wet = m_water / m_water_0;
        moist_gate = 1.0 - wet;
        if (moist_gate < 0.0) moist_gate = 0.0;
      } else {
        moist_gate = 1.0;
      }
      if (moist_gate > 0.0) {
        double k_th = A_MD * exp(-E_MD / (R_GAS * T_s));
        double k_op = 0.0;
        if (Y_O2 > Y_O2_MIN_OP) k_op = A_OP * exp(-E_OP / (R_GAS * T_s)) * Y_O2;
        double k_tot = k_th + k_op;
        if (k_tot > 0.0) {
          double m_new = m_solid * exp(-k_tot * B.dt);
          double dm_full = m_solid - m_new;
          double dm_pyro = dm_full * moist_gate;
          rate_pyro = dm_pyro * B.inv_dt;
          f_thermal = k_th / k_tot;
          f_op = k_op / k_tot;
          m_char += CHAR_YIELD * dm_pyro;
          m_solid -= dm_pyro;
          if (m_char > P.m_char_max[p]) P.m_char_max[p] = m_char;
        }
      }
    }
    const double A_p_now = sav * (m_solid + m_char) / B.rho_true;
    double Q_char_p = 0.0;
    if (B.do_char && m_char > 1.0e-12 && T_s >= T_CHAR_ONSET && Y_O2 >= Y_O2_MIN_CHAR) {
      double k_ch = A_CHAR * exp(-E_CHAR / (R_GAS * T_s));
      double m_dot = k_ch * m_char * Y_O2;
      double m_cons = m_dot * B.dt;
      if (m_cons > 0.5 * m_char) m_cons = 0.5 * m_char;
      double A_re = A_p_now;
      if (B.ash_exp > 0.0 && P.m_char_max[p] > 1.0e-15) {
        double bf = m_char / P.m_char_max[p];
        if (bf < 0.0) bf = 0.0;
        A_re *= pow(bf, B.ash_exp);
      }
      double Q_cap = B.char_cap * A_re;
      double Q_arr = (m_cons * HOC_CHAR) * B.inv_dt;
      if (Q_arr > Q_cap) m_cons = Q_cap / (HOC_CHAR * B.inv_dt);
      Q_char_p = (m_cons * HOC_CHAR) * B.inv_dt;
      m_char -= m_cons;
    }
    double Q_smold_p = 0.0;
    if (B.do_smold && T_s >= T_SMOLD_ONSET && Y_O2 >= Y_O2_MIN_SMOLD) {
      double m_av = m_solid + m_char;
      if (m_av > 1.0e-12) {
        double k_sm = A_SMOLD * exp(-E_SMOLD / (R_GAS * T_s));
        double m_dot = k_sm * m_av * Y_O2;
        double m_cons = m_dot * B.dt;
        if (m_cons > 0.5 * m_av) m_cons = 0.5 * m_av;
        double Q_cap = 4.0e4 * A_p_now;
        double Q_arr = (m_cons * HOC_SMOLD) * B.inv_dt;
        if (Q_arr > Q_cap) m_cons = Q_cap / (HOC_SMOLD * B.inv_dt);
        if (m_av > 0.0) {
          double fs = m_solid / m_av;
          double dms = fs * m_cons;
          double dmc = (1.0 - fs) * m_cons;
          m_solid -= dms;
          m_char -= dmc;
        }
        Q_smold_p = (m_cons * HOC_SMOLD) * B.inv_dt;
      }
    }
    aS_pyro += B.eta * rate_pyro * inv_V;
    aS_dry += dm_evap * B.inv_dt * inv_V;
    aQ_pyro += (rate_pyro * (f_thermal * HEAT_OF_PYRO + f_op * HOR_OP)) * inv_V;
    aQ_dry += dm_evap * L_VAP * B.inv_dt * inv_V;
    aYF += B.eta * rate_pyro * inv_V;
    aQ_char += Q_char_p * inv_V;
    aQ_smold += Q_smold_p * inv_V;

    const double m_total = m_solid + m_water + m_char;
    double Q_conv = 0.0;
    if (m_total > 0.0) {
      double A_p = sav * (m_solid + m_char) / B.rho_true;
      Q_conv = B.h_conv * A_p * (T_g - T_s);
      double Q_rxn = -rate_pyro * (f_thermal * HEAT_OF_PYRO + f_op * HOR_OP);
      double Q_dry_part = -dm_evap * L_VAP * B.inv_dt;
      double Q_ext_p = 0.0;
      if (B.n_split > 0) Q_ext_p = Qsx * V_cell / (double)B.n_split;
      double f_geom = 1.0;
      if (B.geometric) {
        double h_above = B.h_bed - P.z[p];
        if (h_above < 0.0) h_above = 0.0;
        f_geom = exp(-B.kappa_bed * h_above);
      }
      double C_rad = B.eps_solid * SIGMA_SB * A_p * B.view * f_geom;
      double mc = m_total * B.cp_solid;
      double Ta4 = B.T_amb * B.T_amb * B.T_amb * B.T_amb;
      double Q_other = Q_conv + Q_rxn + Q_dry_part + Q_char_p + Q_smold_p + Q_ext_p;
      double mc_inv_dt = mc / B.dt;
      double T_old = T_s, T_it = T_s;
      for (int it = 0; it < 5; ++it) {
        double T2 = T_it * T_it;
        double T3 = T2 * T_it;
        double T4 = T3 * T_it;
        double F = mc_inv_dt * (T_it - T_old) - Q_other + C_rad * (T4 - Ta4);
        double Fp = mc_inv_dt + 4.0 * C_rad * T3;
        T_it = T_it - F / Fp;
        if (T_it < B.T_amb) T_it = B.T_amb;
      }
      T_s = T_it;
      if (T_s > 1.0e4) T_s = 1.0e4;
      if (B.do_dry && (B.mode == 1 || B.mode == 2) && m_water > 0.0 && T_s > T_BOIL) {
        double ex = mc * (T_s - T_BOIL);
        double dm_eq = ex / L_VAP;
        if (dm_eq >= m_water) {
          double res = ex - m_water * L_VAP;
          dm_eq = m_water;
          m_water = 0.0;
          T_s = T_BOIL + (mc > 0.0 ? res / mc : 0.0);
        } else {
          m_water -= dm_eq;
          T_s = T_BOIL;
        }
        aS_dry += dm_eq * B.inv_dt * inv_V;
        aQ_dry += dm_eq * L_VAP * B.inv_dt * inv_V;
      }
    }
    aQ_gconv += Q_conv * inv_V;
    P.T_s[p] = T_s;
    P.m_solid[p] = m_solid;
    P.m_water[p] = m_water;
    P.m_char[p] = m_char;
    if (m_total < 1.0e-8) P.alive[p] = 0;
  }
  O.S_pyro[c] = aS_pyro;
  O.S_dry[c] = aS_dry;
  O.Q_pyro[c] = aQ_pyro;
  O.Q_dry[c] = aQ_dry;
  O.YF_src[c] = aYF;
  O.Q_char[c] = aQ_char;
  O.Q_smold[c] = aQ_smold;
  O.Q_gconv[c] = aQ_gconv;
}

int launch_bed_step(const GridDev& g, const BedPartH& ph, const BedSegH& sh, const BedOutH& oh,
                    const BedParamsH& bp, const double* Tg, const double* YO2, cudaStream_t st) {
  BedPart P{ph.x, ph.y, ph.z, ph.alive, ph.m_solid, ph.m_water, ph.m_char, ph.T_s, ph.m_water_0,
            ph.sav, ph.m_char_max};
  BedSeg S{sh.nseg, sh.seg_start, sh.seg_cell, sh.perm};
  BedOut O{oh.S_pyro, oh.S_dry, oh.Q_pyro, oh.Q_dry, oh.YF_src, oh.Q_char, oh.Q_smold, oh.Q_gconv};
  BedParams B{};
  B.dt = bp.dt; B.inv_dt = bp.dt > 0.0 ? 1.0 / bp.dt : 0.0;
  B.h_conv = bp.h_conv; B.rho_true = bp.rho_true; B.cp_solid = bp.cp_solid;
  B.eps_solid = bp.eps_solid; B.T_amb = bp.T_amb; B.view = bp.view; B.h_bed = bp.h_bed;
  B.kappa_bed = bp.kappa_bed; B.char_cap = bp.char_cap; B.ash_exp = bp.ash_exp;
  B.dxdy = g.dx * g.dy; B.eta = 1.0 - 0.15;
  double qd = 30000.0 / (bp.h_bed > 1e-3 ? bp.h_bed : 1e-3);
  B.q_drip_solid = 0.80 * qd;
  B.qrad_max = 1.0e5;
  B.do_dry = bp.do_dry; B.do_pyro = bp.do_pyro; B.do_char = bp.do_char; B.do_smold = bp.do_smold;
  B.mode = bp.mode; B.geometric = bp.geometric; B.n_split = bp.n_split;
  B.n_z_bed = bp.n_z_bed; B.i_src0 = bp.i_src0; B.i_src1 = bp.i_src1; B.drip_on = bp.drip_on;
  B.q_rad = bp.q_rad; B.Qsx = bp.Qsx;
  if (!B.q_rad && !B.Qsx) return FS_EARG;
  if (S.nseg > 0) {
    k_bed_step<<<blocks_for(S.nseg, 128), 128, 0, st>>>(g, P, S, O, B, Tg, YO2); fs_count_launch(); }
  return cuda_status();
}

// Mass-weighted particle T_s into the cell grid (lagrangian_bed_3d.py:501-546).
// Mode 1: M_local = sum m_water / sum m_solid (lagrangian_bed_3d.py:550-590).
__global__ void k_bed_aggregate(BedPart P, BedSeg S, double* out, int mode) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.nseg) return;
  double num = 0.0, den = 0.0;
  for (int q = S.seg_start[s]; q < S.seg_start[s + 1]; ++q) {
    int p = S.perm[q];
    if (P.alive[p] == 0) continue;
    if (mode == 0) {
      double mt = P.m_solid[p] + P.m_water[p] + P.m_char[p];
      if (mt <= 0.0) continue;
      num += P.T_s[p] * mt;
      den += mt;
    } else {
      num += P.m_water[p];
      den += P.m_solid[p];
    }
  }
  int c = S.seg_cell[s];
  if (mode == 0) {
    if (den > 0.0) out[c] = num / den;
  } else {
    out[c] = den > 0.0 ? num / den : 0.0;
  }
}

int launch_bed_aggregate(const BedPartH& ph, const BedSegH& sh, double* out, int mode,
                         cudaStream_t st) {
  BedPart P{ph.x, ph.y, ph.z, ph.alive, ph.m_solid, ph.m_water, ph.m_char, ph.T_s, ph.m_water_0,
            ph.sav, ph.m_char_max};
  BedSeg S{sh.nseg, sh.seg_start, sh.seg_cell, sh.perm};
  if (S.nseg > 0) {
    k_bed_aggregate<<<blocks_for(S.nseg, 128), 128, 0, st>>>(P, S, out, mode); fs_count_launch(); }
  return cuda_status();
}

// Horizontal solid conduction on the bed T_s grid and scatter of the cell
// increment to the cell's particles (lagrangian_bed_3d.py:428-497).
// One thread per bed-layer cell; T_old is the grid before this call.
__global__ void k_bed_hcond(GridDev g, const double* __restrict__ T_old, double* T_new,
                            const double* __restrict__ as, int n_z_bed, double diff,
                            double inv_dx2, double inv_dy2, double dt, BedPart P, BedSeg S,
                            const int* __restrict__ seg_of_cell) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= n_z_bed) return;
  const int nx = g.nx, ny = g.ny;
  int64_t c = cidx(g, k, j, i);
  if (as[c] <= 0.0) return;
  double Tc = T_old[c];
  double Txp = (i + 1 < nx && as[c + 1] > 0.0) ? T_old[c + 1] : Tc;
  double Txm = (i - 1 >= 0 && as[c - 1] > 0.0) ? T_old[c - 1] : Tc;
  int jp = j + 1 < ny ? j + 1 : 0;
  int jm = j - 1 >= 0 ? j - 1 : ny - 1;
  int64_t cp = cidx(g, k, jp, i), cm = cidx(g, k, jm, i);
  double Typ = as[cp] > 0.0 ? T_old[cp] : Tc;
  double Tym = as[cm] > 0.0 ? T_old[cm] : Tc;
  double lap = (Txp - 2.0 * Tc + Txm) * inv_dx2 + (Typ - 2.0 * Tc + Tym) * inv_dy2;
  double dT = diff * lap * dt;
  T_new[c] = Tc + dT;
  int s = seg_of_cell[c];
  if (s >= 0) {
    for (int q = S.seg_start[s]; q < S.seg_start[s + 1]; ++q) {
      int p = S.perm[q];
      if (P.alive[p] == 0) continue;
      P.T_s[p] += dT;
    }
  }
}

int launch_bed_hcond(const GridDev& g, double* T_grid, double* scratch, const double* as,
                     int n_z_bed, double k_solid, double rho_true, double cp_solid, double dt,
                     const BedPartH& ph, const BedSegH& sh, const int* seg_of_cell,
                     cudaStream_t st) {
  BedPart P{ph.x, ph.y, ph.z, ph.alive, ph.m_solid, ph.m_water, ph.m_char, ph.T_s, ph.m_water_0,
            ph.sav, ph.m_char_max};
  BedSeg S{sh.nseg, sh.seg_start, sh.seg_cell, sh.perm};
  int nzb = n_z_bed < g.nz ? n_z_bed : g.nz;
  if (nzb <= 0) return FS_OK;
  // the conduction stencil reads the grid as it was before this call
  size_t bytes = sizeof(double) * (size_t)nzb * g.ny * g.nx;
  cudaMemcpyAsync(scratch, T_grid, bytes, cudaMemcpyDeviceToDevice, st);
  Launch3 L = launch_cells(g);
  L.grid.z = nzb;
  double diff = k_solid / (rho_true * cp_solid);
  k_bed_hcond<<<L.grid, L.block, 0, st>>>(g, scratch, T_grid, as, nzb, diff,
                                          1.0 / (g.dx * g.dx), 1.0 / (g.dy * g.dy), dt, P, S,
                                          seg_of_cell); fs_count_launch();
  return cuda_status();
}
