// Internal launcher declarations shared by the .cu files and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/firestep.h"

typedef FsBedParticles BedPartH;
typedef FsBedSegments BedSegH;
typedef FsBedSources BedOutHPub;

struct BedOutH {
  double *S_pyro, *S_dry, *Q_pyro, *Q_dry, *YF_src, *Q_char, *Q_smold, *Q_gconv;
};

struct BedParamsH {
  double dt, h_conv, rho_true, cp_solid, eps_solid, T_amb, view, h_bed, kappa_bed;
  double char_cap, ash_exp;
  int do_dry, do_pyro, do_char, do_smold, mode, geometric, n_split;
  const double* Qsx;
  const double* q_rad;
  int drip_on, n_z_bed, i_src0, i_src1;
};

struct GridDev;

int launch_species(const GridDev& g, int nspec, const double* const* Y, double* const* Yo,
                   const double* const* S, const double* Y_inlet, const double* rho,
                   const double* u, const double* v, const double* w, double dt, double D,
                   cudaStream_t st);
int launch_species_sources(int64_t n, const double* Sp, const double* Sd, const double* YF,
                           const double* YO, const double* YH, double* SF, double* SO,
                           double* SH, cudaStream_t st);
int launch_advect_scalar(const GridDev& g, const double* phi, const double* u, const double* v,
                         const double* w, double* rhs, double phi_inlet, cudaStream_t st);
int launch_gas_energy_adv(const GridDev& g, const double* T, const double* u, const double* v,
                          const double* w, double* To, double dt, double alpha, double T_amb,
                          cudaStream_t st);
int launch_turb_diff(const GridDev& g, int nfield, const double* const* f, double* const* fo,
                     const double* nu_t, double sc_t, double dt_sub, int clip, const double* lo,
                     const double* hi, cudaStream_t st);
int launch_drag(int64_t n, const double* u, const double* v, const double* w, const double* rho,
                const double* as, double sigma, double C_D, double* Fx, double* Fy, double* Fz,
                cudaStream_t st);
int launch_momentum(const GridDev& g, const double* u, const double* v, const double* w,
                    const double* rho, const double* T, const double* Fx, const double* Fy,
                    const double* Fz, const double* alpha_s, double sigma, double C_D,
                    const double* u_in, const double* v_in, const double* w_in, double* uo,
                    double* vo, double* wo, double dt, double T_amb, cudaStream_t st);
int launch_sponge(const GridDev& g, double* u, const double* u_t, const double* sig_x,
                  const double* YF, double skip, double dt, cudaStream_t st);
int launch_keps(const GridDev& g, const double* k, const double* e, const double* u,
                const double* v, const double* w, const double* T, const double* alpha_s,
                const double* u_in, const double* kwall, const double* ewall, double* ko,
                double* eo, double* nuo, double* S2o, double* O2o, double sigma, double dt,
                double T_amb, double beta_p, double beta_d, cudaStream_t st);
int launch_solid_cond(const GridDev& g, const double* Ts, const double* as, double* To,
                      double k_solid, double rho_s, double cp_s, double dt, int nz_active,
                      cudaStream_t st, int cap = 0, double lo = 0.0, double hi = 0.0);
int launch_soil(int nsoil, int ny, int nx, double* T, const double* qin, double dt,
                const double* sdz, const double* sda, const double* sdb, double k_s,
                double rho_s, double cp_s, double eps_s, double T_amb, cudaStream_t st);

int edc_scratch_bytes(int64_t n);
int launch_edc(int64_t n, const double* rho, double* Tg, double* Yf, double* YO, const double* kt,
               const double* et, const double* YH, double* omega, double chi_rad, double cp_g,
               double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
               void* scratch, cudaStream_t st);
int launch_gas_update(const GridDev& g, double* Tg, const double* rho, const double* YH,
                      const double* Ts, const double* Sp, const double* Sd, const double* Qgc,
                      const double* qrg, double* Qcomb_out, unsigned long long* qc_max,
                      double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                      int i_src0, int i_src1, cudaStream_t st);
int launch_gas_solid(const GridDev& g, double* Tg, const double* rho, const double* YH,
                     const double* Ts, const double* Sp, const double* Sd, const double* Qgc,
                     const double* qrg, double* Qcomb_out, double dt_sub, double T_amb,
                     double h_bed, int drip_on, int n_z_bed, int i_src0, int i_src1,
                     const double* as, double* Ts_out, double k_solid, double rho_s, double cp_s,
                     double lo, double hi, cudaStream_t st);
int launch_eos(const GridDev& g, double* rho, double* rho_prev, const double* Tg, double* YO,
               double P0, double R_air, double T_amb, cudaStream_t st);
int launch_clip(int64_t n, double* f, double lo, double hi, cudaStream_t st);
int launch_max(const GridDev& g, const double* f, int mode, unsigned long long* out_key,
               cudaStream_t st);
int launch_init_keys(unsigned long long* out, int n, int mode2_mask, cudaStream_t st);
int launch_keys_to_double(const unsigned long long* in, double* out, int n, cudaStream_t st);

void* proj_create(const GridDev& g);
void proj_destroy(void* h);
double* proj_pressure(void* h);
const double* proj_inv_rho(void* h);
int proj_nlevels(void* h);
int proj_rebuild(void* h, const double* rho, cudaStream_t st);
int proj_project(void* h, double* u, double* v, double* w, const double* u_in,
                 const double* target, double dt, double rtol, int maxiter, int* iters,
                 cudaStream_t st);
int proj_apply(void* h, const double* x, double* y, cudaStream_t st);
int proj_configure(void* h, int nu, double omega);
int proj_set_coarse_tail(void* h, int on);
int proj_set_fine_sweeps(void* h, int nu0);
int proj_set_precision(void* h, int fp32);
void proj_stats(void* h, double* out8);
// learned preconditioner (flexible CG); net = NULL returns to the V-cycle
int proj_set_learned(void* h, void* net, int max_learned, double stall);
// copies of the residual and the iterate at the start of every solve (NULL: off)
int proj_set_log(void* h, double* r0, double* x0);
void proj_fcg_stats(void* h, double* out4);

// U-Net (unet.cu)
int launch_species_step(const GridDev& g, const double* const* Y, double* const* Yo,
                        const double* Sp, const double* Sd, const double* Y_inlet,
                        const double* rho, const double* u, const double* v, const double* w,
                        double dt, double D, double o2_cap, cudaStream_t st);
int64_t unet_nparams();
int unet_create(int nz, int ny, int nx, void** out);
void unet_destroy(void* h);
int unet_set_params(void* h, const float* host, int64_t n, cudaStream_t st);
int unet_get(void* h, int which, float* host, int64_t n, cudaStream_t st);
int unet_apply(void* h, const double* r, double* z, cudaStream_t st);
int unet_forward_f32(void* h, const float* r, float* z, cudaStream_t st);
int unet_grad(void* h, const float* r, const float* tau, double* loss, cudaStream_t st);
int unet_train_step(void* h, const float* r, const float* tau, float lr, double* loss,
                    cudaStream_t st);
int unet_correct(void* h, const float* r, const float* base, float* out, cudaStream_t st);
int unet_set_output_scale(void* h, float s);
int64_t unet_cells(void* h);
int proj_smooth_pair(void* h, const double* r0, const double* e0, float* r1, float* e1,
                     cudaStream_t st);
int launch_div_resid_max(const GridDev& g, const double* u, const double* v, const double* w,
                         const double* u_in, const double* target, double* div_out,
                         unsigned long long* out_key, cudaStream_t st);

void* dom_create(const GridDev& g, int M, const double* ox, const double* oy, const double* oz,
                 const double* w, double kgmax);
void dom_destroy(void* h);
double* dom_intensity(void* h);
int dom_set_mode(void* h, int mode, int cluster_ctas);
int dom_begin(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH,
              const double* rho, const double* Mloc, cudaStream_t st);
int dom_end(void* h, double* q_solid, double* q_gas, double* q_in_soil, cudaStream_t st);
int dom_set_groups(void* h, int groups);
int dom_mode(void* h);
int dom_set_sweep_kernel(void* h, int kernel);
int dom_sweep_kernel(void* h);
int dom_launch_shape(void* h, int* out5);
int dom_set_wait_test(void* h, int plane);
int dom_set_precision(void* h, int fp32);
int dom_load_intensity(void* h, const double* I_full, cudaStream_t st);
int64_t dom_wrap_size(void* h);
int dom_get_wrap(void* h, double* dst, cudaStream_t st);
int dom_set_wrap(void* h, const double* src, cudaStream_t st);
double* dom_G(void* h);
int dom_last_iters(void* h);
void dom_set_timing(void* h, int on);
void dom_sweep_stats(void* h, double* ms, long long* count);
int dom_solve(void* h, const double* Ts, const double* Tg, const double* as, const double* om,
              double sigma, double T_amb, const double* Tsoil0, const double* YH, const double* rho,
              const double* Mloc, double* q_solid, double* q_gas, double* q_in_soil,
              cudaStream_t st);

int launch_bed_step(const GridDev& g, const BedPartH& ph, const BedSegH& sh, const BedOutH& oh,
                    const BedParamsH& bp, const double* Tg, const double* YO2, cudaStream_t st);
int launch_bed_aggregate(const BedPartH& ph, const BedSegH& sh, double* out, int mode,
                         cudaStream_t st);
int launch_bed_hcond(const GridDev& g, double* T_grid, double* scratch, const double* as,
                     int n_z_bed, double k_solid, double rho_true, double cp_solid, double dt,
                     const BedPartH& ph, const BedSegH& sh, const int* seg_of_cell,
                     cudaStream_t st);

int launch_levelset(const GridDev& g, const double* phi, const double* aux, double* out,
                    double coef, int mode, cudaStream_t st);
int launch_active_count(int64_t n, const double* om, const double* Tg, const double* YF,
                        unsigned long long* count, unsigned char* mask, cudaStream_t st);
int launch_div_target(int64_t n, const double* rho, const double* rho_prev, const double* Sp,
                      const double* Sd, double dt, double* out, cudaStream_t st);
int launch_ignition_pulse(const GridDev& g, double* q, int k, int i0, int i1, double q_add,
                          cudaStream_t st);
int coldiag_slices(const GridDev& g);
int64_t coldiag_scratch_bytes(const GridDev& g);
int launch_coldiag(const GridDev& g, const double* Ts, const double* om, const double* Sp,
                   const double* Sd, double T_ign, double T_front, double scale, double* hrr_x,
                   void* scratch, cudaStream_t st);
int launch_coldiag_keys(const void* scratch, double* out4, cudaStream_t st);
// stencil kernels with TMA-staged inputs: the bounded-wait failure flag
// (read, optionally cleared; -1 on a CUDA error) and the on/off switch
int stencil_status(int clear);
void set_tma(int on);
int launch_edc_carry(int nb, const signed char* agg, signed char* carry, cudaStream_t st);
// single-precision sub-step kernels (substep32.cu)
int launch_convert(int64_t n, int nf, const void* const* src, void* const* dst, int to_f32,
                   cudaStream_t st);
int64_t edc32_scratch_bytes(int64_t n);
int launch_edc32(int64_t n, const float* rho, float* Tg, float* Yf, float* YO, const float* kt,
                 const float* et, const float* YH, float* omega, double chi_rad, double cp_g,
                 double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
                 void* scratch, cudaStream_t st);
int launch_species_step32(const GridDev& g, const float* const* Y, float* const* Yo,
                          const float* Sp, const float* Sd, const double* Y_inlet,
                          const float* rho, const float* u, const float* v, const float* w,
                          double dt, double D, double o2_cap, cudaStream_t st);
int launch_turb_diff32(const GridDev& g, int nfield, const float* const* f, float* const* fo,
                       const float* nu_t, double sc_t, double dt_sub, int clip, const double* lo,
                       const double* hi, cudaStream_t st);
int launch_gas_update32(const GridDev& g, float* Tg, const float* rho, const float* YH,
                        const double* Ts, const float* Sp, const float* Sd, const float* Qgc,
                        const double* qrg, float* Qcomb_out, double dt_sub, double T_amb,
                        double h_bed, int drip_on, int n_z_bed, int i_src0, int i_src1,
                        cudaStream_t st);
int launch_clip32(int64_t n, float* f, double lo, double hi, cudaStream_t st);

