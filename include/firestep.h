/*
 * firestep.h -- C ABI of libfirestep.so, the sm_100a implementation of the
 * Tier-3 step of the FireWebApp 3D grass-fire solver
 * (src/model_outdoor/spread_3d.py driving src/model_outdoor/physics_3d/).
 *
 * Conventions (the same contract the reference kernels follow):
 *  - every 3D field is a C-contiguous float64 array (Nz, Ny, Nx) in device
 *    memory, cell (k,j,i) at (k*Ny + j)*Nx + i (spread_3d.py:88-155);
 *  - the caller owns every field; solver objects own their workspaces;
 *  - entry points take a cudaStream_t passed as void* and never synchronise
 *    the host, except where the name says so or the reference loop is
 *    data-dependent (documented per function);
 *  - every function returns an int status:
 *      0 ok, 1 bad argument, 2 non-finite value, 3 solver did not converge,
 *      4 device wait timed out, 5 CUDA error; fs_last_error() has the text.
 *
 * Each declaration names the reference function it replaces (file:line).
 */
#ifndef FIRESTEP_H
#define FIRESTEP_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define FS_OK 0
#define FS_EARG 1
#define FS_ENONFINITE 2
#define FS_ENOCONV 3
#define FS_ETIMEOUT 4 /* reserved: a bounded device wait gave up */
#define FS_ECUDA 5

/* Grid3D geometry (spread_3d.py:158-188): dz, d_above, d_below are device
 * arrays of length nz (dz_arr, d_face_above, d_face_below). */
typedef struct FsGrid {
  int nx, ny, nz;
  double dx, dy;
  const double* dz;
  const double* d_above;
  const double* d_below;
} FsGrid;

/* Lagrangian bed particle buffers (lagrangian_bed_3d.py:193-218). */
typedef struct FsBedParticles {
  double *x, *y, *z;
  signed char* alive;
  double *m_solid, *m_water, *m_char, *T_s, *m_water_0, *sav, *m_char_max;
} FsBedParticles;

/* Occupied cells and their particle slots in slot order (built on the host
 * from the fixed particle positions: particles do not move). */
typedef struct FsBedSegments {
  int nseg;
  const int* seg_start; /* [nseg+1] offsets into perm */
  const int* seg_cell;  /* [nseg] flat cell index */
  const int* perm;      /* slots grouped by cell */
} FsBedSegments;

/* Per-cell source grids written by fs_bed_step (lagrangian_bed_3d.py:610-619). */
typedef struct FsBedSources {
  double *S_pyro, *S_drying, *Q_pyro, *Q_drying, *Y_F_source, *Q_char, *Q_smold, *Q_g_conv;
} FsBedSources;

typedef struct FsBedParams {
  double dt, h_conv, rho_true, cp_solid, eps_solid, T_amb, view, h_bed, kappa_bed;
  double char_cap, ash_exp;
  int do_dry, do_pyro, do_char, do_smold, mode, geometric, n_split;
  /* Q_solid_ext: either a per-cell grid (Qsx) or assembled in-kernel from
   * the previous q_rad and the ignition drip (spread_3d.py:2078-2103). */
  const double* Qsx;
  const double* q_rad;
  int drip_on, n_z_bed, i_src0, i_src1;
} FsBedParams;

const char* fs_last_error(void);
int fs_version(void);
/* number of kernel launches this library has issued since it was loaded */
unsigned long long fs_launch_count(void);

/* species_3d.py:41 step_species_transport, up to 3 species in one pass,
 * out-of-place (Y -> Y_out, clipped to [0,1]). */
int fs_species_transport(const FsGrid* g, int nspec, const double* const* Y, double* const* Y_out,
                         const double* const* S, const double* Y_inlet, const double* rho,
                         const double* u, const double* v, const double* w, double dt, double D,
                         void* stream);

/* spread_3d.py:2996-3004 dilution-form species sources (Lagrangian bed). */
int fs_species_sources(int64_t n, const double* S_pyro, const double* S_drying,
                       const double* Y_F, const double* Y_O2, const double* Y_H2O, double* S_F,
                       double* S_O2, double* S_H2O, void* stream);

/* The sub-step's species work fused into one pass (no reference counterpart
 * as a single call): fs_species_sources, then fs_species_transport of
 * (Y_F, Y_O2, Y_H2O) with those sources, then fs_clip(Y_O2, 0, o2_cap)
 * (spread_3d.py:2996-3004, 3015-3038, 3059); the same results as the three
 * calls, without the source arrays. */
int fs_species_step(const FsGrid* g, const double* const* Y, double* const* Y_out,
                    const double* S_pyro, const double* S_drying, const double* Y_inlet,
                    const double* rho, const double* u, const double* v, const double* w,
                    double dt, double D, double o2_cap, void* stream);

/* muscl_3d.py:68 advect_3d_scalar_muscl: rhs -= u . grad(phi). */
int fs_advect_scalar_muscl(const FsGrid* g, const double* phi, const double* u, const double* v,
                           const double* w, double* rhs, double phi_inlet, void* stream);

/* spread_3d.py:3827 _adv_gas_energy, out-of-place. */
int fs_gas_energy_adv(const FsGrid* g, const double* T_g, const double* u, const double* v,
                      const double* w, double* T_out, double dt, double alpha_th, double T_amb,
                      void* stream);

/* turbulence_3d.py:862 apply_turbulent_diffusion: the sub-step count
 * (host result, synchronises the stream) ... */
int fs_turb_diffusion_nsub(const FsGrid* g, const double* nu_t, double sc_t, double dt,
                           int* n_sub, double* dt_sub, void* stream);
/* ... and one sub-step for up to 4 fields, out-of-place, optional clip. */
int fs_turb_diffusion_substep(const FsGrid* g, int nfield, const double* const* f,
                              double* const* f_out, const double* nu_t, double sc_t, double dt_sub,
                              int clip, const double* lo, const double* hi, void* stream);

/* drag_3d.py:100 step_drag_force. */
int fs_drag_force(int64_t n, const double* u, const double* v, const double* w, const double* rho,
                  const double* alpha_s, double sigma_sav, double C_D, double* Fx, double* Fy,
                  double* Fz, void* stream);

/* momentum_3d.py:42 step_tentative_velocity, out-of-place.  With Fx == NULL
 * the drag force is evaluated in-kernel from alpha_s (drag_3d.py:100). */
int fs_tentative_velocity(const FsGrid* g, const double* u, const double* v, const double* w,
                          const double* rho, const double* T_g, const double* Fx, const double* Fy,
                          const double* Fz, const double* alpha_s, double sigma_sav, double C_D,
                          const double* u_inlet, const double* v_inlet, const double* w_inlet,
                          double* u_out, double* v_out, double* w_out, double dt, double T_amb,
                          void* stream);

/* momentum_3d.py:293 apply_outflow_sponge, in place. */
int fs_outflow_sponge(const FsGrid* g, double* u, const double* u_target, const double* sigma_x,
                      const double* Y_F, double Y_F_skip, double dt, void* stream);

/* turbulence_3d.py:482 step_k_epsilon (with :392 _strain_and_vorticity_squared
 * evaluated in-kernel; S2/O2 outputs optional), out-of-place.  Only the
 * production options: bvg_factor = L_min = durbin_alpha = 0. */
int fs_k_epsilon(const FsGrid* g, const double* k, const double* eps, const double* u,
                 const double* v, const double* w, const double* T_g, const double* alpha_s,
                 const double* u_inlet, const double* k_wall, const double* eps_wall, double* k_out,
                 double* eps_out, double* nu_t_out, double* S2_out, double* O2_out,
                 double sigma_sav, double dt, double T_amb, double beta_p, double beta_d,
                 void* stream);

/* chemistry_closures/edc.py:134 step_chemistry_ode_edc, in place; scratch of
 * fs_edc_scratch_bytes(n) bytes.  The H2O-quench flag of cells that skip the
 * reacting branch is the one left by the previous cell in flat k-j-i order
 * (the reference's one-thread behaviour, edc.py:223). */
int64_t fs_edc_scratch_bytes(int64_t n);
int fs_edc(int64_t n, const double* rho, double* T_g, double* Y_F, double* Y_O2, const double* k,
           const double* eps, const double* Y_H2O, double* omega, double chi_rad, double cp_g,
           double dt, int n_substeps, double s_stoich, double hoc_J, int extinction, void* scratch,
           void* stream);

/* No counterpart in the reference: fs_edc for callers that cannot allocate
 * device memory, such as a host whose own allocator owns all device memory
 * (fixed arena, caching allocator) or a loop that cannot afford the
 * synchronisation of cudaMalloc.  Same arguments and results as fs_edc
 * without the scratch buffer; the flag scan uses a static device array (about
 * 256 KiB per GPU that loads the library, held until exit) sized for at most
 * FS_EDC_NOALLOC_MAX_CELLS cells (larger n is rejected with FS_EARG).  The
 * first call on a device looks the array up (make it before any stream
 * capture); all calls share the array, so calls whose kernels overlap on the
 * GPU race.  It calls no allocation routine.  The looked-up address is kept
 * for the life of the process: it is valid in the device's primary context
 * (the one the CUDA runtime and torch use) and not after cudaDeviceReset or
 * in another context made on the same device. */
#define FS_EDC_NOALLOC_MAX_CELLS (1LL << 27)
int fs_edc_noalloc(int64_t n, const double* rho, double* T_g, double* Y_F, double* Y_O2,
                   const double* k, const double* eps, const double* Y_H2O, double* omega,
                   double chi_rad, double cp_g, double dt, int n_substeps, double s_stoich,
                   double hoc_J, int extinction, void* stream);

/* spread_3d.py:2916-2957 + 3104-3146: drip + q_rad_gas into Q_comb and the
 * Lagrangian-branch gas-energy update, in place. */
int fs_gas_energy_update(const FsGrid* g, double* T_g, const double* rho, const double* Y_H2O,
                         const double* T_s, const double* S_pyro, const double* S_drying,
                         const double* Q_g_conv, const double* q_rad_gas, double* Q_comb_out,
                         double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                         int i_src0, int i_src1, void* stream);

/* The sub-step's gas-energy update and its capped solid conduction in one
 * pass: the results of fs_gas_energy_update(g, T_g, ..., i_src1) followed by
 * fs_solid_conduction_capped(g, T_s, alpha_s, T_s_out, k_solid, rho_solid,
 * cp_solid, dt_sub, Ts_lo, Ts_hi), bit for bit (both read the old T_s; neither
 * reads what the other writes).  T_s_out must not be T_s. */
int fs_gas_energy_solid_update(const FsGrid* g, double* T_g, const double* rho,
                               const double* Y_H2O, const double* T_s, const double* S_pyro,
                               const double* S_drying, const double* Q_g_conv,
                               const double* q_rad_gas, double* Q_comb_out, double dt_sub,
                               double T_amb, double h_bed, int drip_on, int n_z_bed, int i_src0,
                               int i_src1, const double* alpha_s, double* T_s_out,
                               double k_solid, double rho_solid, double cp_solid, double Ts_lo,
                               double Ts_hi, void* stream);

/* spread_3d.py:2300-2317 (with S_pyro = S_pyro_bed + S_drying_bed,
 * :2147-2148): div_target = (S_pyro - (rho - rho_prev)/dt) / max(rho, 0.1),
 * the right-hand side of the pressure iterations; overwrites div_target. */
int fs_div_target(int64_t n, const double* rho, const double* rho_prev, const double* S_pyro,
                  const double* S_drying, double dt, double* div_target, void* stream);

/* spread_3d.py:2528-2532: the external ignition pulse, q_rad[k, :, i0:i1] +=
 * q_add (k = n_z_bed - 1, q_add = 240 kW/m2 x ignition_q_mult), in place. */
int fs_ignition_pulse(const FsGrid* g, double* q_rad, int k, int i0, int i1, double q_add,
                      void* stream);

/* The stencil kernels whose inputs are staged in shared memory by the
 * tensor memory accelerator (the fused species step; see fs_species_step)
 * wait on mbarriers with a bound.  fs_stencil_status returns 1 if such a wait
 * gave up since the flag was last cleared (the kernel's results are then not
 * to be trusted: the caller reports FS_ETIMEOUT), 0 if not, -1 on a CUDA
 * error; clear = 1 clears it.  Synchronous.  fs_set_tma(0) makes those
 * kernels read their inputs directly instead (the same results); 1, the
 * default, stages them where the grid allows (even nx). */
int fs_stencil_status(int clear);
int fs_set_tma(int on);

/* ---- Single-precision sub-step kernels (mixed-precision form; no
 * counterpart in the reference, which is FP64 throughout).  The ten
 * chemistry/transport sub-steps of an outer step (spread_3d.py:2678-3196) run
 * on FP32 copies: fs_convert widens or narrows nf device arrays of n elements
 * (to_f32 = 1: double -> float, 0: float -> double).  Each kernel restates its
 * FP64 entry point in float arithmetic with the same arguments, float arrays
 * in place of double ones:
 *   fs_edc_f32                    = fs_edc (same flat-order flag scan; scratch
 *                                   of fs_edc_f32_scratch_bytes(n) bytes)
 *   fs_species_step_f32           = fs_species_step
 *   fs_turb_diffusion_substep_f32 = fs_turb_diffusion_substep (1 or 3 fields)
 *   fs_gas_energy_update_f32      = fs_gas_energy_update (T_s and q_rad_gas
 *                                   stay FP64 inputs)
 *   fs_clip_f32                   = fs_clip */
int fs_convert(int64_t n, int nf, const void* const* src, void* const* dst, int to_f32,
               void* stream);
int64_t fs_edc_f32_scratch_bytes(int64_t n);
int fs_edc_f32(int64_t n, const float* rho, float* T_g, float* Y_F, float* Y_O2, const float* k,
               const float* eps, const float* Y_H2O, float* omega, double chi_rad, double cp_g,
               double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
               void* scratch, void* stream);
int fs_species_step_f32(const FsGrid* g, const float* const* Y, float* const* Y_out,
                        const float* S_pyro, const float* S_drying, const double* Y_inlet,
                        const float* rho, const float* u, const float* v, const float* w,
                        double dt, double D, double o2_cap, void* stream);
int fs_turb_diffusion_substep_f32(const FsGrid* g, int nfield, const float* const* f,
                                  float* const* f_out, const float* nu_t, double sc_t,
                                  double dt_sub, int clip, const double* lo, const double* hi,
                                  void* stream);
int fs_gas_energy_update_f32(const FsGrid* g, float* T_g, const float* rho, const float* Y_H2O,
                             const double* T_s, const float* S_pyro, const float* S_drying,
                             const float* Q_g_conv, const double* q_rad_gas, float* Q_comb_out,
                             double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                             int i_src0, int i_src1, void* stream);
int fs_clip_f32(int64_t n, float* f, double lo, double hi, void* stream);

/* Per-step diagnostics over x columns, one pass over T_s, omega and the bed
 * sources (spread_3d.py:3503-3512 maxima and ignited-cell count; ROS_Ts front
 * test of _cheney_phase16_worker.py:208-231; HRRPUA(x)):
 *   hrr_x[i] = hrr_scale * sum_{k,j} omega * dz_k  (device, Nx; may be NULL),
 *   lead_i   = largest column i with any float32(T_s) >= T_front, or -1,
 *   n_ign    = count of T_s >= T_ign,  S_pyro_max = max(S_pyro + S_drying),
 *   hrr_max  = max_i hrr_x[i].
 * Column sums are added in a fixed order (reproducible).  scratch: device,
 * fs_column_diag_scratch_bytes(g) bytes.  Waits for the stream (host result). */
typedef struct {
  int64_t n_ign;
  int lead_i;
  double S_pyro_max;
  double hrr_max;
} FsColumnDiag;
int64_t fs_column_diag_scratch_bytes(const FsGrid* g);
int fs_column_diag(const FsGrid* g, const double* T_s, const double* omega, const double* S_pyro,
                   const double* S_drying, double T_ign, double T_front, double hrr_scale,
                   double* hrr_x, void* scratch, FsColumnDiag* out, void* stream);

/* spread_3d.py:2042 / :3440 EoS; with rho_prev != NULL also copies the old
 * rho (:1984) and with Y_O2 != NULL sets the inlet column to 0.232 (:2050). */
int fs_eos(const FsGrid* g, double* rho, double* rho_prev, const double* T_g, double* Y_O2,
           double T_amb, void* stream);

/* numpy clip (minimum then maximum), in place. */
int fs_clip(int64_t n, double* f, double lo, double hi, void* stream);

/* solid_conduction_3d.py:56 step_solid_conduction_vertical, out-of-place. */
int fs_solid_conduction(const FsGrid* g, const double* T_s, const double* alpha_s, double* T_out,
                        double k_solid, double rho_solid, double cp_solid, double dt,
                        void* stream);

/* fs_solid_conduction followed by fs_clip(T_out, lo, hi) in one pass (the
 * T_s cap of spread_3d.py:3193-3196); the same results as the two calls. */
int fs_solid_conduction_capped(const FsGrid* g, const double* T_s, const double* alpha_s,
                               double* T_out, double k_solid, double rho_solid, double cp_solid,
                               double dt, double lo, double hi, void* stream);

/* soil_3d.py:106 step_soil_conduction, in place. */
int fs_soil_step(int nsoil, int ny, int nx, double* T_soil, const double* q_in, double dt,
                 const double* soil_dz, const double* d_above, const double* d_below, double k_s,
                 double rho_s, double cp_s, double eps_s, double T_amb, void* stream);

/* projection_3d.py:178 ProjectionSolver3D (fft_pcg path): create/destroy,
 * :317 rebuild_for_rho, :677 project (synchronises once per CG iteration;
 * warm start from the previous solution) and :847 divergence. */
int fs_proj_create(const FsGrid* g, void** handle);
void fs_proj_destroy(void* handle);
int fs_proj_rebuild(void* handle, const double* rho, void* stream);
int fs_proj_project(void* handle, double* u, double* v, double* w, const double* u_inlet,
                    const double* div_target, double dt, double rtol, int maxiter, int* iters,
                    void* stream);
double* fs_proj_pressure(void* handle);
int fs_proj_apply(void* handle, const double* x, double* y, void* stream);
/* Multigrid preconditioner: nu damped-Jacobi sweeps (weight omega) before and
 * after each coarse correction (default 4 and 0.9).  The reference's
 * preconditioner (projection_3d.py:236-246, an FFT solve) has no such knob;
 * only the converged solution is shared. */
int fs_proj_configure(void* handle, int nu, double omega);
/* Jacobi sweeps before and after the coarse correction on the finest level
 * only (nu0 = 0: the same as the coarser levels, fs_proj_configure's nu). */
int fs_proj_set_fine_sweeps(void* handle, int nu0);
/* on = 1 (default): the coarse end of the V-cycle (the levels whose operators
 * and vectors fit in one CTA's shared memory) runs in one single-CTA launch;
 * 0: one launch per sweep.  The correction, and so the solve, is
 * bit-identical either way. */
int fs_proj_set_coarse_tail(void* handle, int on);
/* fp32 = 1: the mixed-precision form of the preconditioner (V-cycle
 * coefficients, vectors and coarse inverse in FP32); the CG itself, its
 * operator, residuals, dot products and the solution stay FP64, so the
 * tolerance still applies to the FP64 residual.  No counterpart in the
 * reference. */
int fs_proj_set_precision(void* handle, int fp32);
/* Host-side timings of the last fs_proj_project (ms): total, fetch waits
 * (sum, max), iteration launch calls (sum, max), then the number of fetches,
 * queued iterations and CG iterations (diagnostics; no reference counterpart). */
int fs_proj_stats(void* handle, double* out8);

/* Learned form (no counterpart in the reference): with net != NULL (a
 * fs_unet_create handle for the same grid; the context must be in the FP32
 * preconditioner form, fs_proj_set_precision(h, 1)) fs_proj_project runs
 * flexible CG truncated to one previous direction,
 *   z = M(r), p = z - (z.q_prev / p.q_prev) p_prev, q = S p,
 *   alpha = p.r / p.q, x += alpha p, r -= alpha q,
 * with the same stopping test.  M is a two-level cycle on the FP32 level-0
 * operator whose coarse correction is the network: nu damped-Jacobi sweeps
 * from 0 give t, r1 = r - S t, s = t + N(r1 / rms(r1)) rms(r1) c (c from
 * fs_unet_set_output_scale), then nu sweeps from s (nu and the damping of
 * fs_proj_configure).  When the residual norm shrinks by less than `stall`
 * per iteration (geometric mean of the last three) or after `max_learned`
 * iterations, the residual is recomputed and V-cycle PCG continues from the
 * current iterate (the fallback).  net = NULL restores V-cycle PCG. */
int fs_proj_set_learned(void* handle, void* net, int max_learned, double stall);
/* A training pair for the network from a logged solve (r0, e0 with
 * S e0 = r0, device doubles): r1 = r0 - S t and e1 = e0 - t after M's
 * pre-smoothing t, as device floats (FP32 form; the operator of the last
 * rebuild). */
int fs_proj_smooth_pair(void* handle, const double* r0, const double* e0, float* r1, float* e1,
                        void* stream);
/* Copy the residual and the iterate at the start of every solve into r0 and
 * x0 (device arrays of Nx*Ny*Nz doubles; both NULL turns it off).  The pair
 * (r0, x_solved - x0) solves S e = r0: the learned preconditioner's training
 * data. */
int fs_proj_set_log(void* handle, double* r0, double* x0);
/* Last solve: learned iterations, V-cycle iterations after a fallback, fell
 * back (0/1); then the number of fallbacks since creation. */
int fs_proj_fcg_stats(void* handle, double* out4);

/* The learned preconditioner: a 3-D conv U-Net (4 levels, 16/32/48/64
 * channels, bfloat16 activations, fp32 master weights, mma.sync tensor-core
 * convolutions), sized for one (nz, ny, nx) grid.  Parameters are a flat fp32
 * vector of fs_unet_nparams() values: per conv layer W[27][cin][cout] then
 * bias[cout], then the 1x1 head's w[16] and b. */
int64_t fs_unet_nparams(void);
int fs_unet_create(int nz, int ny, int nx, void** handle);
void fs_unet_destroy(void* handle);
/* host <-> device parameter copies (synchronous); set resets Adam's state */
int fs_unet_set_params(void* handle, const float* host, int64_t n, void* stream);
int fs_unet_get_params(void* handle, float* host, int64_t n, void* stream);
/* gradient of the last fs_unet_grad / fs_unet_train_step (synchronous) */
int fs_unet_get_grads(void* handle, float* host, int64_t n, void* stream);
/* c in the learned cycle's coarse correction N(r / rms(r)) rms(r) c (default
 * 1; 0 leaves only the smoothing sweeps) */
int fs_unet_set_output_scale(void* handle, float s);
/* z = N(r / rms(r)), device doubles */
int fs_unet_apply(void* handle, const double* r, double* z, void* stream);
/* z = N(r), device floats, no scaling */
int fs_unet_forward(void* handle, const float* r, float* z, void* stream);
/* mean squared error of N(r) against tau and its gradient (synchronous) */
int fs_unet_grad(void* handle, const float* r, const float* tau, double* loss, void* stream);
/* fs_unet_grad, then one Adam step (lr; betas 0.9, 0.999; eps 1e-8) */
int fs_unet_train_step(void* handle, const float* r, const float* tau, float lr, double* loss,
                       void* stream);
/* max |div(u) - target| to *result (synchronises); div_out optional. */
int fs_divergence_max(const FsGrid* g, const double* u, const double* v, const double* w,
                      const double* u_inlet, const double* div_target, double* div_out,
                      double* result, void* stream);

/* dom_3d.py:230 DOMRadiationSolver: create (ordinates/weights host arrays),
 * :286 solve (synchronises once per source iteration). */
int fs_dom_create(const FsGrid* g, int M, const double* ox, const double* oy, const double* oz,
                  const double* w, double kappa_gas_max, void** handle);
void fs_dom_destroy(void* handle);
int fs_dom_solve(void* handle, const double* T_s, const double* T_g, const double* alpha_s,
                 const double* omega, double sigma_sav, double T_amb, const double* T_soil0,
                 const double* Y_H2O, const double* rho, const double* M_local, double* q_rad_solid,
                 double* q_rad_gas, double* q_in_soil, void* stream);
/* fs_dom_solve in two halves (no counterpart in the reference, which solves
 * in one call): fs_dom_begin reads the fields (absorption, emission, ground
 * emission) and fs_dom_end runs the source iterations and writes the
 * radiative sources.  Once fs_dom_begin's work has run on its stream the
 * solve reads none of its input fields again, so other streams may update
 * them while fs_dom_end runs; the result is that of fs_dom_solve. */
int fs_dom_begin(void* handle, const double* T_s, const double* T_g, const double* alpha_s,
                 const double* omega, double sigma_sav, double T_amb, const double* T_soil0,
                 const double* Y_H2O, const double* rho, const double* M_local, void* stream);
int fs_dom_end(void* handle, double* q_rad_solid, double* q_rad_gas, double* q_in_soil,
               void* stream);
/* Full intensity field (M x Nz x Ny x Nx) for sweep path 3; NULL for the
 * default octant-cluster path, which keeps only the y-periodic inflow rows
 * (the part of I_set that a later sweep reads, dom_3d.py:147-211). */
double* fs_dom_intensity(void* handle);
/* Sweep path: 0 auto (path 8 when the quadrature is octant-major and a
 * cluster shape fits the grid, else path 3), 3 one launch per hyperplane
 * over all ordinates with the full intensity field stored (any quadrature,
 * FP64 only), 8 octant clusters: one thread-block cluster per octant (or per
 * half of its ordinates), the cluster's CTAs splitting the k' rows and
 * handing each hyperplane's last row to the next CTA through a ring in its
 * shared memory, one or two pencils per thread, planned so that all
 * clusters are resident at once where the part allows it; cluster_ctas 0 =
 * automatic, else CTAs per octant (1..16).  Only before the first solve or
 * intensity load.  Path 8 computes the numerator with fused multiply-adds
 * and the quotient from a Newton-Raphson reciprocal (within about one ulp),
 * so its FP64 results differ from path 3's by rounding only. */
int fs_dom_set_sweep_mode(void* handle, int mode, int cluster_ctas);
/* Path 8 only: clusters per octant, 1 (all ordinates of the octant in one
 * cluster) or 2 (half each, the octant partials of G then summed per half);
 * 0 (default) plans it.  Only before the first solve or intensity load. */
int fs_dom_set_octant_groups(void* handle, int groups);
/* The path in use (0 before the first solve or intensity load). */
int fs_dom_sweep_mode(void* handle);
/* Path 8's kernel: 1 one pencil per thread (a hyperplane's intensities pass
 * through shared memory, one barrier over all pencil warps; the default, also
 * for 0), 2 lane column (a lane owns one y column of all of the CTA's k' rows
 * and keeps their intensities in registers, y-neighbours by warp shuffles;
 * built for ten ordinates per cluster, 4 to 8 rows per CTA and ny <= 128;
 * FS_EARG at the first solve for other shapes).  Both give the same results
 * bit for bit; the lane-column kernel is the slower one on the S8 workload
 * (3.85 ms per FP64 sweep at 400 x 120 x 60, about twice the other).  Only before the
 * first solve or intensity load.  fs_dom_sweep_kernel: the kernel in use (0
 * before the path is resolved or on path 3). */
int fs_dom_set_sweep_kernel(void* handle, int kernel);
int fs_dom_sweep_kernel(void* handle);
/* The division by a run-time invariant divisor that the kernels use to split
 * a flat cell index into (i, j, k): q[t] = x[t] / d for t < n, computed on the
 * host by the same multiply-high formula.  FS_EARG for d == 0 or n < 0. */
int fs_index_divide(uint32_t d, int64_t n, const uint32_t* x, uint32_t* q);
/* Test switch for the bounded waits of path 8's row hand-off: with plane >= 0
 * the first CTA of every octant cluster withholds its ring fill of that
 * hyperplane, so the next CTA's wait for it runs out; the sweep then stops
 * all hand-off traffic, every CTA finishes, and the solve returns
 * FS_ETIMEOUT with the object still usable.  plane < 0 (the default) turns
 * it off.  No counterpart in the reference. */
int fs_dom_set_wait_test(void* handle, int plane);
/* Path 8's launch shape, once the path is resolved: out[0] CTAs per cluster,
 * out[1] k' rows per CTA, out[2] threads per CTA, out[3] dynamic shared
 * memory per CTA in bytes, out[4] clusters (ordinate groups) per octant.
 * FS_EARG before the first solve or when another path is in use. */
int fs_dom_launch_shape(void* handle, int* out5);
/* fp32 = 1: the mixed-precision form of the sweep (path 8 with kappa,
 * kappa*B, intensities and octant partials in FP32 and the quotient of
 * __fdividef, about 2 ulp; G, the ground exchange and all outputs in FP64).
 * No counterpart in the reference, which is FP64 throughout.  Only before the
 * first solve or intensity load. */
int fs_dom_set_precision(void* handle, int fp32);
/* Load the persistent intensity state from a full device field
 * (M x Nz x Ny x Nx), as a reference I_set would seed the next solve. */
int fs_dom_load_intensity(void* handle, const double* I_full, void* stream);
/* The persistent DOM state for checkpoints: the y-periodic inflow rows
 * (M x Nz x Nx doubles, device memory), read out of or written into
 * whichever storage the sweep path uses.  The reference keeps the whole
 * I_set between calls (dom_3d.py:286-300); these rows are the part of it a
 * later sweep reads. */
int64_t fs_dom_wrap_size(void* handle);
int fs_dom_get_wrap(void* handle, double* dst, void* stream);
int fs_dom_set_wrap(void* handle, const double* src, void* stream);
int fs_dom_iterations(void* handle);
/* enable >= 0 turns per-sweep event timing on/off (and resets it); the
 * accumulated sweep time and sweep count are returned when pointers are given */
int fs_dom_sweep_timing(void* handle, int enable, double* total_ms, long long* sweeps);

/* lagrangian_bed_3d.py:594 step_bed_particles (sources overwritten only in
 * occupied cells; zero the grids once), :501 aggregate_particles_to_T_s_grid
 * (mode 0) and :550 aggregate_particles_to_M_local_grid (mode 1), :428
 * step_horizontal_solid_conduction_scatter (T_s in place; scratch of
 * n_z_bed*Ny*Nx doubles). */
int fs_bed_step(const FsGrid* g, const FsBedParticles* p, const FsBedSegments* s,
                const FsBedSources* o, const FsBedParams* prm, const double* T_g,
                const double* Y_O2, void* stream);
int fs_bed_aggregate(const FsBedParticles* p, const FsBedSegments* s, double* out, int mode,
                     void* stream);
int fs_bed_hcond(const FsGrid* g, double* T_s_grid, double* scratch, const double* alpha_s,
                 int n_z_bed, double k_solid, double rho_true, double cp_solid, double dt,
                 const FsBedParticles* p, const FsBedSegments* s, const int* seg_of_cell,
                 void* stream);

/* flame_front_3d.py:114 godunov_grad_norm (mode 0), :332 evolve (mode 1,
 * aux = v_n, coef = dt), one :339 reinitialize sub-step (mode 2,
 * aux = phi_0, coef = dtau); out-of-place. */
int fs_levelset(const FsGrid* g, const double* phi, const double* aux, double* out, double coef,
                int mode, void* stream);
/* flame_front_3d.py:756-813 active-flame mask and its cell count (device
 * counter, accumulated). */
int fs_active_count(int64_t n, const double* omega, const double* T_g, const double* Y_F,
                    unsigned long long* count, unsigned char* mask, void* stream);

/* Copy device bytes to host memory and wait (the thread sleeps on a
 * blocking-sync event rather than spinning).  Host-side reads of the
 * reference loop's scalars (active-flame count, front row) go through it. */
int fs_copy_to_host(void* dst, const void* src, int64_t bytes, void* stream);
/* max reductions: mode 0 max|f|, 1 max f (NaN propagates), 2 interior max
 * ignoring NaN from 0 (turbulence_3d.py:894-900); results to host.  The
 * synchronous reductions (this, fs_field_max_multi, fs_divergence_max) stage
 * through per-thread device words and pinned memory made on a thread's first
 * call, so threads that step different cases on their own streams may call
 * them at the same time. */
int fs_field_max(const FsGrid* g, const double* f, int mode, double* result, void* stream);
/* several maxima in one pass; scratch: >= 256 bytes of device memory;
 * results: nf doubles in host memory (synchronises once). */
int fs_field_max_multi(const FsGrid* g, int nf, const double* const* f, const int* modes,
                       double* results, void* scratch, void* stream);

/* ---- Whole steps ----------------------------------------------------------
 * The outer loop of run_3d_spread (spread_3d.py:1897-3512) in the
 * production configuration (Lagrangian bed, k-epsilon, EDC, DOM, passive
 * level set, periodic y, log-law inlet), operator by operator in the
 * reference's order, device-resident and driven from C++: the host only
 * reads back the scalars the loop branches on (dt, the pressure-iteration
 * test, the DOM source-iteration test, the turbulent-diffusion sub-step
 * count, the exit tests).  The context owns every buffer (state, workspaces,
 * the projection's and the DOM's solver objects) and frees them in
 * fs_ctx_destroy.  One context is driven by one host thread at a time; the
 * DOM solve runs on a second stream from a worker thread of the context.
 * No counterpart in the reference as a C call. */
typedef struct FsCaseDesc {
  /* grid (Grid3D, spread_3d.py:158-188); dz, d_above, d_below: host arrays of nz */
  int nx, ny, nz, n_z_bed;
  double dx, dy;
  const double *dz, *d_above, *d_below;
  /* constants of the case (spread_3d.py:563-1500), as resolved from its deck */
  double T_amb, h_bed, sav, cfl, dz_min, U_mf, min_dt_s, dt0;
  double ignition_duration_s, ignition_q_mult, canopy_C_d, canopy_beta_p, canopy_beta_d;
  double h_conv, rho_solid_true, cp_solid, eps_solid, view_factor, kappa_bed_eff;
  double char_ox_flux_cap, char_ox_ash_exp, chi_rad, T_ign, proj_div_tol, x_front0, bed_x_end;
  int drying_mode, view_factor_geometric, n_per_cell, i_src_start, i_src_end;
  int proj_max_iter, dom_subcycle_every, edc_extinction_enable;
  /* DOM quadrature: M ordinates (host arrays) */
  int M;
  const double *ox, *oy, *oz, *w;
  /* soil column (soil_3d.py:73-103): host arrays of n_soil */
  int n_soil;
  const double *soil_dz, *soil_d_above, *soil_d_below;
  /* solver options: form 0 plain FP64, 1 mixed (FP32 DOM sweep, V-cycle and
   * chemistry/transport sub-steps);
   * the CG tolerance and iteration cap of each pressure solve; overlap_dom 1
   * runs the DOM solve on a second stream concurrently with momentum, the
   * projection and k-epsilon (results identical either way) */
  int form;
  double projection_rtol;
  int proj_maxiter;
  int overlap_dom;
} FsCaseDesc;

/* Initial state, host arrays (C-order (nz, ny, nx) unless noted). */
typedef struct FsInitState {
  const double *rho, *u, *v, *w, *T_g, *Y_fuel, *Y_O2, *Y_H2O, *T_s, *alpha_s, *k_turb,
      *eps_turb, *nu_t, *phi;
  const double* u_inlet; /* (nz, ny) */
  const double* sigma_x; /* (nx) outflow sponge */
  const double* T_soil;  /* (n_soil, ny, nx) */
  int64_t n_particles;
  const double *px, *py, *pz, *m_solid, *m_water, *m_char, *pT_s, *m_water_0, *psav,
      *m_char_max;
  const signed char* alive;
} FsInitState;

typedef struct FsStepOut {
  int steps;          /* outer steps taken by this call */
  int finished;       /* 1 once the loop's exit tests fired (spread_3d.py:3413-3437) */
  int64_t step_count; /* steps since creation */
  double t, dt;       /* clock after the last step and that step's dt */
  int cg_iters;       /* CG iterations of the last step (all its pressure solves) */
  int proj_iters;     /* pressure iterations of the last step */
  int dom_iters;      /* DOM source iterations of the last step */
  double div_max;     /* last max |div u - div_target| */
} FsStepOut;

/* State and work fields of a context, for fs_ctx_field / fs_ctx_read /
 * fs_ctx_write.  Cell fields hold nx*ny*nz doubles, FS_F_T_SOIL
 * n_soil*ny*nx, particle fields n_particles doubles (FS_P_ALIVE bytes). */
enum {
  FS_F_RHO = 0, FS_F_U, FS_F_V, FS_F_W, FS_F_T_G, FS_F_Y_FUEL, FS_F_Y_O2, FS_F_Y_H2O,
  FS_F_T_S, FS_F_ALPHA_S, FS_F_K_TURB, FS_F_EPS_TURB, FS_F_NU_T, FS_F_PHI,
  FS_F_OMEGA, FS_F_Q_RAD, FS_F_Q_RAD_GAS, FS_F_M_LOCAL, FS_F_S_PYRO, FS_F_S_DRYING,
  FS_F_Q_G_CONV, FS_F_Q_COMB, FS_F_PRESSURE, FS_F_T_SOIL,
  FS_P_X, FS_P_Y, FS_P_Z, FS_P_M_SOLID, FS_P_M_WATER, FS_P_M_CHAR, FS_P_T_S, FS_P_M_WATER_0,
  FS_P_SAV, FS_P_M_CHAR_MAX, FS_P_ALIVE,
  FS_FIELD_COUNT
};

typedef struct FsCtx FsCtx;
int fs_ctx_create(const FsCaseDesc* desc, const FsInitState* init, FsCtx** out);
void fs_ctx_destroy(FsCtx* ctx);
/* the context's last error message (the thread's fs_last_error() as well) */
const char* fs_ctx_last_error(FsCtx* ctx);
/* n_steps outer steps, fewer if the exit tests fire; out may be NULL */
int fs_step(FsCtx* ctx, int n_steps, FsStepOut* out);
/* n_steps outer steps of every context, each on its own host thread and
 * streams at the same time (cases share nothing); outs[i] (may be NULL)
 * receives context i's summary.  Returns the first failing status. */
int fs_batch_run(FsCtx* const* ctxs, int n, int n_steps, FsStepOut* outs);
/* number of elements of a field (-1 for an unknown id) */
int64_t fs_ctx_field_size(FsCtx* ctx, int id);
/* current device buffer of a field (valid until the next fs_step) */
void* fs_ctx_field(FsCtx* ctx, int id);
/* copy a field to / from host memory (synchronous) */
int fs_ctx_read(FsCtx* ctx, int id, void* host_dst);
int fs_ctx_write(FsCtx* ctx, int id, const void* host_src);
/* the context's main stream (every fs_step launch is ordered on it) */
void* fs_ctx_stream(FsCtx* ctx);

#ifdef __cplusplus
}
#endif
#endif
