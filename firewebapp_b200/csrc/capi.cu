// extern "C" entry points of libfirestep.so (declared in include/firestep.h).
#include <cstdarg>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <thread>
#include "common.cuh"
#include "kernels.h"

#include <atomic>

static thread_local char g_err[512] = "";
// set when a message was written since the last status check consumed one, so
// that check() keeps a specific message instead of a generic one
static thread_local bool g_err_fresh = false;
static std::atomic<unsigned long long> g_launches{0};

void fs_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void fs_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  g_err_fresh = true;
}

// Host wait for a stream through a blocking-sync event: the calling thread
// sleeps instead of spinning, so waits do not consume the process's CPU time
// (spinning threads can get a CPU-quota-limited process throttled).
// Wait for a stream: poll an event (yielding the core between polls) for up
// to FS_SPIN_US microseconds, then sleep on a blocking-sync event recorded at
// the same point.  The step's host decisions wait on queues of 0.01-15 ms (a
// reduction, a CG batch, the DOM's queued source iterations), and the work
// queued after a wait starts only when the host wakes; longer waits (a
// stalled device) still sleep.
#define FS_SPIN_US 50000
int fs_stream_wait(cudaStream_t st) {
  static thread_local cudaEvent_t ev_poll[64] = {};
  static thread_local cudaEvent_t ev_block[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FS_ECUDA;
  if (!ev_poll[dev] &&
      cudaEventCreateWithFlags(&ev_poll[dev], cudaEventDisableTiming) != cudaSuccess)
    return FS_ECUDA;
  if (!ev_block[dev] && cudaEventCreateWithFlags(&ev_block[dev], cudaEventBlockingSync |
                                                                     cudaEventDisableTiming) !=
                            cudaSuccess)
    return FS_ECUDA;
  if (cudaEventRecord(ev_poll[dev], st) != cudaSuccess) return FS_ECUDA;
  if (cudaEventRecord(ev_block[dev], st) != cudaSuccess) return FS_ECUDA;
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    const cudaError_t q = cudaEventQuery(ev_poll[dev]);
    if (q == cudaSuccess) return FS_OK;
    if (q != cudaErrorNotReady) return FS_ECUDA;
    if (std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(FS_SPIN_US)) break;
    std::this_thread::yield();
  }
  return cudaEventSynchronize(ev_block[dev]) == cudaSuccess ? FS_OK : FS_ECUDA;
}

// Per-thread, per-device scratch for the synchronous reductions (a few device
// words and a pinned host staging area), made on a thread's first call, so the
// hot-path reductions neither allocate per call nor copy into pageable memory,
// and threads that step different cases on different streams never wait for
// each other's streams.
struct SmallScratch {
  unsigned long long* dkey;  // 32 words
  double* dres;              // 32 doubles
  double* hpin;              // 32 doubles, pinned
};
static thread_local SmallScratch g_small[64];

static SmallScratch* small_scratch() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  SmallScratch& sc = g_small[dev];
  if (!sc.dkey) {
    void* p = nullptr;
    if (cudaMalloc(&p, 64 * sizeof(double)) != cudaSuccess) return nullptr;
    void* h = nullptr;
    if (cudaMallocHost(&h, 32 * sizeof(double)) != cudaSuccess) {
      cudaFree(p);
      return nullptr;
    }
    sc.dkey = (unsigned long long*)p;
    sc.dres = (double*)p + 32;
    sc.hpin = (double*)h;
  }
  return &sc;
}

static int check(int st, const char* where) {
  if (st == FS_OK) {
    g_err_fresh = false;
    return st;
  }
  cudaError_t e = cudaGetLastError();
  if (g_err_fresh && st != FS_ECUDA && strncmp(g_err, where, strlen(where)) != 0) {
    // the failing function said what was wrong: keep it, naming the entry point
    char inner[sizeof(g_err)];
    memcpy(inner, g_err, sizeof(g_err));
    fs_set_error("%s: %s", where, inner);
  } else if (g_err_fresh && st != FS_ECUDA) {
    // already names the entry point
  } else if (st == FS_ECUDA)
    fs_set_error("%s: CUDA error: %s", where, cudaGetErrorString(e));
  else if (st == FS_EARG)
    fs_set_error("%s: bad argument", where);
  else if (st == FS_ENONFINITE)
    fs_set_error("%s: non-finite value", where);
  else if (st == FS_ENOCONV)
    fs_set_error("%s: solver did not converge", where);
  else if (st == FS_ETIMEOUT)
    fs_set_error("%s: a bounded device wait gave up (results of that call not valid)", where);
  else
    fs_set_error("%s: status %d", where, st);
  g_err_fresh = false;
  return st;
}

static bool to_grid(const FsGrid* g, GridDev& d, const char* where) {
  if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1 || !g->dz || !g->d_above || !g->d_below ||
      !(g->dx > 0.0) || !(g->dy > 0.0)) {
    fs_set_error("%s: invalid grid", where);
    return false;
  }
  if ((long long)g->nx * g->ny * g->nz >= (1ll << 31)) {
    fs_set_error("%s: grid of %lld cells (at most 2^31 - 1)", where,
                 (long long)g->nx * g->ny * g->nz);
    return false;
  }
  d.nx = g->nx; d.ny = g->ny; d.nz = g->nz; d.dx = g->dx; d.dy = g->dy;
  d.dz = g->dz; d.da = g->d_above; d.db = g->d_below;
  d.fnx = fastdiv_make((uint32_t)g->nx);
  d.fny = fastdiv_make((uint32_t)g->ny);
  return true;
}

#define ST(s) ((cudaStream_t)(s))
#define GRID(name)                           \
  GridDev gd;                                \
  if (!to_grid(g, gd, name)) return FS_EARG;

extern "C" {

const char* fs_last_error(void) { return g_err; }
int fs_version(void) { return 1; }
unsigned long long fs_launch_count(void) { return g_launches.load(); }

int fs_species_transport(const FsGrid* g, int nspec, const double* const* Y, double* const* Y_out,
                         const double* const* S, const double* Y_inlet, const double* rho,
                         const double* u, const double* v, const double* w, double dt, double D,
                         void* stream) {
  GRID("fs_species_transport");
  if (!Y || !Y_out || !S || !Y_inlet || nspec < 1 || nspec > 3) {
    fs_set_error("fs_species_transport: bad species arguments");
    return FS_EARG;
  }
  return check(launch_species(gd, nspec, Y, Y_out, S, Y_inlet, rho, u, v, w, dt, D, ST(stream)),
               "fs_species_transport");
}

int fs_species_step(const FsGrid* g, const double* const* Y, double* const* Y_out,
                    const double* S_pyro, const double* S_drying, const double* Y_inlet,
                    const double* rho, const double* u, const double* v, const double* w,
                    double dt, double D, double o2_cap, void* stream) {
  GRID("fs_species_step");
  if (!Y || !Y_out || !S_pyro || !S_drying || !Y_inlet) {
    fs_set_error("fs_species_step: bad species arguments");
    return FS_EARG;
  }
  return check(launch_species_step(gd, Y, Y_out, S_pyro, S_drying, Y_inlet, rho, u, v, w, dt, D,
                                   o2_cap, ST(stream)),
               "fs_species_step");
}

int fs_species_sources(int64_t n, const double* S_pyro, const double* S_drying, const double* Y_F,
                       const double* Y_O2, const double* Y_H2O, double* S_F, double* S_O2,
                       double* S_H2O, void* stream) {
  if (n < 0) return FS_EARG;
  return check(launch_species_sources(n, S_pyro, S_drying, Y_F, Y_O2, Y_H2O, S_F, S_O2, S_H2O,
                                      ST(stream)),
               "fs_species_sources");
}

int fs_advect_scalar_muscl(const FsGrid* g, const double* phi, const double* u, const double* v,
                           const double* w, double* rhs, double phi_inlet, void* stream) {
  GRID("fs_advect_scalar_muscl");
  return check(launch_advect_scalar(gd, phi, u, v, w, rhs, phi_inlet, ST(stream)),
               "fs_advect_scalar_muscl");
}

int fs_gas_energy_adv(const FsGrid* g, const double* T_g, const double* u, const double* v,
                      const double* w, double* T_out, double dt, double alpha_th, double T_amb,
                      void* stream) {
  GRID("fs_gas_energy_adv");
  return check(launch_gas_energy_adv(gd, T_g, u, v, w, T_out, dt, alpha_th, T_amb, ST(stream)),
               "fs_gas_energy_adv");
}

int fs_copy_to_host(void* dst, const void* src, int64_t bytes, void* stream) {
  if (!dst || !src || bytes < 0) return FS_EARG;
  if (cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost, ST(stream)) != cudaSuccess)
    return check(FS_ECUDA, "fs_copy_to_host");
  return check(fs_stream_wait(ST(stream)), "fs_copy_to_host");
}

int fs_field_max(const FsGrid* g, const double* f, int mode, double* result, void* stream) {
  GRID("fs_field_max");
  SmallScratch* sc = small_scratch();
  if (!sc) {
    fs_set_error("fs_field_max: scratch allocation failed");
    return FS_ECUDA;
  }
  launch_init_keys(sc->dkey, 1, mode == 2 ? 1 : 0, ST(stream));
  launch_max(gd, f, mode, sc->dkey, ST(stream));
  launch_keys_to_double(sc->dkey, sc->dres, 1, ST(stream));
  cudaMemcpyAsync(sc->hpin, sc->dres, sizeof(double), cudaMemcpyDeviceToHost, ST(stream));
  if (fs_stream_wait(ST(stream)) != FS_OK) return check(FS_ECUDA, "fs_field_max");
  *result = sc->hpin[0];
  return check(cuda_status(), "fs_field_max");
}

int fs_field_max_multi(const FsGrid* g, int nf, const double* const* f, const int* modes,
                       double* results, void* scratch, void* stream) {
  GRID("fs_field_max_multi");
  if (nf < 1 || nf > 16 || !scratch) return FS_EARG;
  unsigned long long* key = (unsigned long long*)scratch;
  double* dres = (double*)(key + 16);
  int mask2 = 0;
  for (int q = 0; q < nf; ++q)
    if (modes[q] == 2) mask2 |= 1 << q;
  launch_init_keys(key, nf, mask2, ST(stream));
  for (int q = 0; q < nf; ++q) launch_max(gd, f[q], modes[q], key + q, ST(stream));
  launch_keys_to_double(key, dres, nf, ST(stream));
  SmallScratch* sc = small_scratch();
  if (!sc) {
    fs_set_error("fs_field_max_multi: scratch allocation failed");
    return FS_ECUDA;
  }
  cudaMemcpyAsync(sc->hpin, dres, sizeof(double) * nf, cudaMemcpyDeviceToHost, ST(stream));
  if (fs_stream_wait(ST(stream)) != FS_OK) return check(FS_ECUDA, "fs_field_max_multi");
  for (int q = 0; q < nf; ++q) results[q] = sc->hpin[q];
  return check(cuda_status(), "fs_field_max_multi");
}

int fs_turb_diffusion_nsub(const FsGrid* g, const double* nu_t, double sc_t, double dt,
                           int* n_sub, double* dt_sub, void* stream) {
  GRID("fs_turb_diffusion_nsub");
  // turbulence_3d.py:880-915
  double dz_min = 0.0;
  {
    double* h = nullptr;
    if (cudaMallocHost(&h, sizeof(double) * gd.nz) != cudaSuccess) return check(FS_ECUDA, "nsub");
    cudaMemcpyAsync(h, gd.dz, sizeof(double) * gd.nz, cudaMemcpyDeviceToHost, ST(stream));
    if (fs_stream_wait(ST(stream)) != FS_OK) {
      cudaFreeHost(h);
      return check(FS_ECUDA, "nsub");
    }
    dz_min = h[0];
    for (int k = 1; k < gd.nz; ++k)
      if (h[k] < dz_min) dz_min = h[k];
    cudaFreeHost(h);
  }
  double dx2 = gd.dx * gd.dx, dy2 = gd.dy * gd.dy, dz2 = dz_min * dz_min;
  double h_min2 = dx2 < (dy2 < dz2 ? dy2 : dz2) ? dx2 : (dy2 < dz2 ? dy2 : dz2);
  double nu_max = 0.0;
  int st = fs_field_max(g, nu_t, 2, &nu_max, stream);
  if (st) return st;
  *n_sub = 0;
  *dt_sub = 0.0;
  double D_max = nu_max / sc_t;
  if (D_max <= 1.0e-12) return FS_OK;
  if (!(D_max - D_max == 0.0)) return FS_OK;  // non-finite: skipped
  double dt_sub_max = 0.4 * h_min2 / D_max;
  if (dt_sub_max <= 0.0) return FS_OK;
  double target = dt / dt_sub_max;
  if (target > 1000.0) return FS_OK;
  int n = (int)ceil(target);
  if (n < 1) n = 1;
  *n_sub = n;
  *dt_sub = dt / n;
  return FS_OK;
}

int fs_turb_diffusion_substep(const FsGrid* g, int nfield, const double* const* f,
                              double* const* f_out, const double* nu_t, double sc_t, double dt_sub,
                              int clip, const double* lo, const double* hi, void* stream) {
  GRID("fs_turb_diffusion_substep");
  return check(launch_turb_diff(gd, nfield, f, f_out, nu_t, sc_t, dt_sub, clip, lo, hi,
                                ST(stream)),
               "fs_turb_diffusion_substep");
}

int fs_drag_force(int64_t n, const double* u, const double* v, const double* w, const double* rho,
                  const double* alpha_s, double sigma_sav, double C_D, double* Fx, double* Fy,
                  double* Fz, void* stream) {
  return check(launch_drag(n, u, v, w, rho, alpha_s, sigma_sav, C_D, Fx, Fy, Fz, ST(stream)),
               "fs_drag_force");
}

int fs_tentative_velocity(const FsGrid* g, const double* u, const double* v, const double* w,
                          const double* rho, const double* T_g, const double* Fx, const double* Fy,
                          const double* Fz, const double* alpha_s, double sigma_sav, double C_D,
                          const double* u_inlet, const double* v_inlet, const double* w_inlet,
                          double* u_out, double* v_out, double* w_out, double dt, double T_amb,
                          void* stream) {
  GRID("fs_tentative_velocity");
  return check(launch_momentum(gd, u, v, w, rho, T_g, Fx, Fy, Fz, alpha_s, sigma_sav, C_D, u_inlet,
                               v_inlet, w_inlet, u_out, v_out, w_out, dt, T_amb, ST(stream)),
               "fs_tentative_velocity");
}

int fs_outflow_sponge(const FsGrid* g, double* u, const double* u_target, const double* sigma_x,
                      const double* Y_F, double Y_F_skip, double dt, void* stream) {
  GRID("fs_outflow_sponge");
  return check(launch_sponge(gd, u, u_target, sigma_x, Y_F, Y_F_skip, dt, ST(stream)),
               "fs_outflow_sponge");
}

int fs_k_epsilon(const FsGrid* g, const double* k, const double* eps, const double* u,
                 const double* v, const double* w, const double* T_g, const double* alpha_s,
                 const double* u_inlet, const double* k_wall, const double* eps_wall, double* k_out,
                 double* eps_out, double* nu_t_out, double* S2_out, double* O2_out,
                 double sigma_sav, double dt, double T_amb, double beta_p, double beta_d,
                 void* stream) {
  GRID("fs_k_epsilon");
  return check(launch_keps(gd, k, eps, u, v, w, T_g, alpha_s, u_inlet, k_wall, eps_wall, k_out,
                           eps_out, nu_t_out, S2_out, O2_out, sigma_sav, dt, T_amb, beta_p, beta_d,
                           ST(stream)),
               "fs_k_epsilon");
}

int64_t fs_edc_scratch_bytes(int64_t n) { return (int64_t)edc_scratch_bytes(n); }

int fs_edc(int64_t n, const double* rho, double* T_g, double* Y_F, double* Y_O2, const double* k,
           const double* eps, const double* Y_H2O, double* omega, double chi_rad, double cp_g,
           double dt, int n_substeps, double s_stoich, double hoc_J, int extinction, void* scratch,
           void* stream) {
  if (n < 0 || !scratch) {
    fs_set_error("fs_edc: bad argument");
    return FS_EARG;
  }
  if (n == 0) return FS_OK;
  return check(launch_edc(n, rho, T_g, Y_F, Y_O2, k, eps, Y_H2O, omega, chi_rad, cp_g, dt,
                          n_substeps, s_stoich, hoc_J, extinction, scratch, ST(stream)),
               "fs_edc");
}

int fs_gas_energy_update(const FsGrid* g, double* T_g, const double* rho, const double* Y_H2O,
                         const double* T_s, const double* S_pyro, const double* S_drying,
                         const double* Q_g_conv, const double* q_rad_gas, double* Q_comb_out,
                         double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                         int i_src0, int i_src1, void* stream) {
  GRID("fs_gas_energy_update");
  return check(launch_gas_update(gd, T_g, rho, Y_H2O, T_s, S_pyro, S_drying, Q_g_conv, q_rad_gas,
                                 Q_comb_out, nullptr, dt_sub, T_amb, h_bed, drip_on, n_z_bed,
                                 i_src0, i_src1, ST(stream)),
               "fs_gas_energy_update");
}

int fs_gas_energy_solid_update(const FsGrid* g, double* T_g, const double* rho,
                               const double* Y_H2O, const double* T_s, const double* S_pyro,
                               const double* S_drying, const double* Q_g_conv,
                               const double* q_rad_gas, double* Q_comb_out, double dt_sub,
                               double T_amb, double h_bed, int drip_on, int n_z_bed, int i_src0,
                               int i_src1, const double* alpha_s, double* T_s_out,
                               double k_solid, double rho_solid, double cp_solid, double Ts_lo,
                               double Ts_hi, void* stream) {
  GRID("fs_gas_energy_solid_update");
  if (!T_s || !T_s_out || T_s_out == T_s || !alpha_s) {
    fs_set_error("fs_gas_energy_solid_update: T_s_out must be a buffer other than T_s");
    return FS_EARG;
  }
  return check(launch_gas_solid(gd, T_g, rho, Y_H2O, T_s, S_pyro, S_drying, Q_g_conv, q_rad_gas,
                                Q_comb_out, dt_sub, T_amb, h_bed, drip_on, n_z_bed, i_src0,
                                i_src1, alpha_s, T_s_out, k_solid, rho_solid, cp_solid, Ts_lo,
                                Ts_hi, ST(stream)),
               "fs_gas_energy_solid_update");
}

int fs_eos(const FsGrid* g, double* rho, double* rho_prev, const double* T_g, double* Y_O2,
           double T_amb, void* stream) {
  GRID("fs_eos");
  const double R_air = 8.314 / 0.029;
  return check(launch_eos(gd, rho, rho_prev, T_g, Y_O2, 101325.0, R_air, T_amb, ST(stream)),
               "fs_eos");
}

int fs_div_target(int64_t n, const double* rho, const double* rho_prev, const double* S_pyro,
                  const double* S_drying, double dt, double* div_target, void* stream) {
  if (n < 0 || !(dt > 0.0) || (n > 0 && (!rho || !rho_prev || !S_pyro || !S_drying ||
                                         !div_target))) {
    fs_set_error("fs_div_target: bad argument");
    return FS_EARG;
  }
  return check(launch_div_target(n, rho, rho_prev, S_pyro, S_drying, dt, div_target, ST(stream)),
               "fs_div_target");
}

int fs_ignition_pulse(const FsGrid* g, double* q_rad, int k, int i0, int i1, double q_add,
                      void* stream) {
  GRID("fs_ignition_pulse");
  if (!q_rad || k < 0 || k >= gd.nz || i0 < 0 || i1 > gd.nx || i0 > i1) {
    fs_set_error("fs_ignition_pulse: bad argument (k=%d, i0=%d, i1=%d)", k, i0, i1);
    return FS_EARG;
  }
  return check(launch_ignition_pulse(gd, q_rad, k, i0, i1, q_add, ST(stream)),
               "fs_ignition_pulse");
}

int fs_stencil_status(int clear) { return stencil_status(clear); }

int fs_set_tma(int on) {
  set_tma(on);
  return FS_OK;
}

// ---- single-precision sub-step kernels (mixed-precision form) ----
int fs_convert(int64_t n, int nf, const void* const* src, void* const* dst, int to_f32,
               void* stream) {
  if (!src || !dst || n < 0 || nf < 1 || nf > 16) {
    fs_set_error("fs_convert: bad argument");
    return FS_EARG;
  }
  return check(launch_convert(n, nf, src, dst, to_f32, ST(stream)), "fs_convert");
}

int64_t fs_edc_f32_scratch_bytes(int64_t n) { return n < 0 ? -1 : edc32_scratch_bytes(n); }

int fs_edc_f32(int64_t n, const float* rho, float* T_g, float* Y_F, float* Y_O2, const float* k,
               const float* eps, const float* Y_H2O, float* omega, double chi_rad, double cp_g,
               double dt, int n_substeps, double s_stoich, double hoc_J, int extinction,
               void* scratch, void* stream) {
  if (n < 0 || !scratch) {
    fs_set_error("fs_edc_f32: bad argument");
    return FS_EARG;
  }
  return check(launch_edc32(n, rho, T_g, Y_F, Y_O2, k, eps, Y_H2O, omega, chi_rad, cp_g, dt,
                            n_substeps, s_stoich, hoc_J, extinction, scratch, ST(stream)),
               "fs_edc_f32");
}

int fs_species_step_f32(const FsGrid* g, const float* const* Y, float* const* Y_out,
                        const float* S_pyro, const float* S_drying, const double* Y_inlet,
                        const float* rho, const float* u, const float* v, const float* w,
                        double dt, double D, double o2_cap, void* stream) {
  GRID("fs_species_step_f32");
  if (!Y || !Y_out || !S_pyro || !S_drying || !Y_inlet) {
    fs_set_error("fs_species_step_f32: bad species arguments");
    return FS_EARG;
  }
  return check(launch_species_step32(gd, Y, Y_out, S_pyro, S_drying, Y_inlet, rho, u, v, w, dt,
                                     D, o2_cap, ST(stream)),
               "fs_species_step_f32");
}

int fs_turb_diffusion_substep_f32(const FsGrid* g, int nfield, const float* const* f,
                                  float* const* f_out, const float* nu_t, double sc_t,
                                  double dt_sub, int clip, const double* lo, const double* hi,
                                  void* stream) {
  GRID("fs_turb_diffusion_substep_f32");
  if (!f || !f_out || (clip && (!lo || !hi))) {
    fs_set_error("fs_turb_diffusion_substep_f32: bad argument");
    return FS_EARG;
  }
  return check(launch_turb_diff32(gd, nfield, f, f_out, nu_t, sc_t, dt_sub, clip, lo, hi,
                                  ST(stream)),
               "fs_turb_diffusion_substep_f32");
}

int fs_gas_energy_update_f32(const FsGrid* g, float* T_g, const float* rho, const float* Y_H2O,
                             const double* T_s, const float* S_pyro, const float* S_drying,
                             const float* Q_g_conv, const double* q_rad_gas, float* Q_comb_out,
                             double dt_sub, double T_amb, double h_bed, int drip_on, int n_z_bed,
                             int i_src0, int i_src1, void* stream) {
  GRID("fs_gas_energy_update_f32");
  return check(launch_gas_update32(gd, T_g, rho, Y_H2O, T_s, S_pyro, S_drying, Q_g_conv,
                                   q_rad_gas, Q_comb_out, dt_sub, T_amb, h_bed, drip_on, n_z_bed,
                                   i_src0, i_src1, ST(stream)),
               "fs_gas_energy_update_f32");
}

int fs_clip_f32(int64_t n, float* f, double lo, double hi, void* stream) {
  if (n < 0) return FS_EARG;
  return check(launch_clip32(n, f, lo, hi, ST(stream)), "fs_clip_f32");
}

int64_t fs_column_diag_scratch_bytes(const FsGrid* g) {
  GridDev gd;
  if (!to_grid(g, gd, "fs_column_diag_scratch_bytes")) return -1;
  return coldiag_scratch_bytes(gd);
}

int fs_column_diag(const FsGrid* g, const double* T_s, const double* omega, const double* S_pyro,
                   const double* S_drying, double T_ign, double T_front, double hrr_scale,
                   double* hrr_x, void* scratch, FsColumnDiag* out, void* stream) {
  GRID("fs_column_diag");
  if (!T_s || !omega || !S_pyro || !S_drying || !scratch || !out) {
    fs_set_error("fs_column_diag: bad argument");
    return FS_EARG;
  }
  SmallScratch* sc = small_scratch();
  if (!sc) {
    fs_set_error("fs_column_diag: scratch allocation failed");
    return FS_ECUDA;
  }
  int rc = launch_coldiag(gd, T_s, omega, S_pyro, S_drying, T_ign, T_front, hrr_scale, hrr_x,
                          scratch, ST(stream));
  if (rc != FS_OK) return check(rc, "fs_column_diag");
  launch_coldiag_keys(scratch, sc->dres, ST(stream));
  cudaMemcpyAsync(sc->hpin, sc->dres, 4 * sizeof(double), cudaMemcpyDeviceToHost, ST(stream));
  if (fs_stream_wait(ST(stream)) != FS_OK) return check(FS_ECUDA, "fs_column_diag");
  out->n_ign = (int64_t)sc->hpin[0];
  out->S_pyro_max = sc->hpin[1];
  out->hrr_max = sc->hpin[2];
  out->lead_i = (int)sc->hpin[3];
  return check(cuda_status(), "fs_column_diag");
}

int fs_clip(int64_t n, double* f, double lo, double hi, void* stream) {
  return check(launch_clip(n, f, lo, hi, ST(stream)), "fs_clip");
}

int fs_solid_conduction(const FsGrid* g, const double* T_s, const double* alpha_s, double* T_out,
                        double k_solid, double rho_solid, double cp_solid, double dt,
                        void* stream) {
  GRID("fs_solid_conduction");
  return check(launch_solid_cond(gd, T_s, alpha_s, T_out, k_solid, rho_solid, cp_solid, dt, gd.nz,
                                 ST(stream)),
               "fs_solid_conduction");
}

int fs_solid_conduction_capped(const FsGrid* g, const double* T_s, const double* alpha_s,
                               double* T_out, double k_solid, double rho_solid, double cp_solid,
                               double dt, double lo, double hi, void* stream) {
  GRID("fs_solid_conduction_capped");
  return check(launch_solid_cond(gd, T_s, alpha_s, T_out, k_solid, rho_solid, cp_solid, dt, gd.nz,
                                 ST(stream), 1, lo, hi),
               "fs_solid_conduction_capped");
}

int fs_soil_step(int nsoil, int ny, int nx, double* T_soil, const double* q_in, double dt,
                 const double* soil_dz, const double* d_above, const double* d_below, double k_s,
                 double rho_s, double cp_s, double eps_s, double T_amb, void* stream) {
  if (nsoil < 1 || ny < 1 || nx < 1) return FS_EARG;
  return check(launch_soil(nsoil, ny, nx, T_soil, q_in, dt, soil_dz, d_above, d_below, k_s, rho_s,
                           cp_s, eps_s, T_amb, ST(stream)),
               "fs_soil_step");
}

int fs_proj_create(const FsGrid* g, void** handle) {
  GRID("fs_proj_create");
  *handle = proj_create(gd);
  if (!*handle) {
    fs_set_error("fs_proj_create: allocation failed");
    return FS_ECUDA;
  }
  return FS_OK;
}

void fs_proj_destroy(void* handle) { proj_destroy(handle); }

int fs_proj_rebuild(void* handle, const double* rho, void* stream) {
  if (!handle) return FS_EARG;
  return check(proj_rebuild(handle, rho, ST(stream)), "fs_proj_rebuild");
}

int fs_proj_project(void* handle, double* u, double* v, double* w, const double* u_inlet,
                    const double* div_target, double dt, double rtol, int maxiter, int* iters,
                    void* stream) {
  if (!handle || !iters || !(dt > 0.0)) return FS_EARG;
  return check(proj_project(handle, u, v, w, u_inlet, div_target, dt, rtol, maxiter, iters,
                            ST(stream)),
               "fs_proj_project");
}

double* fs_proj_pressure(void* handle) { return handle ? proj_pressure(handle) : nullptr; }

int fs_proj_stats(void* handle, double* out8) {
  if (!handle || !out8) return FS_EARG;
  proj_stats(handle, out8);
  return FS_OK;
}

int fs_proj_set_learned(void* handle, void* net, int max_learned, double stall) {
  if (!handle) return check(FS_EARG, "fs_proj_set_learned");
  return check(proj_set_learned(handle, net, max_learned, stall), "fs_proj_set_learned");
}
int fs_proj_set_log(void* handle, double* r0, double* x0) {
  if (!handle) return check(FS_EARG, "fs_proj_set_log");
  return check(proj_set_log(handle, r0, x0), "fs_proj_set_log");
}
int fs_proj_fcg_stats(void* handle, double* out4) {
  if (!handle || !out4) return FS_EARG;
  proj_fcg_stats(handle, out4);
  return FS_OK;
}

int fs_proj_smooth_pair(void* handle, const double* r0, const double* e0, float* r1, float* e1,
                        void* stream) {
  if (!handle || !r0 || !e0 || !r1 || !e1) return check(FS_EARG, "fs_proj_smooth_pair");
  return check(proj_smooth_pair(handle, r0, e0, r1, e1, (cudaStream_t)stream),
               "fs_proj_smooth_pair");
}
int fs_unet_set_output_scale(void* handle, float s) {
  if (!handle) return check(FS_EARG, "fs_unet_set_output_scale");
  return check(unet_set_output_scale(handle, s), "fs_unet_set_output_scale");
}

int64_t fs_unet_nparams(void) { return unet_nparams(); }
int fs_unet_create(int nz, int ny, int nx, void** handle) {
  if (!handle) return check(FS_EARG, "fs_unet_create");
  return check(unet_create(nz, ny, nx, handle), "fs_unet_create");
}
void fs_unet_destroy(void* handle) { unet_destroy(handle); }
int fs_unet_set_params(void* handle, const float* host, int64_t n, void* stream) {
  if (!handle || !host) return check(FS_EARG, "fs_unet_set_params");
  return check(unet_set_params(handle, host, n, (cudaStream_t)stream), "fs_unet_set_params");
}
int fs_unet_get_params(void* handle, float* host, int64_t n, void* stream) {
  if (!handle || !host) return check(FS_EARG, "fs_unet_get_params");
  return check(unet_get(handle, 0, host, n, (cudaStream_t)stream), "fs_unet_get_params");
}
int fs_unet_get_grads(void* handle, float* host, int64_t n, void* stream) {
  if (!handle || !host) return check(FS_EARG, "fs_unet_get_grads");
  return check(unet_get(handle, 1, host, n, (cudaStream_t)stream), "fs_unet_get_grads");
}
int fs_unet_apply(void* handle, const double* r, double* z, void* stream) {
  if (!handle || !r || !z) return check(FS_EARG, "fs_unet_apply");
  return check(unet_apply(handle, r, z, (cudaStream_t)stream), "fs_unet_apply");
}
int fs_unet_forward(void* handle, const float* r, float* z, void* stream) {
  if (!handle || !r || !z) return check(FS_EARG, "fs_unet_forward");
  return check(unet_forward_f32(handle, r, z, (cudaStream_t)stream), "fs_unet_forward");
}
int fs_unet_grad(void* handle, const float* r, const float* tau, double* loss, void* stream) {
  if (!handle || !r || !tau) return check(FS_EARG, "fs_unet_grad");
  return check(unet_grad(handle, r, tau, loss, (cudaStream_t)stream), "fs_unet_grad");
}
int fs_unet_train_step(void* handle, const float* r, const float* tau, float lr, double* loss,
                       void* stream) {
  if (!handle || !r || !tau || !loss || !(lr > 0.f)) return check(FS_EARG, "fs_unet_train_step");
  return check(unet_train_step(handle, r, tau, lr, loss, (cudaStream_t)stream),
               "fs_unet_train_step");
}

int fs_proj_set_precision(void* handle, int fp32) {
  if (!handle) return FS_EARG;
  return check(proj_set_precision(handle, fp32), "fs_proj_set_precision");
}

int fs_proj_configure(void* handle, int nu, double omega) {
  if (!handle) return FS_EARG;
  return check(proj_configure(handle, nu, omega), "fs_proj_configure");
}
int fs_proj_set_fine_sweeps(void* handle, int nu0) {
  if (!handle) return check(FS_EARG, "fs_proj_set_fine_sweeps");
  return check(proj_set_fine_sweeps(handle, nu0), "fs_proj_set_fine_sweeps");
}

int fs_proj_set_coarse_tail(void* handle, int on) {
  if (!handle) return check(FS_EARG, "fs_proj_set_coarse_tail");
  return check(proj_set_coarse_tail(handle, on), "fs_proj_set_coarse_tail");
}

int fs_proj_apply(void* handle, const double* x, double* y, void* stream) {
  if (!handle) return FS_EARG;
  return check(proj_apply(handle, x, y, ST(stream)), "fs_proj_apply");
}

int fs_divergence_max(const FsGrid* g, const double* u, const double* v, const double* w,
                      const double* u_inlet, const double* div_target, double* div_out,
                      double* result, void* stream) {
  GRID("fs_divergence_max");
  SmallScratch* sc = small_scratch();
  if (!sc) {
    fs_set_error("fs_divergence_max: scratch allocation failed");
    return FS_ECUDA;
  }
  int st = launch_div_resid_max(gd, u, v, w, u_inlet, div_target, div_out, sc->dkey, ST(stream));
  cudaMemcpyAsync(sc->hpin, sc->dkey, sizeof(double), cudaMemcpyDeviceToHost, ST(stream));
  if (fs_stream_wait(ST(stream)) != FS_OK) return check(FS_ECUDA, "fs_divergence_max");
  memcpy(result, sc->hpin, sizeof(double));
  return check(st, "fs_divergence_max");
}

int fs_dom_create(const FsGrid* g, int M, const double* ox, const double* oy, const double* oz,
                  const double* w, double kappa_gas_max, void** handle) {
  GRID("fs_dom_create");
  if (M < 1 || !ox || !oy || !oz || !w) return FS_EARG;
  *handle = dom_create(gd, M, ox, oy, oz, w, kappa_gas_max);
  if (!*handle) {
    fs_set_error("fs_dom_create: allocation failed");
    return FS_ECUDA;
  }
  return FS_OK;
}

void fs_dom_destroy(void* handle) { dom_destroy(handle); }

int fs_dom_solve(void* handle, const double* T_s, const double* T_g, const double* alpha_s,
                 const double* omega, double sigma_sav, double T_amb, const double* T_soil0,
                 const double* Y_H2O, const double* rho, const double* M_local, double* q_rad_solid,
                 double* q_rad_gas, double* q_in_soil, void* stream) {
  if (!handle) return FS_EARG;
  return check(dom_solve(handle, T_s, T_g, alpha_s, omega, sigma_sav, T_amb, T_soil0, Y_H2O, rho,
                         M_local, q_rad_solid, q_rad_gas, q_in_soil, ST(stream)),
               "fs_dom_solve");
}

int fs_dom_begin(void* handle, const double* T_s, const double* T_g, const double* alpha_s,
                 const double* omega, double sigma_sav, double T_amb, const double* T_soil0,
                 const double* Y_H2O, const double* rho, const double* M_local, void* stream) {
  if (!handle) return check(FS_EARG, "fs_dom_begin");
  return check(dom_begin(handle, T_s, T_g, alpha_s, omega, sigma_sav, T_amb, T_soil0, Y_H2O, rho,
                         M_local, ST(stream)),
               "fs_dom_begin");
}

int fs_dom_end(void* handle, double* q_rad_solid, double* q_rad_gas, double* q_in_soil,
               void* stream) {
  if (!handle) return check(FS_EARG, "fs_dom_end");
  return check(dom_end(handle, q_rad_solid, q_rad_gas, q_in_soil, ST(stream)), "fs_dom_end");
}

double* fs_dom_intensity(void* handle) { return handle ? dom_intensity(handle) : nullptr; }

int fs_dom_set_sweep_mode(void* handle, int mode, int cluster_ctas) {
  if (!handle) return FS_EARG;
  return check(dom_set_mode(handle, mode, cluster_ctas), "fs_dom_set_sweep_mode");
}

int fs_dom_set_octant_groups(void* handle, int groups) {
  if (!handle) return check(FS_EARG, "fs_dom_set_octant_groups");
  return check(dom_set_groups(handle, groups), "fs_dom_set_octant_groups");
}
int fs_dom_sweep_mode(void* handle) { return handle ? dom_mode(handle) : -1; }
int fs_dom_set_sweep_kernel(void* handle, int kernel) {
  if (!handle) return check(FS_EARG, "fs_dom_set_sweep_kernel");
  return check(dom_set_sweep_kernel(handle, kernel), "fs_dom_set_sweep_kernel");
}
int fs_dom_sweep_kernel(void* handle) { return handle ? dom_sweep_kernel(handle) : -1; }
int fs_index_divide(uint32_t d, int64_t n, const uint32_t* x, uint32_t* q) {
  if (d == 0 || n < 0 || (n > 0 && (!x || !q))) {
    fs_set_error("fs_index_divide: divisor %u, count %lld", d, (long long)n);
    return FS_EARG;
  }
  const FastDiv f = fastdiv_make(d);
  for (int64_t t = 0; t < n; ++t) q[t] = fdiv(x[t], f);
  return FS_OK;
}

int fs_dom_set_wait_test(void* handle, int plane) {
  if (!handle) return check(FS_EARG, "fs_dom_set_wait_test");
  return dom_set_wait_test(handle, plane);
}

int fs_dom_launch_shape(void* handle, int* out5) {
  if (!handle || !out5) {
    fs_set_error("fs_dom_launch_shape: null argument");
    return FS_EARG;
  }
  return dom_launch_shape(handle, out5);
}

int fs_dom_set_precision(void* handle, int fp32) {
  if (!handle) return FS_EARG;
  return check(dom_set_precision(handle, fp32), "fs_dom_set_precision");
}

int64_t fs_dom_wrap_size(void* handle) { return handle ? dom_wrap_size(handle) : -1; }

int fs_dom_get_wrap(void* handle, double* dst, void* stream) {
  if (!handle || !dst) return FS_EARG;
  return check(dom_get_wrap(handle, dst, ST(stream)), "fs_dom_get_wrap");
}

int fs_dom_set_wrap(void* handle, const double* src, void* stream) {
  if (!handle || !src) return FS_EARG;
  return check(dom_set_wrap(handle, src, ST(stream)), "fs_dom_set_wrap");
}

int fs_dom_load_intensity(void* handle, const double* I_full, void* stream) {
  if (!handle || !I_full) return FS_EARG;
  return check(dom_load_intensity(handle, I_full, ST(stream)), "fs_dom_load_intensity");
}

int fs_dom_sweep_timing(void* handle, int enable, double* total_ms, long long* sweeps) {
  if (!handle) return FS_EARG;
  if (enable >= 0) dom_set_timing(handle, enable);
  if (total_ms && sweeps) dom_sweep_stats(handle, total_ms, sweeps);
  return FS_OK;
}
int fs_dom_iterations(void* handle) { return handle ? dom_last_iters(handle) : -1; }

int fs_bed_step(const FsGrid* g, const FsBedParticles* p, const FsBedSegments* s,
                const FsBedSources* o, const FsBedParams* prm, const double* T_g,
                const double* Y_O2, void* stream) {
  GRID("fs_bed_step");
  if (!p || !s || !o || !prm || !(prm->dt > 0.0)) {
    fs_set_error("fs_bed_step: bad argument");
    return FS_EARG;
  }
  BedOutH oh{o->S_pyro, o->S_drying, o->Q_pyro, o->Q_drying, o->Y_F_source, o->Q_char,
             o->Q_smold, o->Q_g_conv};
  BedParamsH b{};
  b.dt = prm->dt; b.h_conv = prm->h_conv; b.rho_true = prm->rho_true; b.cp_solid = prm->cp_solid;
  b.eps_solid = prm->eps_solid; b.T_amb = prm->T_amb; b.view = prm->view; b.h_bed = prm->h_bed;
  b.kappa_bed = prm->kappa_bed; b.char_cap = prm->char_cap; b.ash_exp = prm->ash_exp;
  b.do_dry = prm->do_dry; b.do_pyro = prm->do_pyro; b.do_char = prm->do_char;
  b.do_smold = prm->do_smold; b.mode = prm->mode; b.geometric = prm->geometric;
  b.n_split = prm->n_split; b.Qsx = prm->Qsx; b.q_rad = prm->q_rad; b.drip_on = prm->drip_on;
  b.n_z_bed = prm->n_z_bed; b.i_src0 = prm->i_src0; b.i_src1 = prm->i_src1;
  return check(launch_bed_step(gd, *p, *s, oh, b, T_g, Y_O2, ST(stream)), "fs_bed_step");
}

int fs_bed_aggregate(const FsBedParticles* p, const FsBedSegments* s, double* out, int mode,
                     void* stream) {
  if (!p || !s || (mode != 0 && mode != 1)) return FS_EARG;
  return check(launch_bed_aggregate(*p, *s, out, mode, ST(stream)), "fs_bed_aggregate");
}

int fs_bed_hcond(const FsGrid* g, double* T_s_grid, double* scratch, const double* alpha_s,
                 int n_z_bed, double k_solid, double rho_true, double cp_solid, double dt,
                 const FsBedParticles* p, const FsBedSegments* s, const int* seg_of_cell,
                 void* stream) {
  GRID("fs_bed_hcond");
  if (!p || !s || !scratch || !seg_of_cell) return FS_EARG;
  return check(launch_bed_hcond(gd, T_s_grid, scratch, alpha_s, n_z_bed, k_solid, rho_true,
                                cp_solid, dt, *p, *s, seg_of_cell, ST(stream)),
               "fs_bed_hcond");
}

int fs_levelset(const FsGrid* g, const double* phi, const double* aux, double* out, double coef,
                int mode, void* stream) {
  GRID("fs_levelset");
  if (mode < 0 || mode > 2 || (mode > 0 && !aux)) return FS_EARG;
  return check(launch_levelset(gd, phi, aux, out, coef, mode, ST(stream)), "fs_levelset");
}

int fs_active_count(int64_t n, const double* omega, const double* T_g, const double* Y_F,
                    unsigned long long* count, unsigned char* mask, void* stream) {
  return check(launch_active_count(n, omega, T_g, Y_F, count, mask, ST(stream)),
               "fs_active_count");
}

}  // extern "C"
