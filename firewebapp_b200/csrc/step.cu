// Whole outer steps of the Tier-3 loop (spread_3d.py:1897-3512), driven from
// C++: fs_ctx_create / fs_step / fs_batch_run (include/firestep.h).
//
// The context owns every device buffer and runs the operators of one outer
// step in the reference's order through this library's entry points, on its
// own main stream; the DOM solve runs on a second (high-priority) stream from
// a worker thread of the context, concurrently with momentum, the projection
// and k-epsilon, exactly as the Python stepper (firewebapp_b200/solver.py)
// does: the solve reads only fields those operators leave untouched and
// writes only fields they do not read, and once its inputs have been read
// the flame mask, the gas-temperature advection and the first chemistry
// sub-step's species work run during the sweeps.  The results are those of
// the sequential order.  Host code here reads back only what the loop
// branches on.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <condition_variable>
#include <initializer_list>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int N_SUB = 10;
constexpr double SC_T = 0.7;
constexpr double PR_T = 0.85;
constexpr double K_MIN = 1.0e-8;
constexpr double EPS_MIN = 1.0e-8;
constexpr double T_CAP = 10000.0;
constexpr double KAPPA_SOOT_HOT = 0.5;
constexpr double G_ACC = 9.81;

// Python's max()/min() over floats: keep the first extreme, compare with >/<.
double pymax(std::initializer_list<double> v) {
  double r = *v.begin();
  for (double x : v)
    if (x > r) r = x;
  return r;
}
double pymin(std::initializer_list<double> v) {
  double r = *v.begin();
  for (double x : v)
    if (x < r) r = x;
  return r;
}

}  // namespace

// Cell-field slots of the context: 14 state fields, the fields carried
// between steps and the work buffers the out-of-place kernels write (the
// host swaps the pointers instead of copying).
enum {
  S_RHO = 0, S_U, S_V, S_W, S_TG, S_YF, S_YO, S_YH, S_TS, S_AS, S_K, S_EPS, S_NU, S_PHI,
  W_RHO_PREV, W_OMEGA, W_QRAD, W_QRADG, W_MLOC, W_DIVT, W_T1, W_T2, W_T3, W_T4, W_T5, W_QCOMB,
  W_PHI0,
  B_SP, B_SD, B_QP, B_QD, B_YFS, B_QCH, B_QSM, B_QGC,
  NSLOT
};

// FP32 copies of the mixed form's sub-steps: the fields they update (and
// their work buffers) and the fields they only read
enum {
  F32_TG = 0, F32_YF, F32_YO, F32_YH, F32_T1, F32_T2, F32_T3, F32_T4, F32_RHO, F32_U, F32_V,
  F32_W, F32_K, F32_EPS, F32_NU, F32_SP, F32_SD, F32_QGC, F32_OMEGA, F32_QCOMB, F32_N
};

struct FsCtx {
  FsCaseDesc c;
  std::vector<double> hdz, hda, hdb, hox, hoy, hoz, hw, hsdz, hsda, hsdb;
  int dev = 0;
  int64_t n = 0, n2 = 0;
  double* dz = nullptr;
  double* da = nullptr;
  double* db = nullptr;
  FsGrid g{};
  double* f[NSLOT] = {};
  double *u_inlet = nullptr, *sigma_x = nullptr, *k_wall = nullptr, *eps_wall = nullptr,
         *zero2 = nullptr;
  double *hcond_scratch = nullptr, *max_scratch = nullptr;
  void* edc_scratch = nullptr;
  unsigned long long* active_count = nullptr;
  double *T_soil = nullptr, *q_in_soil = nullptr, *soil_dz = nullptr, *soil_da = nullptr,
         *soil_db = nullptr;
  // FP32 sub-step copies of the mixed form (slots as F32_*), NULL in the plain form
  float* h32[20] = {};
  void* edc32_scratch = nullptr;
  // particles and their per-cell segments
  int64_t np = 0;
  double* pd[10] = {};  // x y z m_solid m_water m_char T_s m_water_0 sav m_char_max
  signed char* alive = nullptr;
  int *seg_start = nullptr, *seg_cell = nullptr, *perm = nullptr, *seg_of_cell = nullptr;
  int nseg = 0;
  FsBedParticles parts{};
  FsBedSegments segs{};
  FsBedSources src{};
  void* proj = nullptr;
  void* dom = nullptr;
  cudaStream_t s_main = nullptr, s_dom = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_inputs = nullptr, ev_done = nullptr;
  // pinned host staging for the exit tests: active count, two phi rows
  unsigned long long* h_count = nullptr;
  double* h_rows = nullptr;
  // clock and loop state
  double t = 0.0, dt = 0.0;
  int64_t step_count = 0, lset_step = 0;
  int extinct_count = 0;
  int finished = 0;
  std::vector<double> front_t, front_x;
  FsStepOut last{};
  // DOM worker
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  bool job = false, quit = false;
  int inputs_rc = -1, done_rc = -1;  // -1 pending
  std::string job_err;
  char err[512] = "";
};

static int ctx_fail(FsCtx* C, int rc, const char* where) {
  if (C) {
    snprintf(C->err, sizeof(C->err), "%s: %s", where, fs_last_error());
    fs_set_error("%s", C->err);
  }
  return rc;
}

#define CK(call, where)                                   \
  do {                                                    \
    int rc_ = (call);                                     \
    if (rc_ != FS_OK) return ctx_fail(C, rc_, (where));   \
  } while (0)

static double* dev_alloc(int64_t n, bool& ok) {
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) ok = false;
  return (double*)p;
}

static void dom_worker(FsCtx* C) {
  cudaSetDevice(C->dev);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(C->mu);
      C->cv.wait(lk, [&] { return C->job || C->quit; });
      if (C->quit) return;
      C->job = false;
    }
    const FsCaseDesc& c = C->c;
    cudaStream_t st = C->s_dom;
    int rc = cudaStreamWaitEvent(st, C->ev_ready, 0) == cudaSuccess ? FS_OK : FS_ECUDA;
    if (rc == FS_OK)
      rc = fs_bed_aggregate(&C->parts, &C->segs, C->f[W_MLOC], 1, st);
    if (rc == FS_OK)
      rc = fs_dom_begin(C->dom, C->f[S_TS], C->f[S_TG], C->f[S_AS], C->f[W_OMEGA], c.sav,
                        c.T_amb, C->T_soil, C->f[S_YH], C->f[S_RHO], C->f[W_MLOC], st);
    if (rc == FS_OK && cudaEventRecord(C->ev_inputs, st) != cudaSuccess) rc = FS_ECUDA;
    std::string msg = rc != FS_OK ? std::string(fs_last_error()) : std::string();
    {
      std::lock_guard<std::mutex> lk(C->mu);
      C->inputs_rc = rc;
      if (rc != FS_OK) C->job_err = "dom_begin: " + msg;
    }
    C->cv.notify_all();
    if (rc == FS_OK) {
      rc = fs_dom_end(C->dom, C->f[W_QRAD], C->f[W_QRADG], C->q_in_soil, st);
      if (rc == FS_OK && cudaEventRecord(C->ev_done, st) != cudaSuccess) rc = FS_ECUDA;
      msg = rc != FS_OK ? std::string(fs_last_error()) : std::string();
    }
    {
      std::lock_guard<std::mutex> lk(C->mu);
      C->done_rc = rc;
      if (rc != FS_OK && C->job_err.empty()) C->job_err = "dom_end: " + msg;
    }
    C->cv.notify_all();
  }
}

static int wait_state(FsCtx* C, int* slot) {
  std::unique_lock<std::mutex> lk(C->mu);
  C->cv.wait(lk, [&] { return *slot >= 0; });
  if (*slot != FS_OK) {
    snprintf(C->err, sizeof(C->err), "DOM solve: %s", C->job_err.c_str());
    fs_set_error("%s", C->err);
  }
  return *slot;
}

// x of the first sign change of phi along a host row (spread_3d.py:3743,
// flame_front_3d.py front_x); +inf when there is none
static double front_from_row(const double* row, int nx, double dx) {
  for (int i = 0; i + 1 < nx; ++i) {
    const double a = row[i], b = row[i + 1];
    if ((a < 0.0 && 0.0 < b) || (b < 0.0 && 0.0 < a)) return (i + (-a / (b - a)) + 0.5) * dx;
  }
  return INFINITY;
}

// turbulence_3d.py:880-915: sub-step count from the interior maximum of nu_t
static void nsub_from(const FsCaseDesc& c, double nu_max, double sc, double dt, int* n,
                      double* dts) {
  const double h_min2 = pymin({c.dx * c.dx, pymin({c.dy * c.dy, c.dz_min * c.dz_min})});
  const double D_max = nu_max / sc;
  *n = 0;
  *dts = 0.0;
  if (D_max <= 1.0e-12 || !std::isfinite(D_max)) return;
  const double dt_sub_max = 0.4 * h_min2 / D_max;
  if (dt_sub_max <= 0.0) return;
  const double target = dt / dt_sub_max;
  if (target > 1000) return;
  const int k = (int)std::ceil(target);
  *n = k > 1 ? k : 1;
  *dts = dt / *n;
}

// particle cells as locate_cell computes them (lagrangian_particles_3d.py:95-140)
// and the per-cell segments in slot order
static void build_segments(FsCtx* C, const FsInitState* s, std::vector<signed char>& alive,
                           std::vector<int>& perm, std::vector<int>& starts,
                           std::vector<int>& segcell) {
  const FsCaseDesc& c = C->c;
  std::vector<double> zf(c.nz + 1, 0.0);
  for (int k = 0; k < c.nz; ++k) zf[k + 1] = zf[k] + c.dz[k];
  const int64_t np = s->n_particles;
  std::vector<int64_t> cell(np, -1);
  for (int64_t p = 0; p < np; ++p) {
    const double x = s->px[p], y = s->py[p], z = s->pz[p];
    int64_t i = x < 0.0 ? -1 : (int64_t)std::trunc(x / c.dx);
    if (i >= c.nx) i = -1;
    int64_t j = y < 0.0 ? -1 : (int64_t)std::trunc(y / c.dy);
    if (j >= c.ny) j = -1;
    int64_t k = -1;
    if (z >= zf[0] && z < zf[c.nz]) {
      k = std::upper_bound(zf.begin() + 1, zf.end(), z) - (zf.begin() + 1);
      if (k > c.nz - 1) k = c.nz - 1;
    }
    if (i >= 0 && j >= 0 && k >= 0) cell[p] = (k * c.ny + j) * c.nx + i;
  }
  alive.assign(s->alive, s->alive + np);
  std::vector<int64_t> valid;
  for (int64_t p = 0; p < np; ++p) {
    if (cell[p] < 0) alive[p] = 0;
    else valid.push_back(p);
  }
  std::stable_sort(valid.begin(), valid.end(),
                   [&](int64_t a, int64_t b) { return cell[a] < cell[b]; });
  perm.assign(valid.begin(), valid.end());
  starts.clear();
  segcell.clear();
  for (size_t q = 0; q < valid.size(); ++q) {
    if (q == 0 || cell[valid[q]] != cell[valid[q - 1]]) {
      starts.push_back((int)q);
      segcell.push_back((int)cell[valid[q]]);
    }
  }
  starts.push_back((int)valid.size());
}

static void ctx_free(FsCtx* C) {
  if (!C) return;
  if (C->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(C->mu);
      C->quit = true;
    }
    C->cv.notify_all();
    C->worker.join();
  }
  if (C->s_main) cudaStreamSynchronize(C->s_main);
  if (C->s_dom) cudaStreamSynchronize(C->s_dom);
  if (C->proj) fs_proj_destroy(C->proj);
  if (C->dom) fs_dom_destroy(C->dom);
  for (int q = 0; q < NSLOT; ++q) cudaFree(C->f[q]);
  for (int q = 0; q < 10; ++q) cudaFree(C->pd[q]);
  for (int q = 0; q < F32_N; ++q) cudaFree(C->h32[q]);
  cudaFree(C->edc32_scratch);
  cudaFree(C->dz); cudaFree(C->da); cudaFree(C->db);
  cudaFree(C->u_inlet); cudaFree(C->sigma_x); cudaFree(C->k_wall); cudaFree(C->eps_wall);
  cudaFree(C->zero2); cudaFree(C->hcond_scratch); cudaFree(C->max_scratch);
  cudaFree(C->edc_scratch); cudaFree(C->active_count); cudaFree(C->T_soil);
  cudaFree(C->q_in_soil); cudaFree(C->soil_dz); cudaFree(C->soil_da); cudaFree(C->soil_db);
  cudaFree(C->alive); cudaFree(C->seg_start); cudaFree(C->seg_cell); cudaFree(C->perm);
  cudaFree(C->seg_of_cell);
  if (C->h_count) cudaFreeHost(C->h_count);
  if (C->h_rows) cudaFreeHost(C->h_rows);
  if (C->ev_ready) cudaEventDestroy(C->ev_ready);
  if (C->ev_inputs) cudaEventDestroy(C->ev_inputs);
  if (C->ev_done) cudaEventDestroy(C->ev_done);
  if (C->s_main) cudaStreamDestroy(C->s_main);
  if (C->s_dom) cudaStreamDestroy(C->s_dom);
  delete C;
}

static bool copy_in(cudaStream_t st, void* dst, const void* src, size_t bytes) {
  if (!src) return false;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
}

extern "C" {

int fs_ctx_create(const FsCaseDesc* desc, const FsInitState* init, FsCtx** out) {
  if (!desc || !init || !out) {
    fs_set_error("fs_ctx_create: bad argument");
    return FS_EARG;
  }
  *out = nullptr;
  const FsCaseDesc& d = *desc;
  if (d.nx < 2 || d.ny < 1 || d.nz < 2 || d.n_z_bed < 0 || d.n_z_bed > d.nz || !d.dz ||
      !d.d_above || !d.d_below || !(d.dx > 0.0) || !(d.dy > 0.0) || d.M < 8 || !d.ox || !d.oy ||
      !d.oz || !d.w || d.n_soil < 1 || !d.soil_dz || !d.soil_d_above || !d.soil_d_below ||
      (d.form != 0 && d.form != 1) || !(d.projection_rtol > 0.0) || d.proj_maxiter < 1 ||
      d.proj_max_iter < 1 || d.i_src_start < 0 || d.i_src_end > d.nx ||
      d.i_src_start > d.i_src_end || init->n_particles < 0) {
    fs_set_error("fs_ctx_create: invalid case description");
    return FS_EARG;
  }
  FsCtx* C = new FsCtx();
  C->c = d;
  C->hdz.assign(d.dz, d.dz + d.nz);
  C->hda.assign(d.d_above, d.d_above + d.nz);
  C->hdb.assign(d.d_below, d.d_below + d.nz);
  C->hox.assign(d.ox, d.ox + d.M); C->hoy.assign(d.oy, d.oy + d.M);
  C->hoz.assign(d.oz, d.oz + d.M); C->hw.assign(d.w, d.w + d.M);
  C->hsdz.assign(d.soil_dz, d.soil_dz + d.n_soil);
  C->hsda.assign(d.soil_d_above, d.soil_d_above + d.n_soil);
  C->hsdb.assign(d.soil_d_below, d.soil_d_below + d.n_soil);
  // the description's arrays are the caller's: keep only the copies
  C->c.dz = C->hdz.data(); C->c.d_above = C->hda.data(); C->c.d_below = C->hdb.data();
  C->c.ox = C->hox.data(); C->c.oy = C->hoy.data(); C->c.oz = C->hoz.data();
  C->c.w = C->hw.data();
  C->c.soil_dz = C->hsdz.data(); C->c.soil_d_above = C->hsda.data();
  C->c.soil_d_below = C->hsdb.data();
  const FsCaseDesc& c = C->c;
  cudaGetDevice(&C->dev);
  C->n = (int64_t)c.nx * c.ny * c.nz;
  C->n2 = (int64_t)c.nx * c.ny;
  const int64_t n = C->n, n2 = C->n2;
  bool ok = true;
  SetupStream ss;  // the copies and clearing below, complete before the first step
  C->dz = dev_alloc(c.nz, ok); C->da = dev_alloc(c.nz, ok); C->db = dev_alloc(c.nz, ok);
  ok = ok && copy_in(ss.s, C->dz, c.dz, 8 * c.nz) && copy_in(ss.s, C->da, c.d_above, 8 * c.nz) &&
       copy_in(ss.s, C->db, c.d_below, 8 * c.nz);
  C->g = FsGrid{c.nx, c.ny, c.nz, c.dx, c.dy, C->dz, C->da, C->db};
  for (int q = 0; q < NSLOT; ++q) C->f[q] = dev_alloc(n, ok);
  const double* init_fields[14] = {init->rho, init->u, init->v, init->w, init->T_g,
                                   init->Y_fuel, init->Y_O2, init->Y_H2O, init->T_s,
                                   init->alpha_s, init->k_turb, init->eps_turb, init->nu_t,
                                   init->phi};
  for (int q = 0; q < 14 && ok; ++q) ok = copy_in(ss.s, C->f[q], init_fields[q], 8 * n);
  for (int q = 14; q < NSLOT && ok; ++q) ok = cudaMemsetAsync(C->f[q], 0, 8 * n, ss.s) == cudaSuccess;
  C->u_inlet = dev_alloc((int64_t)c.nz * c.ny, ok);
  C->sigma_x = dev_alloc(c.nx, ok);
  ok = ok && copy_in(ss.s, C->u_inlet, init->u_inlet, 8 * (size_t)c.nz * c.ny) &&
       copy_in(ss.s, C->sigma_x, init->sigma_x, 8 * (size_t)c.nx);
  C->k_wall = dev_alloc(n2, ok); C->eps_wall = dev_alloc(n2, ok);
  C->zero2 = dev_alloc((int64_t)c.nz * c.ny, ok);
  if (ok) {
    std::vector<double> kw(n2, K_MIN), ew(n2, EPS_MIN);
    ok = copy_in(ss.s, C->k_wall, kw.data(), 8 * n2) && copy_in(ss.s, C->eps_wall, ew.data(), 8 * n2) &&
         cudaMemsetAsync(C->zero2, 0, 8 * (size_t)c.nz * c.ny, ss.s) == cudaSuccess;
  }
  C->hcond_scratch = dev_alloc((int64_t)std::max(c.n_z_bed, 1) * n2, ok);
  C->max_scratch = dev_alloc(64, ok);
  if (cudaMalloc(&C->edc_scratch, (size_t)fs_edc_scratch_bytes(n) + 64) != cudaSuccess) ok = false;
  if (cudaMalloc(&C->active_count, sizeof(unsigned long long)) != cudaSuccess) ok = false;
  if (c.form == 1) {
    for (int q = 0; q < F32_N; ++q)
      if (cudaMalloc(&C->h32[q], sizeof(float) * (size_t)n) != cudaSuccess) ok = false;
    if (cudaMalloc(&C->edc32_scratch, (size_t)fs_edc_f32_scratch_bytes(n) + 64) != cudaSuccess)
      ok = false;
  }
  C->T_soil = dev_alloc((int64_t)c.n_soil * n2, ok);
  C->q_in_soil = dev_alloc(n2, ok);
  C->soil_dz = dev_alloc(c.n_soil, ok); C->soil_da = dev_alloc(c.n_soil, ok);
  C->soil_db = dev_alloc(c.n_soil, ok);
  ok = ok && copy_in(ss.s, C->T_soil, init->T_soil, 8 * (size_t)c.n_soil * n2) &&
       cudaMemsetAsync(C->q_in_soil, 0, 8 * n2, ss.s) == cudaSuccess &&
       copy_in(ss.s, C->soil_dz, c.soil_dz, 8 * c.n_soil) &&
       copy_in(ss.s, C->soil_da, c.soil_d_above, 8 * c.n_soil) &&
       copy_in(ss.s, C->soil_db, c.soil_d_below, 8 * c.n_soil);
  // particles and segments
  C->np = init->n_particles;
  const double* pin[10] = {init->px, init->py, init->pz, init->m_solid, init->m_water,
                           init->m_char, init->pT_s, init->m_water_0, init->psav,
                           init->m_char_max};
  for (int q = 0; q < 10 && ok; ++q) {
    C->pd[q] = dev_alloc(C->np, ok);
    ok = ok && (C->np == 0 || copy_in(ss.s, C->pd[q], pin[q], 8 * (size_t)C->np));
  }
  if (ok && C->np > 0 && (!init->alive || !init->px || !init->py || !init->pz)) ok = false;
  if (ok) {
    std::vector<signed char> alive;
    std::vector<int> perm, starts, segcell;
    if (C->np > 0) build_segments(C, init, alive, perm, starts, segcell);
    else starts.push_back(0);
    C->nseg = (int)segcell.size();
    std::vector<int> soc(n, -1);
    for (int q = 0; q < C->nseg; ++q) soc[segcell[q]] = q;
    ok = cudaMalloc(&C->alive, (size_t)std::max<int64_t>(C->np, 1)) == cudaSuccess &&
         cudaMalloc(&C->perm, sizeof(int) * std::max<size_t>(perm.size(), 1)) == cudaSuccess &&
         cudaMalloc(&C->seg_start, sizeof(int) * starts.size()) == cudaSuccess &&
         cudaMalloc(&C->seg_cell, sizeof(int) * std::max<size_t>(segcell.size(), 1)) ==
             cudaSuccess &&
         cudaMalloc(&C->seg_of_cell, sizeof(int) * (size_t)n) == cudaSuccess;
    ok = ok && (C->np == 0 || copy_in(ss.s, C->alive, alive.data(), (size_t)C->np)) &&
         (perm.empty() || copy_in(ss.s, C->perm, perm.data(), sizeof(int) * perm.size())) &&
         copy_in(ss.s, C->seg_start, starts.data(), sizeof(int) * starts.size()) &&
         (segcell.empty() || copy_in(ss.s, C->seg_cell, segcell.data(), sizeof(int) * segcell.size())) &&
         copy_in(ss.s, C->seg_of_cell, soc.data(), sizeof(int) * (size_t)n);
  }
  C->parts = FsBedParticles{C->pd[0], C->pd[1], C->pd[2], C->alive, C->pd[3], C->pd[4],
                            C->pd[5], C->pd[6], C->pd[7], C->pd[8], C->pd[9]};
  C->segs = FsBedSegments{C->nseg, C->seg_start, C->seg_cell, C->perm};
  C->src = FsBedSources{C->f[B_SP], C->f[B_SD], C->f[B_QP], C->f[B_QD], C->f[B_YFS],
                        C->f[B_QCH], C->f[B_QSM], C->f[B_QGC]};
  if (ok && (cudaMallocHost(&C->h_count, sizeof(unsigned long long)) != cudaSuccess ||
             cudaMallocHost(&C->h_rows, sizeof(double) * 2 * c.nx) != cudaSuccess))
    ok = false;
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (ok && (cudaStreamCreateWithFlags(&C->s_main, cudaStreamNonBlocking) != cudaSuccess ||
             cudaStreamCreateWithPriority(&C->s_dom, cudaStreamNonBlocking, hi) != cudaSuccess ||
             cudaEventCreateWithFlags(&C->ev_ready, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&C->ev_inputs, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&C->ev_done, cudaEventDisableTiming) != cudaSuccess))
    ok = false;
  if (!ok || !ss.sync()) {
    cudaGetLastError();
    fs_set_error("fs_ctx_create: device allocation or copy failed");
    ctx_free(C);
    return FS_ECUDA;
  }
  int rc = fs_proj_create(&C->g, &C->proj);
  if (rc == FS_OK && c.form == 1) rc = fs_proj_set_precision(C->proj, 1);
  if (rc == FS_OK)
    rc = fs_dom_create(&C->g, c.M, c.ox, c.oy, c.oz, c.w, KAPPA_SOOT_HOT, &C->dom);
  if (rc == FS_OK && c.form == 1) rc = fs_dom_set_precision(C->dom, 1);
  if (rc != FS_OK) {
    ctx_fail(C, rc, "fs_ctx_create");
    ctx_free(C);
    return rc;
  }
  C->t = 0.0;
  C->dt = c.dt0;
  C->front_t.assign(1, 0.0);
  C->front_x.assign(1, c.x_front0);
  if (c.overlap_dom) C->worker = std::thread(dom_worker, C);
  *out = C;
  return FS_OK;
}

void fs_ctx_destroy(FsCtx* ctx) { ctx_free(ctx); }

const char* fs_ctx_last_error(FsCtx* ctx) { return ctx ? ctx->err : fs_last_error(); }

void* fs_ctx_stream(FsCtx* ctx) { return ctx ? (void*)ctx->s_main : nullptr; }

}  // extern "C"

static int slot_of(int id) {
  if (id >= FS_F_RHO && id <= FS_F_PHI) return S_RHO + (id - FS_F_RHO);
  switch (id) {
    case FS_F_OMEGA: return W_OMEGA;
    case FS_F_Q_RAD: return W_QRAD;
    case FS_F_Q_RAD_GAS: return W_QRADG;
    case FS_F_M_LOCAL: return W_MLOC;
    case FS_F_S_PYRO: return B_SP;
    case FS_F_S_DRYING: return B_SD;
    case FS_F_Q_G_CONV: return B_QGC;
    case FS_F_Q_COMB: return W_QCOMB;
  }
  return -1;
}

static void* field_ptr(FsCtx* C, int id, int64_t* count, size_t* esize) {
  *esize = 8;
  const int s = slot_of(id);
  if (s >= 0) {
    *count = C->n;
    return C->f[s];
  }
  if (id == FS_F_PRESSURE) {
    *count = C->n;
    return fs_proj_pressure(C->proj);
  }
  if (id == FS_F_T_SOIL) {
    *count = (int64_t)C->c.n_soil * C->n2;
    return C->T_soil;
  }
  if (id >= FS_P_X && id <= FS_P_M_CHAR_MAX) {
    *count = C->np;
    return C->pd[id - FS_P_X];
  }
  if (id == FS_P_ALIVE) {
    *count = C->np;
    *esize = 1;
    return C->alive;
  }
  *count = -1;
  return nullptr;
}

extern "C" {

int64_t fs_ctx_field_size(FsCtx* ctx, int id) {
  if (!ctx) return -1;
  int64_t cnt = 0;
  size_t es = 0;
  field_ptr(ctx, id, &cnt, &es);
  return cnt;
}

void* fs_ctx_field(FsCtx* ctx, int id) {
  if (!ctx) return nullptr;
  int64_t cnt = 0;
  size_t es = 0;
  return field_ptr(ctx, id, &cnt, &es);
}

int fs_ctx_read(FsCtx* ctx, int id, void* host_dst) {
  if (!ctx || !host_dst) return FS_EARG;
  int64_t cnt = 0;
  size_t es = 0;
  void* p = field_ptr(ctx, id, &cnt, &es);
  if (cnt < 0) {
    fs_set_error("fs_ctx_read: unknown field id %d", id);
    return FS_EARG;
  }
  if (cnt == 0) return FS_OK;
  cudaStreamSynchronize(ctx->s_dom);
  if (cudaMemcpyAsync(host_dst, p, es * (size_t)cnt, cudaMemcpyDeviceToHost, ctx->s_main) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->s_main) != cudaSuccess) {
    fs_set_error("fs_ctx_read: copy failed");
    return FS_ECUDA;
  }
  return FS_OK;
}

int fs_ctx_write(FsCtx* ctx, int id, const void* host_src) {
  if (!ctx || !host_src) return FS_EARG;
  int64_t cnt = 0;
  size_t es = 0;
  void* p = field_ptr(ctx, id, &cnt, &es);
  if (cnt < 0) {
    fs_set_error("fs_ctx_write: unknown field id %d", id);
    return FS_EARG;
  }
  if (cnt == 0) return FS_OK;
  cudaStreamSynchronize(ctx->s_dom);
  if (cudaMemcpyAsync(p, host_src, es * (size_t)cnt, cudaMemcpyHostToDevice, ctx->s_main) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->s_main) != cudaSuccess) {
    fs_set_error("fs_ctx_write: copy failed");
    return FS_ECUDA;
  }
  return FS_OK;
}

}  // extern "C"

// ---- one outer step ----------------------------------------------------------
static int flame_mask_and_gas_adv(FsCtx* C, double dt) {
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  if (cudaMemsetAsync(C->active_count, 0, sizeof(unsigned long long), s) != cudaSuccess)
    return ctx_fail(C, FS_ECUDA, "active_count");
  CK(fs_active_count(C->n, f[W_OMEGA], f[S_TG], f[S_YF], C->active_count, nullptr, s),
     "active_count");
  CK(fs_gas_energy_adv(&C->g, f[S_TG], f[S_U], f[S_V], f[S_W], f[W_T1], dt, 2.0e-5, c.T_amb, s),
     "gas_adv");
  std::swap(f[S_TG], f[W_T1]);
  return FS_OK;
}

struct SubCounts {
  int n_sc, n_pr;
  double dts_sc, dts_pr;
};

static int substep_prep(FsCtx* C, double dt, SubCounts* sc) {
  const FsCaseDesc& c = C->c;
  const double dt_sub = dt / N_SUB;
  const double* fl[1] = {C->f[S_NU]};
  const int modes[1] = {2};
  double nu_in = 0.0;
  CK(fs_field_max_multi(&C->g, 1, fl, modes, &nu_in, C->max_scratch, C->s_main), "nu_max");
  nsub_from(c, nu_in, SC_T, dt_sub, &sc->n_sc, &sc->dts_sc);
  nsub_from(c, nu_in, PR_T, dt_sub, &sc->n_pr, &sc->dts_pr);
  return FS_OK;
}

// the mixed form's FP32 copies of the fields the sub-steps read
static int to32(FsCtx* C) {
  if (C->c.form != 1) return FS_OK;
  double** f = C->f;
  float** h = C->h32;
  const void* src[14] = {f[S_TG], f[S_YF], f[S_YO], f[S_YH], f[S_RHO], f[S_U], f[S_V],
                         f[S_W], f[S_K], f[S_EPS], f[S_NU], f[B_SP], f[B_SD], f[B_QGC]};
  void* dst[14] = {h[F32_TG], h[F32_YF], h[F32_YO], h[F32_YH], h[F32_RHO], h[F32_U], h[F32_V],
                   h[F32_W], h[F32_K], h[F32_EPS], h[F32_NU], h[F32_SP], h[F32_SD], h[F32_QGC]};
  CK(fs_convert(C->n, 14, src, dst, 1, C->s_main), "to_f32");
  return FS_OK;
}

// the sub-steps' results back into the FP64 state
static int from32(FsCtx* C) {
  if (C->c.form != 1) return FS_OK;
  double** f = C->f;
  float** h = C->h32;
  const void* src[6] = {h[F32_TG], h[F32_YF], h[F32_YO], h[F32_YH], h[F32_OMEGA], h[F32_QCOMB]};
  void* dst[6] = {f[S_TG], f[S_YF], f[S_YO], f[S_YH], f[W_OMEGA], f[W_QCOMB]};
  CK(fs_convert(C->n, 6, src, dst, 0, C->s_main), "to_f64");
  return FS_OK;
}

static int substep_chem32(FsCtx* C, double dt_sub, const SubCounts& sc) {
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  float** h = C->h32;
  CK(fs_edc_f32(C->n, h[F32_RHO], h[F32_TG], h[F32_YF], h[F32_YO], h[F32_K], h[F32_EPS],
                h[F32_YH], h[F32_OMEGA], c.chi_rad, 1100.0, dt_sub, 1, 1.3, 17000000.0,
                c.edc_extinction_enable, C->edc32_scratch, s),
     "edc_f32");
  {
    const float* Ys[3] = {h[F32_YF], h[F32_YO], h[F32_YH]};
    float* Yo[3] = {h[F32_T1], h[F32_T2], h[F32_T3]};
    const double Yin[3] = {0.0, 0.232, 0.0};
    CK(fs_species_step_f32(&C->g, Ys, Yo, h[F32_SP], h[F32_SD], Yin, h[F32_RHO], h[F32_U],
                           h[F32_V], h[F32_W], dt_sub, 1.0e-5, 0.232, s),
       "species_f32");
    std::swap(h[F32_YF], h[F32_T1]);
    std::swap(h[F32_YO], h[F32_T2]);
    std::swap(h[F32_YH], h[F32_T3]);
  }
  const double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {1.0, 0.232, 1.0};
  for (int q = 0; q < sc.n_sc; ++q) {
    const float* Ys[3] = {h[F32_YF], h[F32_YO], h[F32_YH]};
    float* Yo[3] = {h[F32_T1], h[F32_T2], h[F32_T3]};
    CK(fs_turb_diffusion_substep_f32(&C->g, 3, Ys, Yo, h[F32_NU], SC_T, sc.dts_sc,
                                     q == sc.n_sc - 1 ? 1 : 0, lo, hi, s),
       "turb_diff_Y_f32");
    std::swap(h[F32_YF], h[F32_T1]);
    std::swap(h[F32_YO], h[F32_T2]);
    std::swap(h[F32_YH], h[F32_T3]);
  }
  return FS_OK;
}

static int substep_energy32(FsCtx* C, double dt_sub, int drip, const SubCounts& sc) {
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  float** h = C->h32;
  CK(fs_gas_energy_update_f32(&C->g, h[F32_TG], h[F32_RHO], h[F32_YH], f[S_TS], h[F32_SP],
                              h[F32_SD], h[F32_QGC], f[W_QRADG], h[F32_QCOMB], dt_sub, c.T_amb,
                              c.h_bed, drip, c.n_z_bed, c.i_src_start, c.i_src_end, s),
     "gas_update_f32");
  CK(fs_solid_conduction_capped(&C->g, f[S_TS], f[S_AS], f[W_T4], 0.20, 500.0, 1300.0, dt_sub,
                                c.T_amb, T_CAP, s),
     "solid_cond");
  std::swap(f[S_TS], f[W_T4]);
  if (sc.n_pr > 0) {
    const double lo[1] = {c.T_amb}, hi[1] = {T_CAP};
    for (int q = 0; q < sc.n_pr; ++q) {
      const float* in[1] = {h[F32_TG]};
      float* o[1] = {h[F32_T4]};
      CK(fs_turb_diffusion_substep_f32(&C->g, 1, in, o, h[F32_NU], PR_T, sc.dts_pr,
                                       q == sc.n_pr - 1 ? 1 : 0, lo, hi, s),
         "turb_diff_T_f32");
      std::swap(h[F32_TG], h[F32_T4]);
    }
  } else {
    CK(fs_clip_f32(C->n, h[F32_TG], c.T_amb, T_CAP, s), "cap_Tg_f32");
  }
  return FS_OK;
}

static int substep_chem(FsCtx* C, double dt_sub, const SubCounts& sc) {
  if (C->c.form == 1) return substep_chem32(C, dt_sub, sc);
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  CK(fs_edc(C->n, f[S_RHO], f[S_TG], f[S_YF], f[S_YO], f[S_K], f[S_EPS], f[S_YH], f[W_OMEGA],
            c.chi_rad, 1100.0, dt_sub, 1, 1.3, 17000000.0, c.edc_extinction_enable,
            C->edc_scratch, s),
     "edc");
  {
    const double* Ys[3] = {f[S_YF], f[S_YO], f[S_YH]};
    double* Yo[3] = {f[W_T1], f[W_T2], f[W_T3]};
    const double Yin[3] = {0.0, 0.232, 0.0};
    CK(fs_species_step(&C->g, Ys, Yo, f[B_SP], f[B_SD], Yin, f[S_RHO], f[S_U], f[S_V], f[S_W],
                       dt_sub, 1.0e-5, 0.232, s),
       "species");
    std::swap(f[S_YF], f[W_T1]);
    std::swap(f[S_YO], f[W_T2]);
    std::swap(f[S_YH], f[W_T3]);
  }
  const double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {1.0, 0.232, 1.0};
  for (int q = 0; q < sc.n_sc; ++q) {
    const double* Ys[3] = {f[S_YF], f[S_YO], f[S_YH]};
    double* Yo[3] = {f[W_T1], f[W_T2], f[W_T3]};
    CK(fs_turb_diffusion_substep(&C->g, 3, Ys, Yo, f[S_NU], SC_T, sc.dts_sc,
                                 q == sc.n_sc - 1 ? 1 : 0, lo, hi, s),
       "turb_diff_Y");
    std::swap(f[S_YF], f[W_T1]);
    std::swap(f[S_YO], f[W_T2]);
    std::swap(f[S_YH], f[W_T3]);
  }
  return FS_OK;
}

static int substep_energy(FsCtx* C, double dt_sub, int drip, const SubCounts& sc) {
  if (C->c.form == 1) return substep_energy32(C, dt_sub, drip, sc);
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  // the gas-energy update and the capped solid conduction in one pass
  CK(fs_gas_energy_solid_update(&C->g, f[S_TG], f[S_RHO], f[S_YH], f[S_TS], f[B_SP], f[B_SD],
                                f[B_QGC], f[W_QRADG], f[W_QCOMB], dt_sub, c.T_amb, c.h_bed, drip,
                                c.n_z_bed, c.i_src_start, c.i_src_end, f[S_AS], f[W_T4], 0.20,
                                500.0, 1300.0, c.T_amb, T_CAP, s),
     "gas_update + solid_cond");
  std::swap(f[S_TS], f[W_T4]);
  if (sc.n_pr > 0) {
    const double lo[1] = {c.T_amb}, hi[1] = {T_CAP};
    for (int q = 0; q < sc.n_pr; ++q) {
      const double* in[1] = {f[S_TG]};
      double* o[1] = {f[W_T4]};
      CK(fs_turb_diffusion_substep(&C->g, 1, in, o, f[S_NU], PR_T, sc.dts_pr,
                                   q == sc.n_pr - 1 ? 1 : 0, lo, hi, s),
         "turb_diff_T");
      std::swap(f[S_TG], f[W_T4]);
    }
  } else {
    CK(fs_clip(C->n, f[S_TG], c.T_amb, T_CAP, s), "cap_Tg");
  }
  return FS_OK;
}

static int reinit_levelset(FsCtx* C) {
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  // LevelSetFront3D.reinitialize (flame_front_3d.py:339-355)
  if (cudaMemcpyAsync(f[W_PHI0], f[S_PHI], 8 * (size_t)C->n, cudaMemcpyDeviceToDevice, s) !=
      cudaSuccess)
    return ctx_fail(C, FS_ECUDA, "reinit");
  double dzmin = c.dz[0];
  for (int k = 1; k < c.nz; ++k) dzmin = c.dz[k] < dzmin ? c.dz[k] : dzmin;
  const double dtau = 0.5 * pymin({c.dx, c.dy, dzmin});
  for (int q = 0; q < 5; ++q) {
    CK(fs_levelset(&C->g, f[S_PHI], f[W_PHI0], f[W_T5], dtau, 2, s), "reinit");
    std::swap(f[S_PHI], f[W_T5]);
  }
  return FS_OK;
}

// One outer step; *alive = 0 once the reference loop would exit.
static int one_step(FsCtx* C, int* alive) {
  const FsCaseDesc& c = C->c;
  cudaStream_t s = C->s_main;
  double** f = C->f;
  const FsGrid* gp = &C->g;
  C->step_count += 1;
  FsStepOut d{};
  // --- 0. adaptive dt (spread_3d.py:1906-1941)
  {
    const double* fl[5] = {f[S_U], f[S_V], f[S_W], f[S_NU], f[S_TG]};
    const int modes[5] = {0, 0, 0, 1, 1};
    double m[5];
    CK(fs_field_max_multi(gp, 5, fl, modes, m, C->max_scratch, s), "maxima");
    const double u_now = pymax({m[0], m[1], m[2], c.U_mf, std::sqrt(G_ACC * c.h_bed * 0.5), 0.1});
    const double nu_now = pymax({m[3], 1.0e-3});
    const double dt_adv = c.cfl * pymin({c.dx, c.dy, c.dz_min}) / u_now;
    const double dt_diff = 0.25 * c.dz_min * c.dz_min / nu_now;
    double dt_new = pymin({dt_adv, dt_diff, 0.05});
    dt_new = pymin({dt_new, C->dt * 1.5});
    if (dt_new < c.min_dt_s) dt_new = c.min_dt_s;
    if (!std::isfinite(m[4])) {
      snprintf(C->err, sizeof(C->err), "State NaN/Inf at t=%.3fs -- simulation exploded.", C->t);
      fs_set_error("%s", C->err);
      return FS_ENONFINITE;
    }
    C->dt = dt_new;
  }
  const double dt = C->dt, t = C->t;
  const int ign = t < c.ignition_duration_s ? 1 : 0;
  // --- 1. rho_prev, EoS, inlet O2 (spread_3d.py:1984-2050)
  CK(fs_eos(gp, f[S_RHO], f[W_RHO_PREV], f[S_TG], f[S_YO], c.T_amb, s), "eos");
  // --- 2. Lagrangian bed (spread_3d.py:2064-2181)
  FsBedParams bp{dt, c.h_conv, c.rho_solid_true, c.cp_solid, c.eps_solid, c.T_amb,
                 c.view_factor, c.h_bed, c.kappa_bed_eff, c.char_ox_flux_cap, c.char_ox_ash_exp,
                 1, 1, 1, 1, c.drying_mode, c.view_factor_geometric, c.n_per_cell, nullptr,
                 f[W_QRAD], ign, c.n_z_bed, c.i_src_start, c.i_src_end};
  CK(fs_bed_step(gp, &C->parts, &C->segs, &C->src, &bp, f[S_TG], f[S_YO], s), "bed_step");
  CK(fs_bed_aggregate(&C->parts, &C->segs, f[S_TS], 0, s), "bed_aggregate_Ts");
  CK(fs_bed_hcond(gp, f[S_TS], C->hcond_scratch, f[S_AS], c.n_z_bed, 0.20, c.rho_solid_true,
                  c.cp_solid, dt, &C->parts, &C->segs, C->seg_of_cell, s),
     "bed_hcond");
  // --- 8 (started here). DOM + M_local aggregation on the second stream
  const int every = c.dom_subcycle_every > 1 ? c.dom_subcycle_every : 1;
  const bool dom_now = C->step_count % every == 0;
  const bool overlap = dom_now && c.overlap_dom;
  if (overlap) {
    if (cudaEventRecord(C->ev_ready, s) != cudaSuccess) return ctx_fail(C, FS_ECUDA, "ready");
    {
      std::lock_guard<std::mutex> lk(C->mu);
      C->inputs_rc = -1;
      C->done_rc = -1;
      C->job_err.clear();
      C->job = true;
    }
    C->cv.notify_all();
  }
  // --- 3/4. drag + tentative momentum (spread_3d.py:2223-2276)
  CK(fs_tentative_velocity(gp, f[S_U], f[S_V], f[S_W], f[S_RHO], f[S_TG], nullptr, nullptr,
                           nullptr, f[S_AS], c.sav, c.canopy_C_d, C->u_inlet, C->zero2, C->zero2,
                           f[W_T1], f[W_T2], f[W_T3], dt, c.T_amb, s),
     "momentum");
  std::swap(f[S_U], f[W_T1]);
  std::swap(f[S_V], f[W_T2]);
  std::swap(f[S_W], f[W_T3]);
  // --- 5. projection (spread_3d.py:2300-2360)
  CK(fs_div_target(C->n, f[S_RHO], f[W_RHO_PREV], f[B_SP], f[B_SD], dt, f[W_DIVT], s),
     "div_target");
  CK(fs_proj_rebuild(C->proj, f[S_RHO], s), "proj_rebuild");
  for (int it = 0; it < c.proj_max_iter; ++it) {
    int its = 0;
    CK(fs_proj_project(C->proj, f[S_U], f[S_V], f[S_W], C->u_inlet, f[W_DIVT], dt,
                       c.projection_rtol, c.proj_maxiter, &its, s),
       "proj_project");
    d.cg_iters += its;
    double res = 0.0;
    CK(fs_divergence_max(gp, f[S_U], f[S_V], f[S_W], C->u_inlet, f[W_DIVT], nullptr, &res, s),
       "divergence");
    d.div_max = res;
    d.proj_iters = it + 1;
    if (res < c.proj_div_tol) break;
  }
  // --- 6. outflow sponge (spread_3d.py:2369)
  CK(fs_outflow_sponge(gp, f[S_U], C->u_inlet, C->sigma_x, f[S_YF], 1.0e-3, dt, s), "sponge");
  // --- 7. k-epsilon (spread_3d.py:2409)
  CK(fs_k_epsilon(gp, f[S_K], f[S_EPS], f[S_U], f[S_V], f[S_W], f[S_TG], f[S_AS], C->u_inlet,
                  C->k_wall, C->eps_wall, f[W_T1], f[W_T2], f[W_T3], nullptr, nullptr, c.sav, dt,
                  c.T_amb, c.canopy_beta_p, c.canopy_beta_d, s),
     "k_eps");
  std::swap(f[S_K], f[W_T1]);
  std::swap(f[S_EPS], f[W_T2]);
  std::swap(f[S_NU], f[W_T3]);
  // --- 8. DOM (every dom_subcycle_every steps) + soil (spread_3d.py:2472-2514)
  const double dt_sub = dt / N_SUB;
  SubCounts sc{};
  bool early = false;
  if (overlap) {
    // once the DOM has read its inputs, the flame mask, the gas advection and
    // the chemistry and species half of the first sub-step run during the
    // sweeps (none of it is read by the soil step or the ignition pulse)
    int rc = wait_state(C, &C->inputs_rc);
    if (rc != FS_OK) {
      wait_state(C, &C->done_rc);
      return rc;
    }
    if (cudaStreamWaitEvent(s, C->ev_inputs, 0) != cudaSuccess)
      return ctx_fail(C, FS_ECUDA, "wait inputs");
    rc = flame_mask_and_gas_adv(C, dt);
    if (rc == FS_OK) rc = substep_prep(C, dt, &sc);
    if (rc == FS_OK) rc = to32(C);
    if (rc == FS_OK) rc = substep_chem(C, dt_sub, sc);
    const int rd = wait_state(C, &C->done_rc);
    if (rc != FS_OK) return rc;
    if (rd != FS_OK) return rd;
    if (cudaStreamWaitEvent(s, C->ev_done, 0) != cudaSuccess)
      return ctx_fail(C, FS_ECUDA, "wait dom");
    d.dom_iters = fs_dom_iterations(C->dom);
    early = true;
  } else if (dom_now) {
    CK(fs_bed_aggregate(&C->parts, &C->segs, f[W_MLOC], 1, s), "bed_aggregate_M");
    CK(fs_dom_solve(C->dom, f[S_TS], f[S_TG], f[S_AS], f[W_OMEGA], c.sav, c.T_amb, C->T_soil,
                    f[S_YH], f[S_RHO], f[W_MLOC], f[W_QRAD], f[W_QRADG], C->q_in_soil, s),
       "dom_solve");
    d.dom_iters = fs_dom_iterations(C->dom);
  }
  CK(fs_soil_step(c.n_soil, c.ny, c.nx, C->T_soil, C->q_in_soil, dt, C->soil_dz, C->soil_da,
                  C->soil_db, 0.48, 1500.0, 800.0, 0.85, c.T_amb, s),
     "soil");
  // --- 9. ignition pulse on the top bed layer of the source strip (:2528-2532)
  if (ign && c.n_z_bed > 0)
    CK(fs_ignition_pulse(gp, f[W_QRAD], c.n_z_bed - 1, c.i_src_start, c.i_src_end,
                         240000.0 * c.ignition_q_mult, s),
       "ignition_pulse");
  if (!early) {
    // --- 10/11. flame mask, gas-temperature advection
    int rc = flame_mask_and_gas_adv(C, dt);
    if (rc == FS_OK) rc = substep_prep(C, dt, &sc);
    if (rc == FS_OK) rc = to32(C);
    if (rc == FS_OK) rc = substep_chem(C, dt_sub, sc);
    if (rc != FS_OK) return rc;
  }
  // --- 12. ten chemistry/transport sub-steps (:2678-3196); the first one's
  // chemistry and species half ran above
  for (int sub = 0; sub < N_SUB; ++sub) {
    if (sub > 0) {
      int rc = substep_chem(C, dt_sub, sc);
      if (rc != FS_OK) return rc;
    }
    int rc = substep_energy(C, dt_sub, ign, sc);
    if (rc != FS_OK) return rc;
  }
  {
    int rc = from32(C);
    if (rc != FS_OK) return rc;
  }
  // --- 13. level set (passive: v_n = 0, so evolve leaves phi; reinit every 10)
  C->lset_step += 1;
  if (C->lset_step % 10 == 0) {
    int rc = reinit_levelset(C);
    if (rc != FS_OK) return rc;
  }
  // one wait for the exit tests and the front tracking: the active-cell count
  // and the two phi rows they read (phi does not change again in this step)
  const int jm = c.ny / 2;
  const double* row0 = f[S_PHI] + ((int64_t)1 * c.ny + jm) * c.nx;
  const double* row1 = f[S_PHI] + ((int64_t)(c.n_z_bed / 2) * c.ny + jm) * c.nx;
  if (cudaMemcpyAsync(C->h_count, C->active_count, sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(C->h_rows, row0, 8 * (size_t)c.nx, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(C->h_rows + c.nx, row1, 8 * (size_t)c.nx, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess)
    return ctx_fail(C, FS_ECUDA, "exit readback");
  CK(fs_stream_wait(s), "exit readback");
  if (fs_stencil_status(1) != 0) {
    snprintf(C->err, sizeof(C->err),
             "a stencil kernel's bounded shared-memory staging wait gave up");
    fs_set_error("%s", C->err);
    return FS_ETIMEOUT;
  }
  const unsigned long long n_active = *C->h_count;
  const double front_lset = front_from_row(C->h_rows, c.nx, c.dx);
  bool exit_now = false;
  if (n_active == 0 && t > c.ignition_duration_s + 2.0) {
    C->extinct_count += 1;
    if (C->extinct_count > 50) exit_now = true;
  } else {
    C->extinct_count = 0;
  }
  if (front_lset > c.bed_x_end - c.dx) exit_now = true;
  if (exit_now) {
    C->finished = 1;
    *alive = 0;
    C->last = d;
    return FS_OK;
  }
  // --- 14. closing EoS (:3440) and clock
  CK(fs_eos(gp, f[S_RHO], nullptr, f[S_TG], nullptr, c.T_amb, s), "eos2");
  const double fx = front_from_row(C->h_rows + c.nx, c.nx, c.dx);
  if (std::isfinite(fx) && fx > C->front_x.back()) {
    C->front_t.push_back(t);
    C->front_x.push_back(fx);
  }
  C->t = t + dt;
  d.t = C->t;
  d.dt = dt;
  C->last = d;
  *alive = 1;
  return FS_OK;
}

extern "C" {

int fs_step(FsCtx* ctx, int n_steps, FsStepOut* out) {
  if (!ctx || n_steps < 0) {
    fs_set_error("fs_step: bad argument");
    return FS_EARG;
  }
  FsCtx* C = ctx;
  cudaSetDevice(C->dev);
  int taken = 0, rc = FS_OK;
  for (int q = 0; q < n_steps && !C->finished; ++q) {
    int alive = 0;
    rc = one_step(C, &alive);
    if (rc != FS_OK) break;
    ++taken;
    if (!alive) break;
  }
  if (rc == FS_OK && cudaStreamSynchronize(C->s_main) != cudaSuccess)
    rc = ctx_fail(C, FS_ECUDA, "fs_step");
  if (out) {
    *out = C->last;
    out->steps = taken;
    out->finished = C->finished;
    out->step_count = C->step_count;
    out->t = C->t;
    out->dt = C->dt;
  }
  return rc;
}

int fs_batch_run(FsCtx* const* ctxs, int n, int n_steps, FsStepOut* outs) {
  if (!ctxs || n < 0 || n_steps < 0) {
    fs_set_error("fs_batch_run: bad argument");
    return FS_EARG;
  }
  for (int q = 0; q < n; ++q)
    if (!ctxs[q]) {
      fs_set_error("fs_batch_run: context %d is NULL", q);
      return FS_EARG;
    }
  std::vector<int> rcs(n, FS_OK);
  std::vector<std::string> errs(n);
  std::vector<std::thread> th;
  th.reserve(n);
  for (int q = 0; q < n; ++q) {
    th.emplace_back([&, q] {
      rcs[q] = fs_step(ctxs[q], n_steps, outs ? outs + q : nullptr);
      if (rcs[q] != FS_OK) errs[q] = fs_last_error();
    });
  }
  for (auto& x : th) x.join();
  for (int q = 0; q < n; ++q)
    if (rcs[q] != FS_OK) {
      fs_set_error("fs_batch_run: case %d: %s", q, errs[q].c_str());
      return rcs[q];
    }
  return FS_OK;
}

}  // extern "C"
