// Level-set front (flame_front_3d.py:114-400 LevelSetFront3D) and the
// active-flame mask (flame_front_3d.py:756-813).
#include "common.cuh"
#include "kernels.h"

__device__ __forceinline__ void ls_dz(const GridDev& g, int k, double& im, double& ip) {
  const int nz = g.nz;
  if (k == 0) {
    im = 1.0 / g.dz[0];
    ip = nz > 1 ? 2.0 / (g.dz[0] + g.dz[1]) : 1.0 / g.dz[0];
  } else if (k == nz - 1) {
    ip = 1.0 / g.dz[nz - 1];
    im = 2.0 / (g.dz[nz - 1] + g.dz[nz - 2]);
  } else {
    im = 2.0 / (g.dz[k] + g.dz[k - 1]);
    ip = 2.0 / (g.dz[k] + g.dz[k + 1]);
  }
}

// Godunov |grad phi|; sgn > 0 (or evolve mode) uses the forward form,
// sgn <= 0 the backward form (reinit_godunov_grad, flame_front_3d.py:192-263).
__device__ __forceinline__ double ls_grad(const GridDev& g, const double* __restrict__ phi, int k,
                                          int j, int i, int64_t c, double inv_dx, double inv_dy,
                                          bool forward) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t sy = nx, sz = (int64_t)nx * ny;
  double im, ip;
  ls_dz(g, k, im, ip);
  const double pc = phi[c];
  double dmx = i > 0 ? (pc - phi[c - 1]) * inv_dx : 0.0;
  double dpx = i < nx - 1 ? (phi[c + 1] - pc) * inv_dx : 0.0;
  int jm = j > 0 ? j - 1 : ny - 1;
  int jp = j < ny - 1 ? j + 1 : 0;
  double dmy = (pc - phi[c - (int64_t)j * sy + (int64_t)jm * sy]) * inv_dy;
  double dpy = (phi[c - (int64_t)j * sy + (int64_t)jp * sy] - pc) * inv_dy;
  double dmz = k > 0 ? (pc - phi[c - sz]) * im : 0.0;
  double dpz = k < nz - 1 ? (phi[c + sz] - pc) * ip : 0.0;
  double a, b, cc, d, e, f;
  if (forward) {
    a = dmx > 0.0 ? dmx : 0.0; b = dpx < 0.0 ? dpx : 0.0;
    cc = dmy > 0.0 ? dmy : 0.0; d = dpy < 0.0 ? dpy : 0.0;
    e = dmz > 0.0 ? dmz : 0.0; f = dpz < 0.0 ? dpz : 0.0;
  } else {
    a = dmx < 0.0 ? dmx : 0.0; b = dpx > 0.0 ? dpx : 0.0;
    cc = dmy < 0.0 ? dmy : 0.0; d = dpy > 0.0 ? dpy : 0.0;
    e = dmz < 0.0 ? dmz : 0.0; f = dpz > 0.0 ? dpz : 0.0;
  }
  return sqrt(a * a + b * b + cc * cc + d * d + e * e + f * f);
}

// mode 0: grad_out = |grad phi| (godunov_grad_norm)
// mode 1: phi_out = phi - dt v_n |grad phi|         (LevelSetFront3D.evolve)
// mode 2: phi_out = phi - dtau s(phi0) (|grad| - 1)  (one Sussman reinit sub-step)
__global__ void k_levelset(GridDev g, const double* __restrict__ phi, const double* __restrict__ aux,
                           double* out, double coef, int mode, double inv_dx, double inv_dy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  int64_t c = cidx(g, k, j, i);
  if (mode == 0) {
    out[c] = ls_grad(g, phi, k, j, i, c, inv_dx, inv_dy, true);
  } else if (mode == 1) {
    double gr = ls_grad(g, phi, k, j, i, c, inv_dx, inv_dy, true);
    out[c] = phi[c] - coef * aux[c] * gr;
  } else {
    double p0 = aux[c];
    double s = p0 > 0.0 ? 1.0 : (p0 < 0.0 ? -1.0 : 0.0);
    double gr = ls_grad(g, phi, k, j, i, c, inv_dx, inv_dy, s > 0.0);
    out[c] = phi[c] - coef * s * (gr - 1.0);
  }
}

int launch_levelset(const GridDev& g, const double* phi, const double* aux, double* out,
                    double coef, int mode, cudaStream_t st) {
  Launch3 L = launch_cells(g);
  k_levelset<<<L.grid, L.block, 0, st>>>(g, phi, aux, out, coef, mode, 1.0 / g.dx, 1.0 / g.dy); fs_count_launch();
  return cuda_status();
}

// Active-flame cell count (compute_phi_flame_from_state: active =
// omega > 1e-3 or (T_g > 1000 and Y_F > 1e-3)); flame_body_mask = active.
__global__ void k_active_count(int64_t n, const double* __restrict__ om,
                               const double* __restrict__ Tg, const double* __restrict__ YF,
                               unsigned long long* count, unsigned char* mask) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool a = false;
  if (c < n) {
    a = (om[c] > 1.0e-3) || (Tg[c] > 1000.0 && YF[c] > 1.0e-3);
    if (mask) mask[c] = a ? 1 : 0;
  }
  unsigned b = __ballot_sync(0xffffffffu, a);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, (unsigned long long)__popc(b));
}

int launch_active_count(int64_t n, const double* om, const double* Tg, const double* YF,
                        unsigned long long* count, unsigned char* mask, cudaStream_t st) {
  k_active_count<<<blocks_for(n, 256), 256, 0, st>>>(n, om, Tg, YF, count, mask); fs_count_launch();
  return cuda_status();
}
