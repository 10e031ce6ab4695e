// Learned pressure preconditioner: a 3-D convolutional U-Net applied to the
// CG residual, with its training step (forward, backward, Adam) on the GPU.
//
// No counterpart in the reference, whose pressure solve is BiCGSTAB with an
// FFT preconditioner (projection_3d.py:756-791).  The network:
//   levels 0-3 (each ceil(n/2) per axis), channels 16 / 32 / 48 / 64;
//   encoder: two 3x3x3 conv + ReLU per level, 2x2x2 average (fixed 1/8) down;
//   decoder: nearest-neighbour up, concatenated before the skip, one conv+ReLU;
//   head: 1x1 conv 16 -> 1, no activation.
// Activations are bfloat16 in (Z, Y, X, C) order (channel innermost, C a
// multiple of 16); weights are fp32 masters repacked to bfloat16 tensor-core
// fragments after every update; every convolution (forward, adjoint and
// weight gradient) is an implicit GEMM on mma.sync.m16n8k16 bf16 -> fp32.
// The forward input is the residual scaled to unit RMS in channel 0 (the
// preconditioner is used in flexible CG, where the scale of its output does
// not matter).
#include <cuda_bf16.h>
#include <vector>
#include <cmath>
#include "common.cuh"
#include "kernels.h"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int UN_NL = 11;   // conv layers
constexpr int UN_HEAD = 16;
struct LayerSpec { int cin, cout, level; };
const LayerSpec kSpec[UN_NL] = {
    {16, 16, 0}, {16, 16, 0}, {16, 32, 1}, {32, 32, 1}, {32, 48, 2}, {48, 48, 2},
    {48, 64, 3}, {64, 64, 3}, {112, 48, 2}, {80, 32, 1}, {48, 16, 0}};

constexpr int CONV_WARPS = 4;
constexpr int WG_STAGE = 64;     // voxels staged per weight-gradient step
constexpr int RB = 256;          // reduction blocks

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ uint32_t pack2f(float lo, float hi) {
  return pack2(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi));
}
__device__ __forceinline__ float lo_f(uint32_t v) {
  return __bfloat162float(__ushort_as_bfloat16((unsigned short)(v & 0xFFFFu)));
}
__device__ __forceinline__ float hi_f(uint32_t v) {
  return __bfloat162float(__ushort_as_bfloat16((unsigned short)(v >> 16)));
}

struct Dims { int nz, ny, nx; int64_t n; };

// ---------------------------------------------------------------------------
// convolution (forward and adjoint share this kernel)
//   out[p][co] = act( bias[co] + sum_tap sum_ci in[p + off(tap)][ci] * W[tap][ci][co] )
// then out *= (mask[p][co] > 0) when mask is given.  W arrives packed as
// mma B fragments: [(tap * cin/16 + kc) * NT + nt][lane] (uint2).  Each warp
// owns MT x 16 consecutive voxels and all NT x 8 output channels.  (A
// variant that staged each row's 3x3 neighbour rows in shared memory and read
// the A fragments by ldmatrix measured 9 % slower for the whole network on the
// 400x120x60 grid, so the fragments are loaded directly.)
// ---------------------------------------------------------------------------
struct ConvArgs {
  const bf16* in;
  int cin;
  Dims d;
  const uint2* w;
  const float* bias;
  bf16* out;
  const bf16* mask;
  int relu;
};

template <int NT, int MT>
__global__ void __launch_bounds__(CONV_WARPS * 32) k_un_conv(ConvArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nx = a.d.nx, ny = a.d.ny, nz = a.d.nz;
  const int64_t n = a.d.n;
  const int64_t vbase = ((int64_t)blockIdx.x * CONV_WARPS + warp) * (MT * 16);
  if (vbase >= n) return;
  int vz[MT][2], vy[MT][2], vx[MT][2];
  bool ok[MT][2];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t v = vbase + mt * 16 + g + 8 * h;
      ok[mt][h] = v < n;
      const int64_t vv = ok[mt][h] ? v : 0;
      vx[mt][h] = (int)(vv % nx);
      vy[mt][h] = (int)((vv / nx) % ny);
      vz[mt][h] = (int)(vv / ((int64_t)nx * ny));
    }
  float acc[MT][NT][4];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[mt][nt][q] = 0.f;
  const int KC = a.cin >> 4;
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(a.in);
  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const uint32_t* src[MT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int z2 = vz[mt][h] + dz, y2 = vy[mt][h] + dy, x2 = vx[mt][h] + dx;
        const bool in = ok[mt][h] && z2 >= 0 && z2 < nz && y2 >= 0 && y2 < ny && x2 >= 0 &&
                        x2 < nx;
        src[mt][h] = in ? in32 + (((int64_t)z2 * ny + y2) * nx + x2) * (a.cin >> 1) + t
                        : nullptr;
      }
    const uint2* wp = a.w + (size_t)tap * KC * NT * 32 + lane;
    for (int kc = 0; kc < KC; ++kc) {
      uint32_t af[MT][4];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        af[mt][0] = src[mt][0] ? __ldg(src[mt][0] + kc * 8) : 0u;
        af[mt][1] = src[mt][1] ? __ldg(src[mt][1] + kc * 8) : 0u;
        af[mt][2] = src[mt][0] ? __ldg(src[mt][0] + kc * 8 + 4) : 0u;
        af[mt][3] = src[mt][1] ? __ldg(src[mt][1] + kc * 8 + 4) : 0u;
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const uint2 b = __ldg(wp + (size_t)(kc * NT + nt) * 32);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[mt][nt], af[mt], b.x, b.y);
      }
    }
  }
  const int cout = NT * 8;
  uint32_t* out32 = reinterpret_cast<uint32_t*>(a.out);
  const uint32_t* mask32 = reinterpret_cast<const uint32_t*>(a.mask);
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!ok[mt][h]) continue;
      const int64_t v = vbase + mt * 16 + g + 8 * h;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int co = nt * 8 + 2 * t;
        float y0 = acc[mt][nt][2 * h], y1 = acc[mt][nt][2 * h + 1];
        if (a.bias) { y0 += a.bias[co]; y1 += a.bias[co + 1]; }
        if (a.relu) { y0 = fmaxf(y0, 0.f); y1 = fmaxf(y1, 0.f); }
        const int64_t o = (v * cout + co) >> 1;
        if (mask32) {
          const uint32_t m = mask32[o];
          if (!(lo_f(m) > 0.f)) y0 = 0.f;
          if (!(hi_f(m) > 0.f)) y1 = 0.f;
        }
        out32[o] = pack2f(y0, y1);
      }
    }
}

// Pack W[tap][cin][cout] (fp32) into B fragments.  transpose = 0: the forward
// operator (K = cin, N = cout).  transpose = 1: the adjoint (K = cout, N = cin,
// taps mirrored): element (k, n) of tap t is W[26 - t][n][k].
__global__ void k_un_pack(const float* __restrict__ W, int cin, int cout, int transpose,
                          uint2* out) {
  const int K = transpose ? cout : cin, N = transpose ? cin : cout;
  const int KC = K >> 4, NT = N >> 3;
  const int64_t total = (int64_t)27 * KC * NT * 32;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int lane = (int)(i & 31);
  int64_t r = i >> 5;
  const int nt = (int)(r % NT); r /= NT;
  const int kc = (int)(r % KC);
  const int tap = (int)(r / KC);
  const int g = lane >> 2, t = lane & 3;
  const int nn = nt * 8 + g;
  auto E = [&](int k) -> float {
    if (!transpose) return W[((int64_t)tap * cin + k) * cout + nn];
    return W[((int64_t)(26 - tap) * cin + nn) * cout + k];
  };
  const int k0 = kc * 16 + 2 * t;
  uint2 v;
  v.x = pack2f(E(k0), E(k0 + 1));
  v.y = pack2f(E(k0 + 8), E(k0 + 9));
  out[i] = v;
}

// ---------------------------------------------------------------------------
// input, pooling, up-sampling with concatenation, head, loss
// ---------------------------------------------------------------------------
// partial sums of r^2 (double) over RB blocks
template <typename TI>
__global__ void k_un_sumsq(int64_t n, const TI* __restrict__ r, double* partial) {
  double s = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double v = (double)r[c];
    s += v * v;
  }
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// scale = 1 / rms(r) (0 for r == 0)
__global__ void k_un_scale(const double* __restrict__ partial, int nb, int64_t n, double* scale) {
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) s += partial[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *scale = s > 0.0 ? 1.0 / sqrt(s / (double)n) : 0.0;
}

// x0[p] = (r[p] * scale, 0, ..., 0) in 16 bf16 channels
template <typename TI>
__global__ void k_un_input(int64_t n, const TI* __restrict__ r, const double* __restrict__ scale,
                           bf16* x0) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const float v = scale ? (float)((double)r[c] * *scale) : (float)r[c];
  uint4 q0, q1;
  q0.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v));
  q0.y = q0.z = q0.w = 0u;
  q1.x = q1.y = q1.z = q1.w = 0u;
  uint4* o = reinterpret_cast<uint4*>(x0 + c * 16);
  o[0] = q0;
  o[1] = q1;
}

// d[pc][c] = bf16( 1/8 * sum of the in-domain children ), one thread per channel pair
__global__ void k_un_pool(const bf16* __restrict__ f, Dims fd, Dims cd, int C, bf16* d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int C2 = C >> 1;
  if (i >= cd.n * C2) return;
  const int c2 = (int)(i % C2);
  const int64_t pc = i / C2;
  const int cx = (int)(pc % cd.nx), cy = (int)((pc / cd.nx) % cd.ny);
  const int cz = (int)(pc / ((int64_t)cd.nx * cd.ny));
  const uint32_t* f32p = reinterpret_cast<const uint32_t*>(f);
  float s0 = 0.f, s1 = 0.f;
  for (int q = 0; q < 8; ++q) {
    const int z = 2 * cz + (q >> 2), y = 2 * cy + ((q >> 1) & 1), x = 2 * cx + (q & 1);
    if (z >= fd.nz || y >= fd.ny || x >= fd.nx) continue;
    const uint32_t v = f32p[(((int64_t)z * fd.ny + y) * fd.nx + x) * C2 + c2];
    s0 += lo_f(v);
    s1 += hi_f(v);
  }
  reinterpret_cast<uint32_t*>(d)[i] = pack2f(s0 * 0.125f, s1 * 0.125f);
}

// g_f[p][c] = bf16( (g_f[p][c] + g_d[parent][c] / 8) * (mask[p][c] > 0) )
__global__ void k_un_pool_bwd(const bf16* __restrict__ gd, Dims cd, bf16* gf,
                              const bf16* __restrict__ mask, Dims fd, int C) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int C2 = C >> 1;
  if (i >= fd.n * C2) return;
  const int c2 = (int)(i % C2);
  const int64_t p = i / C2;
  const int x = (int)(p % fd.nx), y = (int)((p / fd.nx) % fd.ny);
  const int z = (int)(p / ((int64_t)fd.nx * fd.ny));
  const int64_t pc = ((int64_t)(z >> 1) * cd.ny + (y >> 1)) * cd.nx + (x >> 1);
  const uint32_t a = reinterpret_cast<const uint32_t*>(gd)[pc * C2 + c2];
  uint32_t* g32 = reinterpret_cast<uint32_t*>(gf);
  const uint32_t b = g32[i];
  const uint32_t m = reinterpret_cast<const uint32_t*>(mask)[i];
  float v0 = lo_f(b) + lo_f(a) * 0.125f, v1 = hi_f(b) + hi_f(a) * 0.125f;
  if (!(lo_f(m) > 0.f)) v0 = 0.f;
  if (!(hi_f(m) > 0.f)) v1 = 0.f;
  g32[i] = pack2f(v0, v1);
}

// c[p] = ( a[parent(p)] (Ca channels), s[p] (Cs channels) ), 16-byte vectors
__global__ void k_un_upcat(const bf16* __restrict__ a, Dims cd, int Ca,
                           const bf16* __restrict__ s, Dims fd, int Cs, bf16* c) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int Va = Ca >> 3, Vs = Cs >> 3, V = Va + Vs;
  if (i >= fd.n * V) return;
  const int vq = (int)(i % V);
  const int64_t p = i / V;
  uint4 v;
  if (vq < Va) {
    const int x = (int)(p % fd.nx), y = (int)((p / fd.nx) % fd.ny);
    const int z = (int)(p / ((int64_t)fd.nx * fd.ny));
    const int64_t pc = ((int64_t)(z >> 1) * cd.ny + (y >> 1)) * cd.nx + (x >> 1);
    v = reinterpret_cast<const uint4*>(a)[pc * Va + vq];
  } else {
    v = reinterpret_cast<const uint4*>(s)[p * Vs + (vq - Va)];
  }
  reinterpret_cast<uint4*>(c)[i] = v;
}

// adjoint of k_un_upcat, coarse part: g_a[pc][c] = bf16( sum over children g_c[ch][c] )
__global__ void k_un_upcat_bwd_a(const bf16* __restrict__ gc, Dims fd, int Ctot, bf16* ga,
                                 Dims cd, int Ca) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int C2 = Ca >> 1;
  if (i >= cd.n * C2) return;
  const int c2 = (int)(i % C2);
  const int64_t pc = i / C2;
  const int cx = (int)(pc % cd.nx), cy = (int)((pc / cd.nx) % cd.ny);
  const int cz = (int)(pc / ((int64_t)cd.nx * cd.ny));
  const uint32_t* g32 = reinterpret_cast<const uint32_t*>(gc);
  const int T2 = Ctot >> 1;
  float s0 = 0.f, s1 = 0.f;
  for (int q = 0; q < 8; ++q) {
    const int z = 2 * cz + (q >> 2), y = 2 * cy + ((q >> 1) & 1), x = 2 * cx + (q & 1);
    if (z >= fd.nz || y >= fd.ny || x >= fd.nx) continue;
    const uint32_t v = g32[(((int64_t)z * fd.ny + y) * fd.nx + x) * T2 + c2];
    s0 += lo_f(v);
    s1 += hi_f(v);
  }
  reinterpret_cast<uint32_t*>(ga)[i] = pack2f(s0, s1);
}

// adjoint of k_un_upcat, skip part: g_s[p] = g_c[p][Ca:]
__global__ void k_un_upcat_bwd_s(const bf16* __restrict__ gc, int Ctot, int Ca, int64_t n,
                                 bf16* gs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int Vs = (Ctot - Ca) >> 3, Vt = Ctot >> 3, Va = Ca >> 3;
  if (i >= n * Vs) return;
  const int64_t p = i / Vs;
  const int vq = (int)(i % Vs);
  reinterpret_cast<uint4*>(gs)[i] = reinterpret_cast<const uint4*>(gc)[p * Vt + Va + vq];
}

// z[p] = bh + sum_c u0[p][c] * wh[c]  (fp32, c ascending)
__global__ void k_un_head(int64_t n, const bf16* __restrict__ u0, const float* __restrict__ wh,
                          const float* __restrict__ bh, float* zf, double* zd) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t* u = reinterpret_cast<const uint32_t*>(u0) + p * 8;
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const uint32_t v = u[q];
    s += lo_f(v) * wh[2 * q];
    s += hi_f(v) * wh[2 * q + 1];
  }
  s += *bh;
  if (zf) zf[p] = s;
  if (zd) zd[p] = (double)s;
}

// dz = 2 (z - tau) / n, partial sums of (z - tau)^2
__global__ void k_un_loss(int64_t n, const float* __restrict__ z, const float* __restrict__ tau,
                          float* dz, double* partial) {
  double s = 0.0;
  const float inv = 2.0f / (float)n;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const float d = z[c] - tau[c];
    dz[c] = d * inv;
    s += (double)d * (double)d;
  }
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// head adjoint: g_u0[p][c] = bf16(dz[p] wh[c]) * (u0 > 0); partials of
// dwh[c] = sum_p u0[p][c] dz[p] and dbh = sum_p dz[p]  (17 per block)
__global__ void k_un_head_bwd(int64_t n, const bf16* __restrict__ u0, const float* __restrict__ dz,
                              const float* __restrict__ wh, bf16* gu0, float* partial) {
  float s[17];
#pragma unroll
  for (int q = 0; q < 17; ++q) s[q] = 0.f;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float d = dz[p];
    const uint32_t* u = reinterpret_cast<const uint32_t*>(u0) + p * 8;
    uint32_t* go = reinterpret_cast<uint32_t*>(gu0) + p * 8;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t v = u[q];
      const float a0 = lo_f(v), a1 = hi_f(v);
      s[2 * q] += a0 * d;
      s[2 * q + 1] += a1 * d;
      const float g0 = a0 > 0.f ? d * wh[2 * q] : 0.f;
      const float g1 = a1 > 0.f ? d * wh[2 * q + 1] : 0.f;
      go[q] = pack2f(g0, g1);
    }
    s[16] += d;
  }
  __shared__ float sh[17][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 17; ++q) {
    float v = s[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 17) {
    float v = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[threadIdx.x][w];
    partial[(int64_t)blockIdx.x * 17 + threadIdx.x] = v;
  }
}

// ---------------------------------------------------------------------------
// weight and bias gradients
// ---------------------------------------------------------------------------
// part[chunk][tap][ci][co] = sum over the chunk's voxels p of
//   x[p + off(tap)][ci] * gy[p][co]
// grid (chunks, 27), one warp per 16 input channels; WG_STAGE voxels are
// staged in shared memory, then each warp runs mma over 16 voxels at a time
// (M = its 16 input channels, N = 8 output channels per tile, K = voxels).
template <int NT>
__global__ void k_un_wgrad(const bf16* __restrict__ x, int cin, const bf16* __restrict__ gy,
                           Dims d, int64_t chunk, float* part) {
  extern __shared__ __align__(16) unsigned char wg_smem[];
  constexpr int COUT = NT * 8;
  const int XS = cin + 8, GS = COUT + 8;  // padded row strides (elements)
  bf16* xs = reinterpret_cast<bf16*>(wg_smem);
  bf16* gs = xs + WG_STAGE * XS;
  const int tap = blockIdx.y;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int ci0 = warp * 16;
  const int64_t p_begin = (int64_t)blockIdx.x * chunk;
  const int64_t p_end = min(p_begin + chunk, d.n);
  const int xv = cin >> 3, gv = COUT >> 3;  // uint4 vectors per voxel row
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
  auto rd2 = [](const bf16* base, int r0, int stride, int col) -> uint32_t {
    return pack2(base[r0 * stride + col], base[(r0 + 1) * stride + col]);
  };
  for (int64_t p0 = p_begin; p0 < p_end; p0 += WG_STAGE) {
    __syncthreads();
    for (int i = threadIdx.x; i < WG_STAGE * xv; i += blockDim.x) {
      const int r = i / xv, vq = i % xv;
      const int64_t p = p0 + r;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (p < p_end) {
        const int px = (int)(p % d.nx), py = (int)((p / d.nx) % d.ny);
        const int pz = (int)(p / ((int64_t)d.nx * d.ny));
        const int z2 = pz + dz, y2 = py + dy, x2 = px + dx;
        if (z2 >= 0 && z2 < d.nz && y2 >= 0 && y2 < d.ny && x2 >= 0 && x2 < d.nx)
          v = reinterpret_cast<const uint4*>(x)[(((int64_t)z2 * d.ny + y2) * d.nx + x2) * xv + vq];
      }
      *reinterpret_cast<uint4*>(xs + r * XS + vq * 8) = v;
    }
    for (int i = threadIdx.x; i < WG_STAGE * gv; i += blockDim.x) {
      const int r = i / gv, vq = i % gv;
      const int64_t p = p0 + r;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (p < p_end) v = reinterpret_cast<const uint4*>(gy)[p * gv + vq];
      *reinterpret_cast<uint4*>(gs + r * GS + vq * 8) = v;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < WG_STAGE / 16; ++ks) {
      const int k0 = ks * 16 + 2 * t;
      uint32_t af[4];
      af[0] = rd2(xs, k0, XS, ci0 + g);
      af[1] = rd2(xs, k0, XS, ci0 + g + 8);
      af[2] = rd2(xs, k0 + 8, XS, ci0 + g);
      af[3] = rd2(xs, k0 + 8, XS, ci0 + g + 8);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const uint32_t b0 = rd2(gs, k0, GS, nt * 8 + g);
        const uint32_t b1 = rd2(gs, k0 + 8, GS, nt * 8 + g);
        mma_bf16(acc[nt], af, b0, b1);
      }
    }
  }
  float* out = part + ((int64_t)blockIdx.x * 27 + tap) * cin * COUT;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    const int co = nt * 8 + 2 * t;
    *reinterpret_cast<float2*>(out + (int64_t)(ci0 + g) * COUT + co) =
        make_float2(acc[nt][0], acc[nt][1]);
    *reinterpret_cast<float2*>(out + (int64_t)(ci0 + g + 8) * COUT + co) =
        make_float2(acc[nt][2], acc[nt][3]);
  }
}

// out[i] = sum_c part[c * m + i]  (fixed order)
__global__ void k_un_reduce(const float* __restrict__ part, int nparts, int64_t m, float* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  float s = 0.f;
  for (int c = 0; c < nparts; ++c) s += part[(int64_t)c * m + i];
  out[i] = s;
}

// part[block][c] = sum over the block's voxels of gy[p][c]
__global__ void k_un_bsum(const bf16* __restrict__ gy, int64_t n, int cout, float* part) {
  __shared__ float sh[256][2];
  const int C2 = cout >> 1;
  const int R = 256 / C2;
  const int c2 = threadIdx.x % C2, r = threadIdx.x / C2;
  float s0 = 0.f, s1 = 0.f;
  if (r < R) {
    const uint32_t* g32 = reinterpret_cast<const uint32_t*>(gy);
    for (int64_t p = (int64_t)blockIdx.x * R + r; p < n; p += (int64_t)gridDim.x * R) {
      const uint32_t v = g32[p * C2 + c2];
      s0 += lo_f(v);
      s1 += hi_f(v);
    }
  }
  sh[threadIdx.x][0] = s0;
  sh[threadIdx.x][1] = s1;
  __syncthreads();
  if (threadIdx.x < C2) {
    float a0 = 0.f, a1 = 0.f;
    for (int q = 0; q < R; ++q) {
      a0 += sh[q * C2 + threadIdx.x][0];
      a1 += sh[q * C2 + threadIdx.x][1];
    }
    part[(int64_t)blockIdx.x * cout + 2 * threadIdx.x] = a0;
    part[(int64_t)blockIdx.x * cout + 2 * threadIdx.x + 1] = a1;
  }
}

__global__ void k_un_adam(int64_t n, float* p, const float* __restrict__ g, float* m, float* v,
                          float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

// out[p] = base[p] + zf[p] * out_scale / scale   (scale = 1 / rms of the input)
__global__ void k_un_correct(int64_t n, const float* __restrict__ zf, const double* __restrict__ scale,
                             float out_scale, const float* __restrict__ base, float* out) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double s = *scale;
  const float f = s > 0.0 ? (float)((double)out_scale / s) : 0.f;
  out[p] = (base ? base[p] : 0.f) + zf[p] * f;
}

__global__ void k_un_dsum(const double* __restrict__ partial, int nb, double* out) {
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) s += partial[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
}

struct UNetCtx {
  Dims lv[4];
  int64_t nparams;
  int64_t woff[UN_NL], boff[UN_NL], hw, hb;
  float *params = nullptr, *grads = nullptr, *am = nullptr, *av = nullptr;
  uint2 *wf[UN_NL] = {}, *wb[UN_NL] = {};
  bf16 *x0, *e0, *e0b, *d1, *e1, *e1b, *d2, *e2, *e2b, *d3, *e3, *e3b, *c2, *u2, *c1, *u1, *c0,
      *u0;
  bf16 *g_u0, *g_c0, *g_u1, *g_e0b, *g_c1, *g_u2, *g_e1b, *g_c2, *g_e3b, *g_e2b, *g_e3, *g_d3,
      *g_e2, *g_d2, *g_e1, *g_d1, *g_e0;
  float *zf = nullptr, *dz = nullptr, *wpart = nullptr, *bpart = nullptr, *hpart = nullptr;
  double *dpart = nullptr, *scale = nullptr, *loss_d = nullptr, *h_loss = nullptr;
  int64_t wchunk[UN_NL];
  int nchunks[UN_NL];
  int step = 0;
  float out_scale = 1.f;  // z = N(r / rms) * rms * out_scale in unet_correct
  bool failed = false;
  std::vector<void*> owned;
};

template <typename T>
T* un_alloc(UNetCtx* U, int64_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) {
    U->failed = true;
    return nullptr;
  }
  U->owned.push_back(p);
  return (T*)p;
}

#define UN_LAUNCH(...) do { __VA_ARGS__; fs_count_launch(); } while (0)

void launch_conv(const bf16* in, int cin, const Dims& d, const uint2* w, const float* bias,
                 bf16* out, int cout, const bf16* mask, int relu, cudaStream_t st) {
  ConvArgs a{in, cin, d, w, bias, out, mask, relu};
  const int nt = cout / 8;
  auto grid = [&](int mt) { return (unsigned)((d.n + CONV_WARPS * mt * 16 - 1) / (CONV_WARPS * mt * 16)); };
  const int thr = CONV_WARPS * 32;
  switch (nt) {
    case 2: UN_LAUNCH((k_un_conv<2, 2><<<grid(2), thr, 0, st>>>(a))); break;
    case 4: UN_LAUNCH((k_un_conv<4, 2><<<grid(2), thr, 0, st>>>(a))); break;
    case 6: UN_LAUNCH((k_un_conv<6, 2><<<grid(2), thr, 0, st>>>(a))); break;
    case 8: UN_LAUNCH((k_un_conv<8, 2><<<grid(2), thr, 0, st>>>(a))); break;
    case 10: UN_LAUNCH((k_un_conv<10, 1><<<grid(1), thr, 0, st>>>(a))); break;
    case 14: UN_LAUNCH((k_un_conv<14, 1><<<grid(1), thr, 0, st>>>(a))); break;
    default: break;
  }
}

size_t wgrad_smem(int cin, int cout) { return (size_t)WG_STAGE * (cin + 8 + cout + 8) * 2; }

void launch_wgrad(UNetCtx* U, int li, const bf16* x, const bf16* gy, cudaStream_t st) {
  const int cin = kSpec[li].cin, cout = kSpec[li].cout;
  const Dims& d = U->lv[kSpec[li].level];
  dim3 grid(U->nchunks[li], 27);
  const int thr = 2 * cin;
  const size_t sm = wgrad_smem(cin, cout);
  switch (cout / 8) {
    case 2: UN_LAUNCH((k_un_wgrad<2><<<grid, thr, sm, st>>>(x, cin, gy, d, U->wchunk[li], U->wpart))); break;
    case 4: UN_LAUNCH((k_un_wgrad<4><<<grid, thr, sm, st>>>(x, cin, gy, d, U->wchunk[li], U->wpart))); break;
    case 6: UN_LAUNCH((k_un_wgrad<6><<<grid, thr, sm, st>>>(x, cin, gy, d, U->wchunk[li], U->wpart))); break;
    case 8: UN_LAUNCH((k_un_wgrad<8><<<grid, thr, sm, st>>>(x, cin, gy, d, U->wchunk[li], U->wpart))); break;
    default: break;
  }
  const int64_t m = (int64_t)27 * cin * cout;
  UN_LAUNCH((k_un_reduce<<<blocks_for(m, 256), 256, 0, st>>>(U->wpart, U->nchunks[li], m,
                                                             U->grads + U->woff[li])));
  UN_LAUNCH((k_un_bsum<<<RB, 256, 0, st>>>(gy, d.n, cout, U->bpart)));
  UN_LAUNCH((k_un_reduce<<<1, 64, 0, st>>>(U->bpart, RB, cout, U->grads + U->boff[li])));
}

void launch_pack(UNetCtx* U, cudaStream_t st) {
  for (int li = 0; li < UN_NL; ++li) {
    const int cin = kSpec[li].cin, cout = kSpec[li].cout;
    const int64_t tot = (int64_t)27 * cin * cout / 4;
    UN_LAUNCH((k_un_pack<<<blocks_for(tot, 256), 256, 0, st>>>(U->params + U->woff[li], cin, cout,
                                                               0, U->wf[li])));
    UN_LAUNCH((k_un_pack<<<blocks_for(tot, 256), 256, 0, st>>>(U->params + U->woff[li], cin, cout,
                                                               1, U->wb[li])));
  }
}

void conv_fwd(UNetCtx* U, int li, const bf16* in, bf16* out, cudaStream_t st) {
  const LayerSpec& s = kSpec[li];
  launch_conv(in, s.cin, U->lv[s.level], U->wf[li], U->params + U->boff[li], out, s.cout, nullptr,
              1, st);
}
// adjoint of layer li applied to gy (cout channels), result cin channels,
// times (mask > 0) when mask is given
void conv_adj(UNetCtx* U, int li, const bf16* gy, bf16* gx, const bf16* mask, cudaStream_t st) {
  const LayerSpec& s = kSpec[li];
  launch_conv(gy, s.cout, U->lv[s.level], U->wb[li], nullptr, gx, s.cin, mask, 0, st);
}
void pool(UNetCtx* U, const bf16* f, int lf, int C, bf16* d, cudaStream_t st) {
  const Dims &fd = U->lv[lf], &cd = U->lv[lf + 1];
  UN_LAUNCH((k_un_pool<<<blocks_for(cd.n * (C / 2), 256), 256, 0, st>>>(f, fd, cd, C, d)));
}
void pool_bwd(UNetCtx* U, const bf16* gd, int lf, int C, bf16* gf, const bf16* mask,
              cudaStream_t st) {
  const Dims &fd = U->lv[lf], &cd = U->lv[lf + 1];
  UN_LAUNCH((k_un_pool_bwd<<<blocks_for(fd.n * (C / 2), 256), 256, 0, st>>>(gd, cd, gf, mask, fd,
                                                                            C)));
}
void upcat(UNetCtx* U, const bf16* a, int Ca, const bf16* s, int lf, int Cs, bf16* c,
           cudaStream_t st) {
  const Dims &fd = U->lv[lf], &cd = U->lv[lf + 1];
  UN_LAUNCH((k_un_upcat<<<blocks_for(fd.n * ((Ca + Cs) / 8), 256), 256, 0, st>>>(a, cd, Ca, s, fd,
                                                                                Cs, c)));
}
void upcat_bwd(UNetCtx* U, const bf16* gc, int lf, int Ca, int Cs, bf16* ga, bf16* gs,
               cudaStream_t st) {
  const Dims &fd = U->lv[lf], &cd = U->lv[lf + 1];
  UN_LAUNCH((k_un_upcat_bwd_a<<<blocks_for(cd.n * (Ca / 2), 256), 256, 0, st>>>(gc, fd, Ca + Cs,
                                                                                ga, cd, Ca)));
  UN_LAUNCH((k_un_upcat_bwd_s<<<blocks_for(fd.n * (Cs / 8), 256), 256, 0, st>>>(gc, Ca + Cs, Ca,
                                                                                fd.n, gs)));
}

void forward(UNetCtx* U, cudaStream_t st) {
  conv_fwd(U, 0, U->x0, U->e0, st);
  conv_fwd(U, 1, U->e0, U->e0b, st);
  pool(U, U->e0b, 0, 16, U->d1, st);
  conv_fwd(U, 2, U->d1, U->e1, st);
  conv_fwd(U, 3, U->e1, U->e1b, st);
  pool(U, U->e1b, 1, 32, U->d2, st);
  conv_fwd(U, 4, U->d2, U->e2, st);
  conv_fwd(U, 5, U->e2, U->e2b, st);
  pool(U, U->e2b, 2, 48, U->d3, st);
  conv_fwd(U, 6, U->d3, U->e3, st);
  conv_fwd(U, 7, U->e3, U->e3b, st);
  upcat(U, U->e3b, 64, U->e2b, 2, 48, U->c2, st);
  conv_fwd(U, 8, U->c2, U->u2, st);
  upcat(U, U->u2, 48, U->e1b, 1, 32, U->c1, st);
  conv_fwd(U, 9, U->c1, U->u1, st);
  upcat(U, U->u1, 32, U->e0b, 0, 16, U->c0, st);
  conv_fwd(U, 10, U->c0, U->u0, st);
}

// gradients of sum(dz * z) into U->grads (dz in U->dz)
void backward(UNetCtx* U, cudaStream_t st) {
  const int64_t n0 = U->lv[0].n;
  UN_LAUNCH((k_un_head_bwd<<<RB, 256, 0, st>>>(n0, U->u0, U->dz, U->params + U->hw, U->g_u0,
                                               U->hpart)));
  UN_LAUNCH((k_un_reduce<<<1, 64, 0, st>>>(U->hpart, RB, 17, U->grads + U->hw)));
  // decoder
  launch_wgrad(U, 10, U->c0, U->g_u0, st);
  conv_adj(U, 10, U->g_u0, U->g_c0, U->c0, st);
  upcat_bwd(U, U->g_c0, 0, 32, 16, U->g_u1, U->g_e0b, st);
  launch_wgrad(U, 9, U->c1, U->g_u1, st);
  conv_adj(U, 9, U->g_u1, U->g_c1, U->c1, st);
  upcat_bwd(U, U->g_c1, 1, 48, 32, U->g_u2, U->g_e1b, st);
  launch_wgrad(U, 8, U->c2, U->g_u2, st);
  conv_adj(U, 8, U->g_u2, U->g_c2, U->c2, st);
  upcat_bwd(U, U->g_c2, 2, 64, 48, U->g_e3b, U->g_e2b, st);
  // encoder, coarsest first
  launch_wgrad(U, 7, U->e3, U->g_e3b, st);
  conv_adj(U, 7, U->g_e3b, U->g_e3, U->e3, st);
  launch_wgrad(U, 6, U->d3, U->g_e3, st);
  conv_adj(U, 6, U->g_e3, U->g_d3, nullptr, st);
  pool_bwd(U, U->g_d3, 2, 48, U->g_e2b, U->e2b, st);
  launch_wgrad(U, 5, U->e2, U->g_e2b, st);
  conv_adj(U, 5, U->g_e2b, U->g_e2, U->e2, st);
  launch_wgrad(U, 4, U->d2, U->g_e2, st);
  conv_adj(U, 4, U->g_e2, U->g_d2, nullptr, st);
  pool_bwd(U, U->g_d2, 1, 32, U->g_e1b, U->e1b, st);
  launch_wgrad(U, 3, U->e1, U->g_e1b, st);
  conv_adj(U, 3, U->g_e1b, U->g_e1, U->e1, st);
  launch_wgrad(U, 2, U->d1, U->g_e1, st);
  conv_adj(U, 2, U->g_e1, U->g_d1, nullptr, st);
  pool_bwd(U, U->g_d1, 0, 16, U->g_e0b, U->e0b, st);
  launch_wgrad(U, 1, U->e0, U->g_e0b, st);
  conv_adj(U, 1, U->g_e0b, U->g_e0, U->e0, st);
  launch_wgrad(U, 0, U->x0, U->g_e0, st);
}

}  // namespace

int64_t unet_nparams() {
  int64_t n = 0;
  for (int li = 0; li < UN_NL; ++li) n += (int64_t)27 * kSpec[li].cin * kSpec[li].cout + kSpec[li].cout;
  return n + UN_HEAD + 1;
}

void unet_destroy(void* h) {
  UNetCtx* U = (UNetCtx*)h;
  if (!U) return;
  for (void* p : U->owned) cudaFree(p);
  if (U->h_loss) cudaFreeHost(U->h_loss);
  delete U;
}

// The instantiated kernels: forward and adjoint convolutions for NT (output
// channels / 8) in {2, 4, 6, 8, 10, 14}, weight gradients for cout / 8 in
// {2, 4, 6, 8}; the layer table must stay within them (checked at creation,
// so the launch switches never meet another value).
static bool conv_nt_ok(int nt) {
  return nt == 2 || nt == 4 || nt == 6 || nt == 8 || nt == 10 || nt == 14;
}

int unet_create(int nz, int ny, int nx, void** out) {
  *out = nullptr;
  if (nz < 1 || ny < 1 || nx < 1) return FS_EARG;
  for (int li = 0; li < UN_NL; ++li) {
    const LayerSpec& s = kSpec[li];
    if (s.cin % 16 || s.cout % 16 || !conv_nt_ok(s.cout / 8) || !conv_nt_ok(s.cin / 8) ||
        s.cout / 8 > 8)
      return FS_EARG;
  }
  UNetCtx* U = new UNetCtx();
  int z = nz, y = ny, x = nx;
  for (int l = 0; l < 4; ++l) {
    U->lv[l] = Dims{z, y, x, (int64_t)z * y * x};
    z = (z + 1) / 2; y = (y + 1) / 2; x = (x + 1) / 2;
  }
  int64_t off = 0, wmax = 0;
  for (int li = 0; li < UN_NL; ++li) {
    const LayerSpec& s = kSpec[li];
    U->woff[li] = off;
    off += (int64_t)27 * s.cin * s.cout;
    U->boff[li] = off;
    off += s.cout;
    const int64_t n = U->lv[s.level].n;
    int64_t ch = (n + 511) / 512;
    ch = ((ch + WG_STAGE - 1) / WG_STAGE) * WG_STAGE;
    if (ch < 4 * WG_STAGE) ch = 4 * WG_STAGE;
    U->wchunk[li] = ch;
    U->nchunks[li] = (int)((n + ch - 1) / ch);
    wmax = std::max(wmax, (int64_t)U->nchunks[li] * 27 * s.cin * s.cout);
  }
  U->hw = off;
  U->hb = off + UN_HEAD;
  U->nparams = off + UN_HEAD + 1;
  const int64_t np = U->nparams;
  U->params = un_alloc<float>(U, np);
  U->grads = un_alloc<float>(U, np);
  U->am = un_alloc<float>(U, np);
  U->av = un_alloc<float>(U, np);
  for (int li = 0; li < UN_NL; ++li) {
    const int64_t c = (int64_t)27 * kSpec[li].cin * kSpec[li].cout / 4;
    U->wf[li] = un_alloc<uint2>(U, c);
    U->wb[li] = un_alloc<uint2>(U, c);
  }
  const int64_t n0 = U->lv[0].n, n1 = U->lv[1].n, n2 = U->lv[2].n, n3 = U->lv[3].n;
  U->x0 = un_alloc<bf16>(U, n0 * 16); U->e0 = un_alloc<bf16>(U, n0 * 16);
  U->e0b = un_alloc<bf16>(U, n0 * 16); U->d1 = un_alloc<bf16>(U, n1 * 16);
  U->e1 = un_alloc<bf16>(U, n1 * 32); U->e1b = un_alloc<bf16>(U, n1 * 32);
  U->d2 = un_alloc<bf16>(U, n2 * 32); U->e2 = un_alloc<bf16>(U, n2 * 48);
  U->e2b = un_alloc<bf16>(U, n2 * 48); U->d3 = un_alloc<bf16>(U, n3 * 48);
  U->e3 = un_alloc<bf16>(U, n3 * 64); U->e3b = un_alloc<bf16>(U, n3 * 64);
  U->c2 = un_alloc<bf16>(U, n2 * 112); U->u2 = un_alloc<bf16>(U, n2 * 48);
  U->c1 = un_alloc<bf16>(U, n1 * 80); U->u1 = un_alloc<bf16>(U, n1 * 32);
  U->c0 = un_alloc<bf16>(U, n0 * 48); U->u0 = un_alloc<bf16>(U, n0 * 16);
  U->g_u0 = un_alloc<bf16>(U, n0 * 16); U->g_c0 = un_alloc<bf16>(U, n0 * 48);
  U->g_u1 = un_alloc<bf16>(U, n1 * 32); U->g_e0b = un_alloc<bf16>(U, n0 * 16);
  U->g_c1 = un_alloc<bf16>(U, n1 * 80); U->g_u2 = un_alloc<bf16>(U, n2 * 48);
  U->g_e1b = un_alloc<bf16>(U, n1 * 32); U->g_c2 = un_alloc<bf16>(U, n2 * 112);
  U->g_e3b = un_alloc<bf16>(U, n3 * 64); U->g_e2b = un_alloc<bf16>(U, n2 * 48);
  U->g_e3 = un_alloc<bf16>(U, n3 * 64); U->g_d3 = un_alloc<bf16>(U, n3 * 48);
  U->g_e2 = un_alloc<bf16>(U, n2 * 48); U->g_d2 = un_alloc<bf16>(U, n2 * 32);
  U->g_e1 = un_alloc<bf16>(U, n1 * 32); U->g_d1 = un_alloc<bf16>(U, n1 * 16);
  U->g_e0 = un_alloc<bf16>(U, n0 * 16);
  U->zf = un_alloc<float>(U, n0);
  U->dz = un_alloc<float>(U, n0);
  U->wpart = un_alloc<float>(U, wmax);
  U->bpart = un_alloc<float>(U, (int64_t)RB * 64);
  U->hpart = un_alloc<float>(U, (int64_t)RB * 17);
  U->dpart = un_alloc<double>(U, RB);
  U->scale = un_alloc<double>(U, 1);
  U->loss_d = un_alloc<double>(U, 1);
  if (cudaMallocHost(&U->h_loss, sizeof(double)) != cudaSuccess) U->h_loss = nullptr;
  if (U->failed || !U->h_loss) {
    cudaGetLastError();
    unet_destroy(U);
    return FS_ECUDA;
  }
  {
    // cleared before any later work is queued, on a private stream
    SetupStream ss;
    cudaMemsetAsync(U->params, 0, sizeof(float) * np, ss.s);
    cudaMemsetAsync(U->am, 0, sizeof(float) * np, ss.s);
    cudaMemsetAsync(U->av, 0, sizeof(float) * np, ss.s);
    ss.sync();
  }
  *out = U;
  return cuda_status();
}

int unet_set_params(void* h, const float* host, int64_t n, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  if (n != U->nparams) return FS_EARG;
  cudaMemcpyAsync(U->params, host, sizeof(float) * n, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(U->am, 0, sizeof(float) * n, st);
  cudaMemsetAsync(U->av, 0, sizeof(float) * n, st);
  U->step = 0;
  launch_pack(U, st);
  if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
  return cuda_status();
}

int unet_get(void* h, int which, float* host, int64_t n, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  if (n != U->nparams) return FS_EARG;
  cudaMemcpyAsync(host, which ? U->grads : U->params, sizeof(float) * n, cudaMemcpyDeviceToHost,
                  st);
  if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
  return cuda_status();
}

// z = N(r / rms(r)) (double in and out; the preconditioner of flexible CG)
int unet_apply(void* h, const double* r, double* z, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  const int64_t n0 = U->lv[0].n;
  UN_LAUNCH((k_un_sumsq<double><<<RB, 256, 0, st>>>(n0, r, U->dpart)));
  UN_LAUNCH((k_un_scale<<<1, 32, 0, st>>>(U->dpart, RB, n0, U->scale)));
  UN_LAUNCH((k_un_input<double><<<blocks_for(n0, 256), 256, 0, st>>>(n0, r, U->scale, U->x0)));
  forward(U, st);
  UN_LAUNCH((k_un_head<<<blocks_for(n0, 256), 256, 0, st>>>(n0, U->u0, U->params + U->hw,
                                                            U->params + U->hb, nullptr, z)));
  return cuda_status();
}

// out = base + N(r / rms(r)) * rms(r) * out_scale  (fp32; the coarse
// correction of the learned preconditioner; base may be NULL)
int unet_correct(void* h, const float* r, const float* base, float* out, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  const int64_t n0 = U->lv[0].n;
  UN_LAUNCH((k_un_sumsq<float><<<RB, 256, 0, st>>>(n0, r, U->dpart)));
  UN_LAUNCH((k_un_scale<<<1, 32, 0, st>>>(U->dpart, RB, n0, U->scale)));
  UN_LAUNCH((k_un_input<float><<<blocks_for(n0, 256), 256, 0, st>>>(n0, r, U->scale, U->x0)));
  forward(U, st);
  UN_LAUNCH((k_un_head<<<blocks_for(n0, 256), 256, 0, st>>>(n0, U->u0, U->params + U->hw,
                                                            U->params + U->hb, U->zf, nullptr)));
  UN_LAUNCH((k_un_correct<<<blocks_for(n0, 256), 256, 0, st>>>(n0, U->zf, U->scale, U->out_scale,
                                                               base, out)));
  return cuda_status();
}

int unet_set_output_scale(void* h, float s) {
  UNetCtx* U = (UNetCtx*)h;
  if (!(s >= 0.f) || !std::isfinite(s)) return FS_EARG;
  U->out_scale = s;
  return FS_OK;
}

int64_t unet_cells(void* h) { return ((UNetCtx*)h)->lv[0].n; }

// z = N(r) for an already normalised fp32 input (training data, tests)
int unet_forward_f32(void* h, const float* r, float* z, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  const int64_t n0 = U->lv[0].n;
  UN_LAUNCH((k_un_input<float><<<blocks_for(n0, 256), 256, 0, st>>>(n0, r, nullptr, U->x0)));
  forward(U, st);
  UN_LAUNCH((k_un_head<<<blocks_for(n0, 256), 256, 0, st>>>(n0, U->u0, U->params + U->hw,
                                                            U->params + U->hb, z, nullptr)));
  return cuda_status();
}

// loss = mean (N(r) - tau)^2 and its gradient in the context (no update)
int unet_grad(void* h, const float* r, const float* tau, double* loss, cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  const int64_t n0 = U->lv[0].n;
  int rc = unet_forward_f32(h, r, U->zf, st);
  if (rc) return rc;
  UN_LAUNCH((k_un_loss<<<RB, 256, 0, st>>>(n0, U->zf, tau, U->dz, U->dpart)));
  UN_LAUNCH((k_un_dsum<<<1, 32, 0, st>>>(U->dpart, RB, U->loss_d)));
  backward(U, st);
  cudaMemcpyAsync(U->h_loss, U->loss_d, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (fs_stream_wait(st) != FS_OK) return FS_ECUDA;
  if (loss) *loss = *U->h_loss / (double)n0;
  return cuda_status();
}

// one Adam step on (r, tau); loss before the step
int unet_train_step(void* h, const float* r, const float* tau, float lr, double* loss,
                    cudaStream_t st) {
  UNetCtx* U = (UNetCtx*)h;
  int rc = unet_grad(h, r, tau, loss, st);
  if (rc) return rc;
  if (!(*loss == *loss)) return FS_ENONFINITE;
  U->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - powf(b1, (float)U->step), bc2 = 1.f - powf(b2, (float)U->step);
  UN_LAUNCH((k_un_adam<<<blocks_for(U->nparams, 256), 256, 0, st>>>(
      U->nparams, U->params, U->grads, U->am, U->av, lr, b1, b2, 1e-8f, bc1, bc2)));
  launch_pack(U, st);
  return cuda_status();
}
