// Tensor-memory-accelerator (TMA) staging of 3-D field tiles into shared
// memory for the stencil kernels, and the mbarrier waits that go with it.
//
// A field is the C-order (nz, ny, nx) float64 array every kernel uses; its
// tensor map describes it as a 3-D tensor (x fastest) and a box of
// bx x by x 1 elements.  One cp.async.bulk.tensor load moves one box (a
// z-plane of a tile with its x and y halo) into a 128-byte aligned shared
// slot and signals an mbarrier with the bytes it delivered.  Coordinates
// outside the tensor read zeros; the box's x origin must be even (16 bytes
// of doubles), and the row and plane strides multiples of 16 bytes, so the
// maps are only made for even nx.  Waits on the mbarrier are bounded: on
// expiry the kernel records the failure in a device flag and carries on.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

// bounded mbarrier wait: about this many try_wait rounds (each may suspend
// the thread for a while) before the kernel gives up
#define TMA_WAIT_LIMIT (1 << 22)

__device__ __forceinline__ uint32_t tma_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tma_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_addr(bar)), "r"(count)
               : "memory");
}

// the barrier initialisation visible to the async proxy (TMA completions)
__device__ __forceinline__ void tma_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// one z-plane box of a 3-D tensor at (x, y, z) into shared memory
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tma_smem_addr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(tma_smem_addr(bar))
      : "memory");
}

// order this thread's generic shared-memory accesses before later
// async-proxy (TMA) writes to the same memory
__device__ __forceinline__ void tma_fence_proxy() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool tma_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(tma_smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for a phase of the barrier; false (and *err set) when it gave up
__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (int it = 0; it < TMA_WAIT_LIMIT; ++it)
    if (tma_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, 1);
  return false;
}

// Host: a tensor map over a C-order (nz, ny, nx) double field with a box of
// bx x by x 1; false when the driver entry point is missing, the layout does
// not meet TMA's alignment rules, or encoding fails.
bool tma_map_field(CUtensorMap* map, const double* base, int nx, int ny, int nz, int bx, int by);
// whether the stencil kernels use TMA staging (fs_set_tma; default on)
bool tma_enabled();
