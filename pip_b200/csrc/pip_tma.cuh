// pip_tma.cuh -- tile staging by the tensor memory accelerator (TMA) for the stage kernels.
//
// A state array of NV planes of ix*jx cells (x fastest) is described to the TMA as a 3D
// tensor (x, y, plane).  A stage kernel's halo tile of all planes -- RX x RY cells x NV
// planes -- arrives with one cp.async.bulk.tensor load per CTA into shared memory in the
// kernel's own layout (plane, row, column), completing on an mbarrier.  Cells outside the
// array read as zero.  No multicast: each CTA loads its own tile.
//
// Alignment: the TMA needs the tile's first x coordinate times the element size to be a
// multiple of 16 bytes, the row and plane strides to be multiples of 16 bytes, the base
// address 16-byte aligned and the shared-memory destination 128-byte aligned.  The host
// builds a map only where every tile meets these rules (tma_tile_ok) and the kernels fall
// back to per-thread loads otherwise.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pip {

// Polls of the tile's mbarrier before a CTA gives up (then flags the stage as failed).
constexpr int kTmaWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t tma_smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tma_bar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tma_smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_bar_expect(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               ::"r"(tma_smem_addr(bar)), "r"(bytes)
               : "memory");
}

// One 3D tile (x0, y0, plane 0) of the map into dst; completes on bar.
__device__ __forceinline__ void tma_load_tile(void *dst, const CUtensorMap *map, int x0, int y0,
                                              unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(tma_smem_addr(dst)), "l"((unsigned long long)map), "r"(x0), "r"(y0), "r"(0),
        "r"(tma_smem_addr(bar))
      : "memory");
}

// Bounded wait on phase 0 of bar: false when `limit` polls ran out.
__device__ __forceinline__ bool tma_bar_wait(unsigned long long *bar, int limit) {
  const uint32_t a = tma_smem_addr(bar);
  for (int k = 0; k < limit; ++k) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Host: whether every tile of a grid of tiles whose first x coordinate is x_first + k*tx
// (k = 0, 1, ...) can be staged from an array of nv planes of ix*jx elements of esize bytes
// at base, with a box of rx x ry x nv elements.
inline bool tma_tile_ok(const void *base, int ix, int jx, int nv, int esize, int x_first, int tx,
                        int rx, int ry) {
  const long long nc = (long long)ix * jx;
  if (((uintptr_t)base & 15u) != 0) return false;
  if (((long long)ix * esize) % 16 != 0 || (nc * esize) % 16 != 0) return false;
  if ((x_first * esize) % 16 != 0 || (tx * esize) % 16 != 0) return false;
  if ((rx * esize) % 16 != 0) return false;
  if (rx > 256 || ry > 256 || nv > 256) return false;
  return true;
}

// Host: encodes the 3D map of such an array (FP32 or FP64 elements) with a box of
// rx x ry x nv; false if the driver entry point or the encoding is unavailable.
bool tma_encode(CUtensorMap *map, const void *base, int ix, int jx, int nv, int esize, int rx,
                int ry);

}  // namespace pip
