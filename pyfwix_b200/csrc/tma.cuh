// Tensor-memory-accelerator (TMA) staging of column tiles for the column passes.
//
// A column pass works on a tile of LX consecutive columns x N rows of one slice.
// With TMA one thread moves the whole tile between HBM and shared memory with
// one or a few cp.async.bulk.tensor instructions (a 3-D tensor map over
// [slices][NY][NX] of 8-byte complex samples), instead of every thread issuing
// one 8-byte copy per sample.  Tiles are row-major in shared memory with the
// 128-byte swizzle (LX = 16 columns = 128 bytes per row): the 16-byte chunk c
// of row y sits at chunk c ^ (y & 7), so the lanes of a line, which read one
// column at rows t, t + 1, ..., touch eight different chunks and the warp's
// request takes the minimum two wavefronts.
//
// Loads complete on an mbarrier (transaction bytes); every wait is bounded.
// TMA loads here never use cluster multicast, and every tensor map covers
// this GPU's own buffers only.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fwix {
namespace tma {

// Tries of a bounded mbarrier wait (each try_wait itself waits a bounded,
// hardware-chosen time): far beyond any copy of a tile, short of a hang.
constexpr unsigned kWaitTries = 1u << 24;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity to complete; false when the
// tries ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  for (unsigned i = 0; i < kWaitTries; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3-D tiled load global -> shared, completing on bar.  x must be a multiple of
// two samples (16 bytes); here it is always a multiple of 16.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// 3-D tiled store shared -> global (bulk group of the issuing thread).
__device__ __forceinline__ void store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void store_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// Waits until the committed stores have read their shared-memory sources.
__device__ __forceinline__ void store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }

// Index (in samples) of sample (y, c) of a row-major tile of 16 columns with
// the 128-byte swizzle: 16-byte chunk c / 2 of row y moves to chunk
// (c / 2) ^ (y & 7).  The tile must start on a 1024-byte boundary.
__device__ __forceinline__ int sw128(int y, int c) { return y * 16 + ((((c >> 1) ^ (y & 7)) << 1) | (c & 1)); }
// The same for a tile of 8 columns (64-byte rows) with the 64-byte swizzle: 16-byte
// chunk c / 2 of row y moves to chunk (c / 2) ^ ((y >> 1) & 3).  The tile must start
// on a 512-byte boundary.
__device__ __forceinline__ int sw64(int y, int c) { return y * 8 + ((((c >> 1) ^ ((y >> 1) & 3)) << 1) | (c & 1)); }
// Tile index of sample (y, c) for LX-column tiles (16: sw128, 8: sw64).
template <int LX>
__device__ __forceinline__ int swz_tile(int y, int c) {
  static_assert(LX == 16 || LX == 8, "TMA column tiles are 8 or 16 columns wide");
  return LX == 16 ? sw128(y, c) : sw64(y, c);
}

}  // namespace tma

// Host side: a 3-D tensor map over 8-byte samples [nz][ny][nx] at base (row
// pitch nx samples, plane pitch ny * nx), box {box_cols, box_rows, 1} with the
// 128-byte swizzle for 16 columns, the 64-byte swizzle for 8.  Maps are cached per (base, sizes, box).  Returns the CUDA error of
// the driver call (cudaErrorInvalidValue when the driver entry point is missing
// or the encoding is refused).
cudaError_t tile_map(CUtensorMap* out, const void* base, int nx, int ny, long long nz, int box_rows, int box_cols = 16);

// Host side: a 3-D tensor map over the quarter-spectrum phase table of one depth,
// [nslices][pnx][pny] 8-byte factors (ky fastest, pny even so that rows are 16-byte
// multiples), box {pny, box_cols, 1} (every ky of box_cols consecutive kx of one
// (reference, frequency) slice), no swizzle.  Cached like tile_map.
cudaError_t qtab_map(CUtensorMap* out, const void* base, int pny, int pnx, long long nslices, int box_cols);

}  // namespace fwix
