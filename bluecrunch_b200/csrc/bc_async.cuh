// bc_async.cuh — asynchronous staging for the pass kernels on sm_100a:
// TMA tensor loads (cp.async.bulk.tensor) completing on shared-memory
// mbarriers, per-thread cp.async copies, and the 128-byte-swizzled tile
// layout the TMA writes.
//
// No load here uses cluster multicast: every CTA fetches its own tiles.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace bc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// ------------------------------------------------------------------ mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of a barrier.  Returns false if it gave up
// (the caller flags the item and skips the tile; nothing waits forever).
constexpr int MBAR_SPINS = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  for (int i = 0; i < MBAR_SPINS; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}
// After some wait of the CTA gave up: wait once more, longer (about 2^24
// polls, seconds), for a copy still in flight on `bar` to land, so that no
// bulk copy writes into the shared memory of a CTA that has exited.  The
// kernel then stops issuing copies and returns; the item is already flagged.
constexpr int MBAR_DRAIN_SPINS = 1 << 24;
__device__ __forceinline__ void mbar_drain(uint64_t *bar, unsigned parity) {
  for (int i = 0; i < MBAR_DRAIN_SPINS; i++) {
    if (mbar_try_wait(bar, parity)) return;
    __nanosleep(256);
  }
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// ------------------------------------------------------------------ TMA loads
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
// Untiled bulk copy of `bytes` contiguous bytes (both addresses 16-byte
// aligned, bytes a multiple of 16) completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

// ------------------------------------------------------------------ cp.async
// 4-byte asynchronous copy; src_bytes = 0 writes a zero word (no read).
__device__ __forceinline__ void cp_async4(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
// 16-byte asynchronous copy (both addresses 16-byte aligned); bytes past
// src_bytes are zero-filled (src_bytes = 0 reads nothing).
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// ------------------------------------------------------------------ programmatic dependent launch
// A pass launched with programmatic stream serialisation may start while the
// previous pass of its stream is still finishing: its CTAs set up shared
// memory from read-only tables, then pdl_wait() blocks until the previous
// grid has completed and its writes are visible (a no-op for a normal
// launch).  Every global access to data another pass reads or writes comes
// after it.  pdl_trigger() lets the next pass of the stream be launched.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------ layout
// A tile of L rows x W complex columns lives as W/8 boxes of L rows x 8
// columns (128 bytes per row); inside a box the 16-byte chunk of column c in
// row r sits at chunk c ^ (r & 7).  This is exactly what a TMA load with
// 128-byte swizzle writes for a box of 16 doubles x L rows placed at a
// 1024-byte-aligned address, and it keeps any 8 lanes touching 8 columns of
// one row, or one column of 8 consecutive rows, on distinct banks.
template <int L>
__device__ __forceinline__ int bidx(int row, int s) {
  return (s >> 3) * (L * 8) + row * 8 + ((s & 7) ^ (row & 7));
}
// A row of L complex points as one box of L/8 lines of 8.
__device__ __forceinline__ int ridx(int e) { return (e & ~7) + ((e & 7) ^ ((e >> 3) & 7)); }

}  // namespace bc
