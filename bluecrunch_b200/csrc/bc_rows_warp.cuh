// bc_rows_warp.cuh — the row pass for 1024-point rows, one warp per row.
//
// Same arithmetic contract as k2_rows<1024> (bc_pipe.cuh): every row r of
// the class gets A_r <- IDFT(DFT(A_r) . DFT(B_r)) (or the square), with the
// forward transform on e^{-2 pi i nk/1024}, the inverse on the conjugate
// roots, both unscaled.  The organisation is different: a lane holds 32
// points of its row in registers (point l + 32 i in v[i] of lane l), so a
// 1024-point transform is two 32-point DFTs in registers around one twiddle
// multiply and ONE transpose through shared memory (the four-step split
// 1024 = 32 x 32), where the 8-points-per-thread block transform needs three
// exchanges and barriers across the row's threads.  Everything a warp does
// is warp-private (__syncwarp only): its rows arrive as 16 KB bulk copies
// into its two row buffers, each buffer serves as the transpose buffer of
// the operand it delivered, and B's spectrum is parked in B's buffer while A
// is transformed.
#pragma once
#include "bc_kernels.cuh"

namespace bc {

constexpr int RW_WARPS = 3;     // rows in flight per CTA (two CTAs per SM)
constexpr int RW_L = 1024;      // row length
constexpr int RW_P = 32;        // points per lane
constexpr unsigned RW_ROW_BYTES = RW_L * 16;
// dynamic shared memory: the twiddle table (32 x 32 entries), then two
// 1024-entry row buffers per warp
constexpr size_t RW_SMEM = (size_t)(RW_L + 2 * RW_WARPS * RW_L) * 16;

// cos and sin of 2 pi j/32, correctly rounded (j < 32).
__device__ __forceinline__ constexpr double cos32(int j) {
  switch (j & 31) {
    case 0: return 1.0;
    case 1: return 0.9807852804032304;
    case 2: return 0.9238795325112867;
    case 3: return 0.8314696123025452;
    case 4: return 0.7071067811865476;
    case 5: return 0.5555702330196022;
    case 6: return 0.3826834323650898;
    case 7: return 0.19509032201612828;
    case 8: return 0.0;
    case 9: return -0.19509032201612828;
    case 10: return -0.3826834323650898;
    case 11: return -0.5555702330196022;
    case 12: return -0.7071067811865476;
    case 13: return -0.8314696123025452;
    case 14: return -0.9238795325112867;
    case 15: return -0.9807852804032304;
    case 16: return -1.0;
    case 17: return -0.9807852804032304;
    case 18: return -0.9238795325112867;
    case 19: return -0.8314696123025452;
    case 20: return -0.7071067811865476;
    case 21: return -0.5555702330196022;
    case 22: return -0.3826834323650898;
    case 23: return -0.19509032201612828;
    case 24: return 0.0;
    case 25: return 0.19509032201612828;
    case 26: return 0.3826834323650898;
    case 27: return 0.5555702330196022;
    case 28: return 0.7071067811865476;
    case 29: return 0.8314696123025452;
    case 30: return 0.9238795325112867;
    default: return 0.9807852804032304;
  }
}
__device__ __forceinline__ constexpr double sin32(int j) { return cos32(j - 8); }

// x * e^{-2 pi i j/32} (forward) or x * e^{+2 pi i j/32} (inverse), j a
// compile-time constant after unrolling.
template <bool INV>
__device__ __forceinline__ double2 rot32(double2 x, int j) {
  if ((j & 31) == 0) return x;
  if ((j & 31) == 8) return cmul_mi<INV>(x);
  if ((j & 31) == 16) return make_double2(-x.x, -x.y);
  if ((j & 31) == 24) return cmul_mi<!INV>(x);
  return ctw<INV>(x, make_double2(cos32(j), -sin32(j)));
}

// 32-point DFT of a[0..31] in registers, natural order in and out, as
// 32 = 8 x 4: n = n1 + 8 n2, k = 4 k1 + k2; DFT-4 over n2, twiddle
// w32^(n1 k2), DFT-8 over n1.
template <bool INV>
__device__ __forceinline__ void dft32(double2 (&a)[RW_P]) {
#pragma unroll
  for (int n1 = 0; n1 < 8; n1++) {
    dft4<INV>(a[n1], a[n1 + 8], a[n1 + 16], a[n1 + 24]);  // a[n1 + 8 k2] = y[n1][k2]
#pragma unroll
    for (int k2 = 1; k2 < 4; k2++) a[n1 + 8 * k2] = rot32<INV>(a[n1 + 8 * k2], n1 * k2);
  }
  double2 o[RW_P];
#pragma unroll
  for (int k2 = 0; k2 < 4; k2++) {
    double2 b[8];
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) b[n1] = a[n1 + 8 * k2];
    dft8<INV>(b);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) o[4 * k1 + k2] = b[k1];
  }
#pragma unroll
  for (int k = 0; k < RW_P; k++) a[k] = o[k];
}

// 1024-point DFT of one row held by a warp: v[i] of lane l is point
// l + 32 i on entry and frequency l + 32 i on exit.  n = n1 + 32 n2 with
// n1 = lane; k = 32 k1 + k2.  twT[k2*32 + l] = e^{-2 pi i l k2/1024}; buf is
// the warp's 1024-entry transpose buffer (16-byte entries, row k2 of the
// transpose XOR-swizzled by k2 & 7 so both the row writes and the column
// reads of 8 consecutive lanes hit distinct banks).
template <bool INV>
__device__ __forceinline__ void row_dft1024(double2 (&v)[RW_P], int lane, double2 *buf, const double2 *twT) {
  dft32<INV>(v);  // over n2: v[k2] = y[n1 = lane][k2]
#pragma unroll
  for (int k2 = 1; k2 < RW_P; k2++) v[k2] = ctw<INV>(v[k2], twT[k2 * 32 + lane]);
#pragma unroll
  for (int k2 = 0; k2 < RW_P; k2++) buf[k2 * 32 + (lane ^ (k2 & 7))] = v[k2];
  __syncwarp();
#pragma unroll
  for (int n1 = 0; n1 < RW_P; n1++) v[n1] = buf[lane * 32 + (n1 ^ (lane & 7))];
  __syncwarp();  // the buffer is free for the next transform
  dft32<INV>(v);  // over n1: v[k1] = X[32 k1 + lane]
}

// Grid: persistent, RW_WARPS warps per CTA; warp w of CTA c takes rows
// c*RW_WARPS + w + k*gridDim.x*RW_WARPS of the class (items' rows are
// contiguous: row q of item i is bufA + q*1024).  Without squaring a warp
// keeps B's next row landing in buffer 1 during the inverse transform and
// A's next row in buffer 0 during B's forward transform; squaring alternates
// its rows between the two buffers.  The tensor maps of the generic row
// kernel's signature are not used.
template <bool SQ>
__global__ void __launch_bounds__(32 * RW_WARPS, 2)
    k2_rows_w1024(ClassParams p, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t bars[RW_WARPS][2];
  double2 *const twT = reinterpret_cast<double2 *>(smraw);
  // twT[k2*32 + l] = e^{-2 pi i m/1024}, m = l*k2 <= 961; the flat table
  // holds m < 768, and e^{-2 pi i m/1024} = -e^{-2 pi i (m-512)/1024}
  for (int i = threadIdx.x; i < RW_L; i += blockDim.x) {
    const int m = (i >> 5) * (i & 31);
    const double2 w = __ldg(&p.twLr[m < 768 ? m : m - 512]);
    twT[i] = m < 768 ? w : make_double2(-w.x, -w.y);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double2 *const buf0 = twT + RW_L * (1 + 2 * wid), *const buf1 = buf0 + RW_L;
  uint64_t *const bar0 = &bars[wid][0], *const bar1 = &bars[wid][1];
  if (lane == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  const unsigned rows_item = p.M / RW_L;
  const unsigned total = (unsigned)p.nitems * rows_item;  // rows of the class, far below 2^32
  const FastDiv fd_rows(rows_item);
  const unsigned stride = gridDim.x * RW_WARPS;
  auto row_base = [&](unsigned row, bool opB) -> double2 * {
    const unsigned item = fd_rows.div(row);
    const ItemDesc &it = p.items[item];
    return (opB ? it.bufB : it.bufA) + (size_t)(row - item * rows_item) * RW_L;
  };
  // all lanes are done with the buffer (the caller's __syncwarp); lane 0
  // hands it to the async proxy and starts the copy
  auto fetch = [&](double2 *dst, uint64_t *bar, unsigned row, bool opB) {
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_expect_tx(bar, RW_ROW_BYTES);
      bulk_load(dst, row_base(row, opB), RW_ROW_BYTES, bar);
    }
  };
  unsigned ph0 = 0, ph1 = 0;  // parity to wait for on bar0 / bar1
  // wait for a row's copy, then move it to registers.  The wait is bounded;
  // false when it gave up on any lane of the warp (the loop then stops).
  auto take = [&](double2 (&v)[RW_P], const double2 *src, uint64_t *bar, unsigned &ph) -> bool {
    const bool ok = mbar_wait(bar, ph);
    if (__any_sync(0xffffffffu, !ok)) return false;
    ph ^= 1u;
#pragma unroll
    for (int i = 0; i < RW_P; i++) v[i] = src[lane + 32 * i];
    __syncwarp();  // the buffer is read: free for the transpose
    return true;
  };
  // after a wait gave up: bit 0 / bit 1 = a copy still in flight on bar0 /
  // bar1, and the row whose item gets flagged
  unsigned drain = 0, bad_row = 0;
  unsigned r = blockIdx.x * RW_WARPS + wid;
  if (SQ) {
    if (r < total) fetch(buf0, bar0, r, false);
    if (r + stride < total) fetch(buf1, bar1, r + stride, false);
    for (int k = 0; r < total; r += stride, k ^= 1) {
      double2 *const bf = k ? buf1 : buf0;
      uint64_t *const bar = k ? bar1 : bar0;
      double2 va[RW_P];
      if (!take(va, bf, bar, k ? ph1 : ph0)) {
        drain = (k ? 2u : 1u) | (r + stride < total ? (k ? 1u : 2u) : 0u);
        bad_row = r;
        break;
      }
      row_dft1024<false>(va, lane, bf, twT);
#pragma unroll
      for (int i = 0; i < RW_P; i++) va[i] = cmul(va[i], va[i]);
      row_dft1024<true>(va, lane, bf, twT);
      if (r + 2 * stride < total) fetch(bf, bar, r + 2 * stride, false);
      double2 *const ra = row_base(r, false);
#pragma unroll
      for (int i = 0; i < RW_P; i++) ra[lane + 32 * i] = va[i];
    }
  } else {
    if (r < total) {
      fetch(buf1, bar1, r, true);
      fetch(buf0, bar0, r, false);
    }
    for (; r < total; r += stride) {
      const bool more = r + stride < total;
      double2 v[RW_P];
      // B: forward transform, spectrum parked in buffer 1 (natural order)
      if (!take(v, buf1, bar1, ph1)) {
        drain = 3u;  // A's row r is in flight too
        bad_row = r;
        break;
      }
      row_dft1024<false>(v, lane, buf1, twT);
#pragma unroll
      for (int i = 0; i < RW_P; i++) buf1[lane + 32 * i] = v[i];
      // A: forward transform, product with B's spectrum (each lane reads
      // back only the entries it wrote)
      if (!take(v, buf0, bar0, ph0)) {
        drain = 1u;  // B's next row is not issued yet
        bad_row = r;
        break;
      }
      row_dft1024<false>(v, lane, buf0, twT);
#pragma unroll
      for (int i = 0; i < RW_P; i++) v[i] = cmul(v[i], buf1[lane + 32 * i]);
      __syncwarp();
      if (more) fetch(buf1, bar1, r + stride, true);
      row_dft1024<true>(v, lane, buf0, twT);
      if (more) fetch(buf0, bar0, r + stride, false);
      double2 *const ra = row_base(r, false);
#pragma unroll
      for (int i = 0; i < RW_P; i++) ra[lane + 32 * i] = v[i];
    }
  }
  if (drain) {
    // flag the row's item, let the warp's copies still in flight land, stop
    if (lane == 0) {
      atomicOr(p.items[fd_rows.div(bad_row)].flags, FLAG_TIMEOUT);
      if (drain & 1u) mbar_drain(bar0, ph0);
      if (drain & 2u) mbar_drain(bar1, ph1);
    }
    __syncwarp();
  }
}

}  // namespace bc
