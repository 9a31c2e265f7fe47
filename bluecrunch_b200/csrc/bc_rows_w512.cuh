// bc_rows_w512.cuh — the row pass for 512-point rows, one warp per row.
//
// Same arithmetic contract as k2_rows<512> (bc_pipe.cuh): every row r of the
// class gets A_r <- IDFT(DFT(A_r) . DFT(B_r)) (or the square), forward on
// e^{-2 pi i nk/512}, inverse on the conjugate roots, both unscaled.  As in
// k2_rows_w1024 a lane holds its row's points in registers, point l + 32 i in
// v[i] of lane l, here 16 of them, and everything a warp does is
// warp-private (__syncwarp only; the block kernel synchronises the two warps
// of a row at named barriers around each of its two exchanges).
//
// The transform, with n = l + 32 i (l = lane) and k = k1 + 16 k2:
//   1. DFT-16 over i in registers: Y[l][k1];
//   2. twiddle e^{-2 pi i l k1/512};
//   3. the remaining DFT-32 over l, split l = l1 + 16 l0 and
//      k2 = 2 k2' + e: lanes l1 and l1 + 16 swap their 16 values by shuffle
//      and form B_e = A_l1 + (-1)^e A_(l1+16) (e = the lane's half), then the
//      upper half multiplies by e^{-2 pi i l1/32};
//   4. one transpose inside each half-warp through shared memory, so that
//      lane L = k1 + 16 e holds B_e(l1, k1) for l1 = 0..15;
//   5. DFT-16 over l1 in registers: v[k2'] = X[k1 + 16 (2 k2' + e)] =
//      X[L + 32 k2'].
// The spectrum lands in the layout the points came in, so A and B meet lane
// by lane, and the same steps on conjugate roots give the inverse.
#pragma once
#include "bc_pass16.cuh"

namespace bc {

constexpr int R5_WARPS = 4;  // rows in flight per CTA (two CTAs per SM)
constexpr int R5_L = 512;    // row length
constexpr int R5_P = 16;     // points per lane
constexpr unsigned R5_ROW_BYTES = R5_L * 16;
// dynamic shared memory: the twiddle table (16 x 32 entries), then two
// 512-entry row buffers per warp
constexpr size_t R5_SMEM = (size_t)(R5_L + 2 * R5_WARPS * R5_L) * 16;

// 512-point DFT of one row held by a warp (the steps above).  twT[k1*32 + l]
// = e^{-2 pi i l k1/512}; buf is the warp's 512-entry transpose buffer
// (entry j of lane l's block at l*16 + (j ^ (l & 15)), so the writes of one
// j and the reads of one l1 by 8 consecutive lanes hit distinct banks).
template <bool INV>
__device__ __forceinline__ void row_dft512(double2 (&v)[R5_P], int lane, double2 *buf, const double2 *twT) {
  dft16<INV>(v);  // over i: v[k1] = Y[lane][k1]
#pragma unroll
  for (int k1 = 1; k1 < R5_P; k1++) v[k1] = ctw<INV>(v[k1], twT[k1 * 32 + lane]);
  const bool upper = lane >= 16;
  const double2 w = twT[(lane & 15) * 32 + 16];  // e^{-2 pi i 16 l1/512} = e^{-2 pi i l1/32}
#pragma unroll
  for (int k1 = 0; k1 < R5_P; k1++) {
    const double2 o = make_double2(__shfl_xor_sync(0xffffffffu, v[k1].x, 16), __shfl_xor_sync(0xffffffffu, v[k1].y, 16));
    const double2 b = upper ? make_double2(o.x - v[k1].x, o.y - v[k1].y) : make_double2(v[k1].x + o.x, v[k1].y + o.y);
    v[k1] = upper ? ctw<INV>(b, w) : b;
  }
#pragma unroll
  for (int k1 = 0; k1 < R5_P; k1++) buf[lane * 16 + (k1 ^ (lane & 15))] = v[k1];
  __syncwarp();
  const int k1 = lane & 15, h = lane & 16;
#pragma unroll
  for (int l1 = 0; l1 < R5_P; l1++) v[l1] = buf[(l1 + h) * 16 + (k1 ^ l1)];
  __syncwarp();  // the buffer is free for the next transform
  dft16<INV>(v);  // over l1: v[k2'] = X[lane + 32 k2']
}

// Occupancy: the kernel holds about 250 registers per thread (a row's 16
// points, the DFT-16 temporaries and the twiddles it loads ahead), so two
// CTAs of four warps share an SM; three CTAs (170 registers) spill and
// measured slower.
// Grid: persistent, R5_WARPS warps per CTA; warp w of CTA c takes rows
// c*R5_WARPS + w + k*gridDim.x*R5_WARPS of the class (row q of item i is
// bufA + q*512).  Buffers, copies and waits as in k2_rows_w1024: without
// squaring, B's spectrum is parked in buffer 1 and B's next row lands there
// during the inverse transform, A's next row in buffer 0 likewise; squaring
// alternates its rows between the two buffers.  The tensor maps of the
// generic row kernel's signature are not used.
template <bool SQ>
__global__ void __launch_bounds__(32 * R5_WARPS, 2)
    k2_rows_w512(ClassParams p, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t bars[R5_WARPS][2];
  double2 *const twT = reinterpret_cast<double2 *>(smraw);
  // twT[k1*32 + l] = e^{-2 pi i m/512}, m = l*k1 <= 465; the flat table holds
  // m < 384, and e^{-2 pi i m/512} = -e^{-2 pi i (m-256)/512}
  for (int i = threadIdx.x; i < R5_L; i += blockDim.x) {
    const int m = (i >> 5) * (i & 31);
    const double2 w = __ldg(&p.twLr[m < 384 ? m : m - 256]);
    twT[i] = m < 384 ? w : make_double2(-w.x, -w.y);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double2 *const buf0 = twT + R5_L * (1 + 2 * wid), *const buf1 = buf0 + R5_L;
  uint64_t *const bar0 = &bars[wid][0], *const bar1 = &bars[wid][1];
  if (lane == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  const unsigned rows_item = p.M / R5_L;
  const unsigned total = (unsigned)p.nitems * rows_item;  // rows of the class, far below 2^32
  const FastDiv fd_rows(rows_item);
  const unsigned stride = gridDim.x * R5_WARPS;
  // row q of item i; B's rows sit in the item's B slot
  auto row_base = [&](unsigned row, bool opB) -> double2 * {
    const unsigned item = fd_rows.div(row);
    const ItemDesc &it = p.items[item];
    return (opB ? it.bufB : it.bufA) + (size_t)(row - item * rows_item) * R5_L;
  };
  // all lanes are done with the buffer (the caller's __syncwarp); lane 0
  // hands it to the async proxy and starts the copy
  auto fetch = [&](double2 *dst, uint64_t *bar, unsigned row, bool opB) {
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_expect_tx(bar, R5_ROW_BYTES);
      bulk_load(dst, row_base(row, opB), R5_ROW_BYTES, bar);
    }
  };
  unsigned ph0 = 0, ph1 = 0;  // parity to wait for on bar0 / bar1
  // wait for a row's copy, then move it to registers; false when the bounded
  // wait gave up on any lane of the warp (the loop then stops)
  auto take = [&](double2 (&v)[R5_P], const double2 *src, uint64_t *bar, unsigned &ph) -> bool {
    const bool ok = mbar_wait(bar, ph);
    if (__any_sync(0xffffffffu, !ok)) return false;
    ph ^= 1u;
#pragma unroll
    for (int i = 0; i < R5_P; i++) v[i] = src[lane + 32 * i];
    __syncwarp();  // the buffer is read: free for the transpose
    return true;
  };
  // after a wait gave up: bit 0 / bit 1 = a copy still in flight on bar0 /
  // bar1, and the row whose item gets flagged
  unsigned drain = 0, bad_row = 0;
  unsigned r = blockIdx.x * R5_WARPS + wid;
  if (SQ) {
    if (r < total) fetch(buf0, bar0, r, false);
    if (r + stride < total) fetch(buf1, bar1, r + stride, false);
    for (int k = 0; r < total; r += stride, k ^= 1) {
      double2 *const bf = k ? buf1 : buf0;
      uint64_t *const bar = k ? bar1 : bar0;
      double2 va[R5_P];
      if (!take(va, bf, bar, k ? ph1 : ph0)) {
        drain = (k ? 2u : 1u) | (r + stride < total ? (k ? 1u : 2u) : 0u);
        bad_row = r;
        break;
      }
      row_dft512<false>(va, lane, bf, twT);
#pragma unroll
      for (int i = 0; i < R5_P; i++) va[i] = cmul(va[i], va[i]);
      row_dft512<true>(va, lane, bf, twT);
      if (r + 2 * stride < total) fetch(bf, bar, r + 2 * stride, false);
      double2 *const ra = row_base(r, false);
#pragma unroll
      for (int i = 0; i < R5_P; i++) ra[lane + 32 * i] = va[i];
    }
  } else {
    if (r < total) {
      fetch(buf1, bar1, r, true);
      fetch(buf0, bar0, r, false);
    }
    for (; r < total; r += stride) {
      const bool more = r + stride < total;
      double2 v[R5_P];
      // B: forward transform, spectrum parked in buffer 1 (natural order)
      if (!take(v, buf1, bar1, ph1)) {
        drain = 3u;  // A's row r is in flight too
        bad_row = r;
        break;
      }
      row_dft512<false>(v, lane, buf1, twT);
#pragma unroll
      for (int i = 0; i < R5_P; i++) buf1[lane + 32 * i] = v[i];
      // A: forward transform, product with B's spectrum (each lane reads
      // back only the entries it wrote)
      if (!take(v, buf0, bar0, ph0)) {
        drain = 1u;  // B's next row is not issued yet
        bad_row = r;
        break;
      }
      row_dft512<false>(v, lane, buf0, twT);
#pragma unroll
      for (int i = 0; i < R5_P; i++) v[i] = cmul(v[i], buf1[lane + 32 * i]);
      __syncwarp();
      if (more) fetch(buf1, bar1, r + stride, true);
      row_dft512<true>(v, lane, buf0, twT);
      if (more) fetch(buf0, bar0, r + stride, false);
      double2 *const ra = row_base(r, false);
#pragma unroll
      for (int i = 0; i < R5_P; i++) ra[lane + 32 * i] = v[i];
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
