// bc_block.cuh — the middle of a three-level product in one persistent kernel.
//
// A three-level transform of M = L1 x L2 x Lr points keeps, after the outer
// pass, L1 independent blocks per operand: block k1 is the L2 x Lr points
// bufA + k1*S1 (S1 = L2*Lr), 2 MB of complex doubles for L2 = 128, Lr = 1024.
// Three passes remain per block, and the separate kernels for them move
// each block through HBM twice more:
//   F  column DFTs of length L2 over the block's Lr columns (A and B), then
//      the twiddle e^{-2 pi i col k2/(L2 Lr)};
//   R  per row: forward DFTs of A's and B's rows (Lr = 1024), product,
//      inverse DFT (A's row is overwritten);
//   I  conjugate twiddle, inverse column DFTs (A only).
// Here one kernel does all three as WORK ITEMS handed to warps: a column
// tile of L2 rows x W columns (one warp, 32 points per lane) is an F or I
// item, a row pair an R item.  Items sit in one global order made of steps;
// step j holds the F items of block j, the R items of block j - LAG_R and
// the I items of block j - LAG_I.  Warp w of the grid takes items w, w + NW,
// w + 2 NW, ... (static), so only a few blocks are in flight at any time
// (LAG_I + 1 of them, 36 MB at L2 = 128): their intermediate values stay in
// L2 between the passes, and B's dead rows are dropped from L2 unwritten.
//
// Measured on B200 (2^24 x 2^24 limbs, M = 2^25): 1.32 ms for the fused
// kernel against 1.08 ms for the three separate passes, with a third of the
// DRAM traffic.  Six warps per SM (two CTAs of three, 255 registers, the
// row pass's 112 KB of shared memory) issue too little FP64 work to hide the
// latencies that the separate column passes hide with sixteen, so the
// separate passes stay the default; this kernel runs with $BC_FUSED=1.
//
// Dependencies: an R item of block b waits until all F items of b have
// finished (fdone[b] counts them), an I item until all R items have
// (rdone[b]).  Every dependency points to an item earlier in the global
// order, each warp takes its items in increasing order, and the launch is
// cooperative (every CTA resident), so the earliest unfinished item always
// belongs to a warp that is working on it: the kernel cannot deadlock.
// Every wait is bounded; a wait that gives up flags the item, the warp lets
// its copies in flight land and stops (the others then give up too).
//
// Each warp owns two 16 KB buffers.  A column tile takes one (W/8 TMA boxes
// of 8 complex columns x L2 rows, unswizzled); a row pair takes both (B's
// row, then A's, 16 KB bulk copies).  The next item's copies are
// issued into whichever buffer frees up first, as soon as its dependency is
// met, so they land while the current item computes.
#pragma once
#include "bc_pipe.cuh"
#include "bc_rows_warp.cuh"

namespace bc {

constexpr int BLK_LAG_R = 4;  // steps between a block's F items and its R items
constexpr int BLK_LAG_I = 8;  // ... and its I items
constexpr int BLK_SPINS = 1 << 22;
// dynamic shared memory: the row pass's (twiddle table, two 16 KB buffers
// per warp) and 128 bytes to align the buffers for TMA
constexpr size_t BLK_SMEM = RW_SMEM + 128;

template <int L2> struct BlkCfg {
  static_assert(L2 == 64 || L2 == 128, "fused middle: L2 = 64 or 128");
  static constexpr int T = L2 / 32;  // lanes per column of a column tile
  static constexpr int W = 32 / T;   // columns per tile (W * L2 = 1024 points, 16 KB)
  static constexpr int J = 32 / T;   // second-stage DFTs per lane
  static constexpr unsigned TILE_BYTES = (unsigned)L2 * W * 16;
};

// L2-point DFTs of the W columns of a tile held by one warp.  Lane
// (t = lane / W, c = lane % W) holds rows t + T i (i < 32) of column c on
// entry and frequencies t + T i on exit.  The split is L2 = 32 x T: a
// 32-point DFT in registers over i, the twiddle e^{-+2 pi i t k/L2}
// (= twT[k*32 + (1024/L2) t], the row pass's table), one exchange through
// the tile buffer (entry (row, c) at tix<L2>(row, c): boxes of 8 columns,
// row-major; the 8 lanes of a quarter-warp touch 8 consecutive columns of
// one row, 128 contiguous bytes), and T-point DFTs over t.
// Tile layout (what an unswizzled TMA box of 8 complex columns x L2 rows
// writes, box after box): entry (row, c) of a W-column tile.
template <int L2>
__device__ __forceinline__ int tix(int row, int c) {
  return (c >> 3) * (L2 * 8) + row * 8 + (c & 7);
}

template <int L2, bool INV>
__device__ __forceinline__ void col_dft_warp(double2 (&v)[RW_P], int t, int c, double2 *buf, const double2 *twT) {
  using C = BlkCfg<L2>;
  constexpr int T = C::T, J = C::J, LS = 1024 / L2;
  dft32<INV>(v);  // v[k] = Y[t][k]
#pragma unroll
  for (int k = 1; k < RW_P; k++) v[k] = ctw<INV>(v[k], twT[k * 32 + LS * t]);
#pragma unroll
  for (int k = 0; k < RW_P; k++) buf[tix<L2>(k * T + t, c)] = v[k];
  __syncwarp();
#pragma unroll
  for (int j = 0; j < J; j++) {
    const int k = t + T * j;
    double2 x[T];
#pragma unroll
    for (int tp = 0; tp < T; tp++) x[tp] = buf[tix<L2>(k * T + tp, c)];
    if constexpr (T == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
    else dft2<INV>(x[0], x[1]);
#pragma unroll
    for (int k1 = 0; k1 < T; k1++) v[j + J * k1] = x[k1];  // frequency k + 32 k1 = t + T (j + J k1)
  }
  __syncwarp();  // the buffer is free
}

// e^{-2 pi i col k2/(L2 Lr)} for k2 = t + T i (i < 32): four runs of 8 from
// the 4M-point table (index 4 L1 col k2), bases b[r] for i = 8r and the step
// e^{-2 pi i col T/(L2 Lr)}; point i takes b[i/8] * st^(i%8).
struct ColTw {
  double2 b[4], st;
};
template <int L2>
__device__ __forceinline__ ColTw col_tw(const ClassParams &p, int col, int t) {
  constexpr int T = BlkCfg<L2>::T;
  const uint64_t f = (uint64_t)4 * (uint64_t)p.L1 * (uint64_t)col;
  ColTw w;
  w.st = tw2_get(p.tw4M, f * T);
#pragma unroll
  for (int r = 0; r < 4; r++) w.b[r] = tw2_get(p.tw4M, f * (uint64_t)(t + 8 * T * r));
  return w;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// One work item of the fused kernel.
struct BlkItem {
  unsigned q;       // global index (>= total: none)
  int kind;         // 0: F, 1: R, 2: I
  unsigned blk;     // block: item blk / L1, k1 = blk % L1
  int op;           // F: operand 0 (A) or 1 (B)
  int idx;          // F/I: column tile; R: row
};

template <int L2, bool SQ>
__global__ void __launch_bounds__(32 * RW_WARPS, 2)
    k4_mid_fused(ClassParams p, const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB) {
  using C = BlkCfg<L2>;
  constexpr int T = C::T, W = C::W, NOPS = SQ ? 1 : 2, PER = NOPS + 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t bars[RW_WARPS][2];
  double2 *const twT = reinterpret_cast<double2 *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
  for (int i = threadIdx.x; i < RW_L; i += blockDim.x) {
    const int m = (i >> 5) * (i & 31);
    const double2 w = __ldg(&p.twLr[m < 768 ? m : m - 512]);
    twT[i] = m < 768 ? w : make_double2(-w.x, -w.y);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = lane / W, c = lane % W;
  double2 *const bufs = twT + RW_L * (1 + 2 * wid);  // buffer h at bufs + h*RW_L
  uint64_t *const bar = bars[wid];
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  const unsigned Lr = (unsigned)p.Lr, S1 = (unsigned)p.S1, L1 = (unsigned)p.L1;
  const unsigned nblk = (unsigned)p.nitems * L1;
  const unsigned per_step = (unsigned)L2 * PER;
  const unsigned total = (nblk + BLK_LAG_I) * per_step;  // far below 2^32
  // warps taking items: all of them, or all but the last CTA's when the
  // grid's warp count is a multiple of the step length (a warp would then
  // meet the same kind of item in every step)
  const unsigned per_step0 = (unsigned)L2 * PER;
  const unsigned NW = (gridDim.x - (gridDim.x > 1 && (gridDim.x * RW_WARPS) % per_step0 == 0 ? 1 : 0)) * RW_WARPS;
  unsigned *const fdone = p.blkdone, *const rdone = p.blkdone + nblk;
  const unsigned nF = (unsigned)NOPS * (Lr / W);  // F items per block
  const FastDiv fd_step(per_step), fd_per((unsigned)PER), fd_L1(L1);

  // the first valid item at or after q in this warp's sequence (q, q+NW, ...)
  auto item_at = [&](unsigned q) -> BlkItem {
    BlkItem it;
    for (; q < total; q += NW) {
      // a step is laid out in kind blocks: NOPS*L2 F items (operand-major),
      // L2 R items, L2 I items.  The grid's warp count is not a multiple of
      // the step length, so a warp's position in successive steps drifts
      // over all kinds and every warp gets the same mix of work.
      const unsigned step = fd_step.div(q), r = q - step * per_step;
      it.q = q;
      if (r < nF) {
        if (step >= nblk) continue;
        it.kind = 0; it.blk = step; it.op = r >= (unsigned)L2; it.idx = (int)(r - (it.op ? L2 : 0));
      } else if (r < nF + L2) {
        if (step < BLK_LAG_R || step - BLK_LAG_R >= nblk) continue;
        it.kind = 1; it.blk = step - BLK_LAG_R; it.op = 0; it.idx = (int)(r - nF);
      } else {
        if (step < BLK_LAG_I || step - BLK_LAG_I >= nblk) continue;
        it.kind = 2; it.blk = step - BLK_LAG_I; it.op = 0; it.idx = (int)(r - nF - L2);
      }
      return it;
    }
    it.q = total; it.kind = -1; it.blk = 0; it.op = 0; it.idx = 0;
    return it;
  };
  // block base of an item's operand (from the class's slabs: no descriptor loads)
  auto block_base = [&](const BlkItem &it, int op) -> double2 * {
    const unsigned item = fd_L1.div(it.blk), k1 = it.blk - item * L1;
    return (op ? p.slabB : p.slabA) + (size_t)item * p.slab_elems + (size_t)k1 * S1;
  };
  auto item_flags = [&](const BlkItem &it) -> unsigned * { return p.items[fd_L1.div(it.blk)].flags; };
  // dependency met?  Every lane reads the counter with acquire semantics
  // (each lane then issues copies of data other SMs wrote); the warp agrees.
  auto dep_ready = [&](const BlkItem &it) -> bool {
    bool ok = true;
    if (it.kind == 1) ok = ld_acquire_u32(&fdone[it.blk]) >= nF;
    else if (it.kind == 2) ok = ld_acquire_u32(&rdone[it.blk]) >= (unsigned)L2;
    return __all_sync(0xffffffffu, ok);
  };
  auto dep_wait = [&](const BlkItem &it) -> bool {
    for (int i = 0; i < BLK_SPINS; i++) {
      if (dep_ready(it)) return true;
      __nanosleep(128);
    }
    return false;
  };

  // ---- copies
  unsigned phb = 0u;   // bit h: parity to wait for on buffer h
  unsigned infl = 0u;  // bit h: a copy in flight into buffer h
  // column tile of item `it` into buffer h: W/8 TMA boxes of 8 columns x L2 rows
  auto load_tile = [&](const BlkItem &it, int h) {
    if (lane == 0) {
      const unsigned item = fd_L1.div(it.blk), k1 = it.blk - item * L1;
      fence_proxy_async_smem();
      fence_proxy_async_global();  // the data may come from other SMs' stores (acquired above)
      mbar_expect_tx(&bar[h], C::TILE_BYTES);
#pragma unroll
      for (int gi = 0; gi < W / 8; gi++)
        tma_load_4d(bufs + h * RW_L + gi * L2 * 8, (it.kind == 0 && it.op) ? &mB : &mA, &bar[h],
                    2 * (it.idx * W + 8 * gi), 0, (int)k1, (int)item);
    }
    infl |= 1u << h;
  };
  auto load_row = [&](const BlkItem &it, int op, int h) {
    if (lane == 0) {
      fence_proxy_async_smem();
      fence_proxy_async_global();
      mbar_expect_tx(&bar[h], RW_ROW_BYTES);
      bulk_load(bufs + h * RW_L, block_base(it, op) + (size_t)it.idx * Lr, RW_ROW_BYTES, &bar[h]);
    }
    infl |= 1u << h;
  };
  // pending copies of an item: F/I one (the tile), R two (B then A; A only
  // when squaring); `buf` records where each went
  struct Plan {
    int need, issued;
    int h0, h1;  // buffers of the first and second copy
  };
  auto plan_of = [&](const BlkItem &it) -> Plan {
    Plan pl;
    pl.need = (it.kind == 1 && !SQ) ? 2 : (it.q < total ? 1 : 0);
    pl.issued = 0;
    pl.h0 = pl.h1 = 0;
    return pl;
  };
  // issue the next pending copy of `it` into free buffer h if its
  // dependency allows (or unconditionally after waiting)
  auto issue_one = [&](const BlkItem &it, Plan &pl, int h) {
    if (it.kind == 1) {
      const int op = SQ ? 0 : (pl.issued == 0 ? 1 : 0);  // B's row first
      load_row(it, op, h);
    } else {
      load_tile(it, h);
    }
    if (pl.issued == 0) pl.h0 = h;
    else pl.h1 = h;
    pl.issued++;
  };
  auto try_issue = [&](const BlkItem &it, Plan &pl, int h) {
    if (pl.issued < pl.need && dep_ready(it)) issue_one(it, pl, h);
  };
  bool failed = false;
  unsigned bad_q = 0;
  // wait for the copy in buffer h
  auto take = [&](int h) -> bool {
    const bool ok = mbar_wait(&bar[h], (phb >> h) & 1u);
    if (__any_sync(0xffffffffu, !ok)) return false;
    phb ^= 1u << h;
    infl &= ~(1u << h);
    return true;
  };
  // completion of an item's stores: the warp's stores are ordered before
  // lane 0's release increment (__syncwarp orders the lanes), so a consumer
  // that acquires the count sees them (and fences its async proxy before
  // copying them)
  // The increment is held back until the warp is about to store again or to
  // wait (flush): by then the stores it covers have long completed and the
  // release costs little.  It is never held across a wait, so no warp waits
  // on a count another waiting warp holds back.
  unsigned *held = nullptr;
  auto signal = [&](unsigned *ctr) { held = ctr; };
  auto flush = [&]() {
    if (held) {
      __syncwarp();
      if (lane == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(held) : "memory");
      held = nullptr;
    }
  };

  BlkItem cur = item_at(blockIdx.x * RW_WARPS + wid < NW ? blockIdx.x * RW_WARPS + wid : total);
  Plan pc = plan_of(cur);
  if (cur.q < total) {
    if (!dep_wait(cur)) { failed = true; bad_q = cur.q; }  // (nothing held yet)
    while (!failed && pc.issued < pc.need) issue_one(cur, pc, pc.issued);
  }
  while (!failed && cur.q < total) {
    const BlkItem nxt = item_at(cur.q + NW);
    Plan pn = plan_of(nxt);
    double2 v[RW_P];
    if (cur.kind == 0 || cur.kind == 2) {
      // ---------------- column tile (F: forward + twiddle; I: twiddle + inverse)
      const int h = pc.h0, other = h ^ 1;
      try_issue(nxt, pn, other);
      const int col = cur.idx * W + c;
      double2 *const g = block_base(cur, cur.kind == 0 ? cur.op : 0) + col;
      const double2 *bf = bufs + h * RW_L;
      if (cur.kind == 0) {
        if (!take(h)) { failed = true; bad_q = cur.q; break; }
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = bf[tix<L2>(t + T * i, c)];
        __syncwarp();
        col_dft_warp<L2, false>(v, t, c, bufs + h * RW_L, twT);
        try_issue(nxt, pn, h);
        const ColTw tw = col_tw<L2>(p, col, t);
        flush();
#pragma unroll
        for (int r = 0; r < 4; r++) {
          double2 w = tw.b[r];
#pragma unroll
          for (int i = 8 * r; i < 8 * r + 8; i++) {
            g[(size_t)(t + T * i) * Lr] = cmul(v[i], w);
            w = cmul(w, tw.st);
          }
        }
        signal(&fdone[cur.blk]);
      } else {
        const ColTw tw = col_tw<L2>(p, col, t);  // global loads before the wait
        if (!take(h)) { failed = true; bad_q = cur.q; break; }
#pragma unroll
        for (int r = 0; r < 4; r++) {
          double2 w = tw.b[r];
#pragma unroll
          for (int i = 8 * r; i < 8 * r + 8; i++) {
            v[i] = cmulc(bf[tix<L2>(t + T * i, c)], w);
            w = cmul(w, tw.st);
          }
        }
        __syncwarp();
        col_dft_warp<L2, true>(v, t, c, bufs + h * RW_L, twT);
        try_issue(nxt, pn, h);
        flush();
#pragma unroll
        for (int i = 0; i < RW_P; i++) g[(size_t)(t + T * i) * Lr] = v[i];
      }
    } else {
      // ---------------- row pair (as k2_rows_w1024)
      double2 *const ra = block_base(cur, 0) + (size_t)cur.idx * Lr;
      if (SQ) {
        const int ha = pc.h0;
        try_issue(nxt, pn, ha ^ 1);
        if (!take(ha)) { failed = true; bad_q = cur.q; break; }
        double2 *const bf = bufs + ha * RW_L;
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = bf[lane + 32 * i];
        __syncwarp();
        row_dft1024<false>(v, lane, bf, twT);
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = cmul(v[i], v[i]);
        row_dft1024<true>(v, lane, bf, twT);
        try_issue(nxt, pn, ha);
      } else {
        const int hb = pc.h0, ha = pc.h1;
        if (!take(hb)) { failed = true; bad_q = cur.q; break; }
        double2 *const bB = bufs + hb * RW_L, *const bA = bufs + ha * RW_L;
        {
          // B's row has reached shared memory and nothing reads it again: drop
          // its L2 lines without a write-back (128 lines of 128 bytes)
          const char *rb = reinterpret_cast<const char *>(block_base(cur, 1) + (size_t)cur.idx * Lr);
#pragma unroll
          for (int k = 0; k < 4; k++)
            asm volatile("discard.global.L2 [%0], 128;" ::"l"(rb + 128 * (lane + 32 * k)) : "memory");
        }
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = bB[lane + 32 * i];
        __syncwarp();
        row_dft1024<false>(v, lane, bB, twT);
#pragma unroll
        for (int i = 0; i < RW_P; i++) bB[lane + 32 * i] = v[i];  // B's spectrum, read back by this lane only
        if (!take(ha)) { failed = true; bad_q = cur.q; break; }
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = bA[lane + 32 * i];
        __syncwarp();
        row_dft1024<false>(v, lane, bA, twT);
#pragma unroll
        for (int i = 0; i < RW_P; i++) v[i] = cmul(v[i], bB[lane + 32 * i]);
        __syncwarp();
        try_issue(nxt, pn, hb);
        row_dft1024<true>(v, lane, bA, twT);
        try_issue(nxt, pn, ha);
      }
      flush();
#pragma unroll
      for (int i = 0; i < RW_P; i++) ra[lane + 32 * i] = v[i];
      signal(&rdone[cur.blk]);
    }
    // the rest of the next item's copies: wait for its dependency now
    if (nxt.q < total && pn.issued < pn.need) {
      flush();
      if (!dep_wait(nxt)) { failed = true; bad_q = nxt.q; break; }
      while (pn.issued < pn.need) {
        const int h = (pn.issued == 1) ? (pn.h0 ^ 1) : (int)(infl & 1u);
        issue_one(nxt, pn, h);
      }
    }
    cur = nxt;
    pc = pn;
  }
  flush();
  if (failed) {
    // flag the item, let this warp's copies in flight land, stop
    if (lane == 0) {
      atomicOr(item_flags(item_at(bad_q)), FLAG_TIMEOUT);
      if (infl & 1u) mbar_drain(&bar[0], phb & 1u);
      if (infl & 2u) mbar_drain(&bar[1], (phb >> 1) & 1u);
    }
    __syncwarp();
  }
}

}  // namespace bc
