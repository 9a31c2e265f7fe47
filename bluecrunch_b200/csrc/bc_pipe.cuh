// bc_pipe.cuh — persistent, double-buffered pass kernels.
//
// Same arithmetic as the passes in bc_kernels.cuh, restructured so that HBM
// traffic overlaps the FP64 work: every CTA walks work units of its class in
// a persistent loop and stages the next unit while it transforms the current
// one.  Complex tiles arrive by TMA (cp.async.bulk.tensor, 128-byte swizzle,
// completion on an mbarrier); the packing pass stages the limb words it needs
// with cp.async.  Results leave by plain coalesced stores from registers.
//
// All items of a class sit in contiguous slabs (item i's buffer at i*M), so
// one tensor map per slab serves the whole class.
#pragma once
#include <type_traits>

#include "bc_async.cuh"
#include "bc_kernels.cuh"

namespace bc {

// Points per unit of the column passes and of the row pass.
#ifndef BC_PASS_POINTS
#define BC_PASS_POINTS 1024
#endif
#ifndef BC_ROW_POINTS
#define BC_ROW_POINTS 1024
#endif

// Tile width (columns) of an L-row pass tile: BC_PASS_POINTS points, at
// least 8 columns (one 128-byte swizzle atom).
__host__ __device__ constexpr int pass_tile_w(int L) {
  return (BC_PASS_POINTS / L) >= 8 ? BC_PASS_POINTS / L : 8;
}

template <int L> struct PassTile {
  static constexpr int W = pass_tile_w(L);
  static constexpr int NT = (L / PTS) * W;
  static constexpr int BOX_ROWS = L > 256 ? 256 : L;
  static constexpr int HALVES = L / BOX_ROWS;
  static constexpr unsigned BYTES = (unsigned)L * W * 16;
  // resident CTAs per SM with at most 128 registers per thread
  static constexpr int MINB = NT >= 512 ? 1 : 512 / NT;
  static constexpr int TWN = tw_entries<L>();     // L-point stage twiddles kept in shared memory
  // dynamic shared memory of k2_mid / k2_outer_inv: two tiles, the stage
  // twiddles, the outer pass's weights (outer_inv only), 1024 bytes of slack
  // for aligning the tiles
  static constexpr size_t SMEM_MID = 2 * (size_t)BYTES + (size_t)TWN * 16 + 2 * (size_t)(L / PTS + 1) * 16 + 1024;
  static constexpr size_t SMEM_OUTER_INV = SMEM_MID + (size_t)L * 16;
};

// Copy n table entries from global to shared memory (all threads of the CTA;
// the caller's next barrier publishes them).
__device__ __forceinline__ void table_to_smem(double2 *dst, const double2 *__restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(&src[i]);
}

__device__ __forceinline__ double2 *align1024(unsigned char *p) {
  return reinterpret_cast<double2 *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Issue the TMA loads of one L x W tile (W/8 boxes, each L rows of 8
// complex; two boxes per column group when L = 512) into dst.
template <int L, int W>
__device__ __forceinline__ void tile_load_4d(double2 *dst, const CUtensorMap *map, uint64_t *bar, int col0, int c2,
                                             int c3) {
  using T = PassTile<L>;
  mbar_expect_tx(bar, (unsigned)L * W * 16);
#pragma unroll
  for (int g = 0; g < W / 8; g++)
#pragma unroll
    for (int h = 0; h < T::HALVES; h++)
      tma_load_4d(dst + g * L * 8 + h * T::BOX_ROWS * 8, map, bar, 2 * (col0 + 8 * g), h * T::BOX_ROWS, c2, c3);
}
template <int L, int W>
__device__ __forceinline__ void tile_load_3d(double2 *dst, const CUtensorMap *map, uint64_t *bar, int col0, int c2) {
  using T = PassTile<L>;
  mbar_expect_tx(bar, (unsigned)L * W * 16);
#pragma unroll
  for (int g = 0; g < W / 8; g++)
#pragma unroll
    for (int h = 0; h < T::HALVES; h++)
      tma_load_3d(dst + g * L * 8 + h * T::BOX_ROWS * 8, map, bar, 2 * (col0 + 8 * g), h * T::BOX_ROWS, c2);
}

// Twiddles of a thread's 8 points in a column pass, w^(m0 + i*dm) for
// i = 0..7: two table lookups (base and step) and a running product, instead
// of a two-level lookup per point.  `conj0` conjugates the base (the outer
// pass's k = 0 term is e^{+2 pi i s/(4M)}).
__device__ __forceinline__ void twiddle_run(const Tw2 &T, uint64_t m0, bool conj0, uint64_t dm, double2 (&w)[PTS]) {
  double2 b = tw2_get(T, m0);
  if (conj0) b.y = -b.y;
  const double2 st = tw2_get(T, dm);
  w[0] = b;
#pragma unroll
  for (int i = 1; i < PTS; i++) w[i] = cmul(w[i - 1], st);
}

// Outer pass: point (col, k1 = t + i*TC) takes e^{-2 pi i col(4 k1 - 1)/(4M)}.
template <int TC>
__device__ __forceinline__ void outer_twiddles(const Tw2 &T, int col, int t, double2 (&w)[PTS]) {
  if (t == 0) twiddle_run(T, (uint64_t)col, true, (uint64_t)col * 4 * TC, w);
  else twiddle_run(T, (uint64_t)col * (4 * t - 1), false, (uint64_t)col * 4 * TC, w);
}

// e^{-2 pi i m/(2 h)} for |m| < 2h: sincospi of m/h.  With h = 2M it is the
// outer passes' e^{-2 pi i m/(4M)}; with h = S1/2 the middle passes'
// e^{-2 pi i m/(L2 Lr)}.
__device__ __forceinline__ double2 t4m(long long m, double h) {
  double sn, cs;
  sincospi((double)m / h, &sn, &cs);
  return make_double2(cs, -sn);
}

// ------------------------------------------------------------------ middle (3 levels)
// Units: (item, operand, block k1, column tile).  Map: 4-d view of a slab,
// (2*Lr doubles, L2 rows, L1 blocks, items).
// Twiddles e^{-2 pi i col k2/(L2 Lr)} of a thread's points k2 = t + TC i,
// col = tile W + s, as a base and a step with a running product; both are
// products of a tile factor and a column factor (T(col x) = T(tile W x)
// T(s x)): the TC + 1 tile factors T(tile W t) (t < TC) and T(tile W TC) are
// computed once per unit by a few lanes of each warp (sincospi) into shared
// memory, the column factors T(s t) and T(s TC) stay in registers.  No
// global twiddle loads remain on the unit's path.
template <int TC, int W, int NT>
__device__ __forceinline__ void mid_tile_tw(double2 *fac, int tile, double h) {
  constexpr int NF = TC + 1, NW = NT / 32, PER = (NF + NW - 1) / NW;
  const int lane = threadIdx.x & 31, j = (threadIdx.x >> 5) * PER + lane;
  if (lane < PER && j < NF) fac[j] = t4m((long long)tile * W * (j < TC ? j : TC), h);
}

template <int L, bool INV>
__global__ void __launch_bounds__(PassTile<L>::NT, PassTile<L>::MINB)
    k2_mid(ClassParams p, const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB) {
  using T = PassTile<L>;
  constexpr int W = T::W, TC = L / PTS, NT = T::NT;
  extern __shared__ unsigned char smraw[];
  __shared__ uint64_t bars[2];
  double2 *const buf0 = align1024(smraw);  // stage st's tile at buf0 + st * L * W
  double2 *twS = buf0 + 2 * L * W;
  double2 *fac = twS + T::TWN;  // tile factors of unit parity st at fac + st * (TC + 1)
  table_to_smem(twS, p.twL2, T::TWN);
  const int tid = threadIdx.x, s = tid % W, t = tid / W;
  const double h = 0.5 * (double)p.S1;
  const double2 cb = t4m((long long)s * t, h), cs = t4m((long long)s * TC, h);
  // unit counts stay far below 2^32 (a class holds at most 2^33 points, 2048 per unit)
  const unsigned tiles = p.Lr / W;
  // forward: the A units of every item, then the B slab's slots (map mB's
  // last coordinate is the slot); inverse: A only
  const unsigned per_op = (unsigned)p.L1 * tiles;
  const unsigned nA = INV ? (unsigned)p.nitems * per_op : fwd_units_a(p, per_op);
  const unsigned total = nA + (INV ? 0u : fwd_units_b(p, per_op));
  const FastDiv fd_op(per_op), fd_tile(tiles);
  auto decode = [&](unsigned u, int &item, int &op, int &slot, int &blk, int &tile) {
    const FwdUnit f = fwd_unit(p, u, nA, fd_op, per_op);
    item = f.item;
    op = f.op;
    slot = f.slot;
    blk = (int)fd_tile.div(f.rest);
    tile = (int)(f.rest - (unsigned)blk * tiles);
  };
  auto issue = [&](unsigned u, int st) {
    int item, op, slot, blk, tile;
    decode(u, item, op, slot, blk, tile);
    fence_proxy_async_smem();
    tile_load_4d<L, W>(buf0 + st * L * W, op ? &mB : &mA, &bars[st], tile * W, blk, slot);
  };
  auto tile_of = [&](unsigned u) -> int {
    int item, op, slot, blk, tile;
    decode(u, item, op, slot, blk, tile);
    return tile;
  };
  // the unit's twiddles from its tile factors (fac) and the column factors
  auto twiddles = [&](const double2 *f, double2 (&w)[PTS]) {
    const double2 step = cmul(f[TC], cs);
    w[0] = cmul(f[t], cb);
#pragma unroll
    for (int i = 1; i < PTS; i++) w[i] = cmul(w[i - 1], step);
  };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  if (blockIdx.x < total) mid_tile_tw<TC, W, NT>(fac, tile_of(blockIdx.x), h);
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  unsigned phases = 0;  // bit st: parity to wait for on bars[st]
  int st = 0;
  unsigned u = blockIdx.x;
  if (tid == 0 && u < total) issue(u, 0);
  for (; u < total; u += gridDim.x) {
    const unsigned un = u + gridDim.x;
    if (tid == 0 && un < total) issue(un, st ^ 1);
    int item, op, slot, blk, tile;
    decode(u, item, op, slot, blk, tile);
    const ItemDesc &it = p.items[item];
    double2 *g = (op ? it.bufB : it.bufA) + (unsigned)blk * (unsigned)p.S1;
    const int col = tile * W + s;
    double2 v[PTS], w[PTS];
    if (INV) twiddles(fac + st * (TC + 1), w);
    const unsigned par = (phases >> st) & 1u;
    const bool ok = mbar_wait(&bars[st], par);
    phases ^= 1u << st;
    double2 *bf = buf0 + st * L * W;
#pragma unroll
    for (int i = 0; i < PTS; i++) {
      v[i] = bf[bidx<L>(t + i * TC, s)];
      if (INV) v[i] = cmulc(v[i], w[i]);
    }
    if (__syncthreads_or(!ok)) {
      // a wait gave up: flag the item, issue nothing more, let the copies in
      // flight land, leave
      if (tid == 0) {
        atomicOr(it.flags, FLAG_TIMEOUT);
        mbar_drain(&bars[st], par);
        if (un < total) mbar_drain(&bars[st ^ 1], (phases >> (st ^ 1)) & 1u);
      }
      return;
    }
    // the next unit's tile factors (its parity's slot was last read before
    // the barrier above)
    if (un < total) mid_tile_tw<TC, W, NT>(fac + (st ^ 1) * (TC + 1), tile_of(un), h);
    block_fft<L, W, INV>(v, t, s, bf, twS);
    if (!INV) twiddles(fac + st * (TC + 1), w);
#pragma unroll
    for (int i = 0; i < PTS; i++) {
      const unsigned k2 = t + i * TC;
      g[k2 * (unsigned)p.Lr + col] = INV ? v[i] : cmul(v[i], w[i]);
    }
    __syncthreads();
    st ^= 1;
  }
}

// ------------------------------------------------------------------ outer inverse
// Units: (item, column tile).  Map: 3-d view of slab A, (2*S1, L1, items).
template <int L>
__global__ void __launch_bounds__(PassTile<L>::NT, PassTile<L>::MINB) k2_outer_inv(ClassParams p, const __grid_constant__ CUtensorMap mA) {
  using T = PassTile<L>;
  constexpr int W = T::W, TC = L / PTS, G = W / 8;
  extern __shared__ unsigned char smraw[];
  __shared__ uint64_t bars[2];
  double2 *const buf0 = align1024(smraw);  // stage st's tile at buf0 + st * L * W
  double2 *twS = buf0 + 2 * L * W;
  double2 *pwS = twS + T::TWN;
  table_to_smem(twS, p.twL1, T::TWN);
  table_to_smem(pwS, p.pw_inv, L);
  const int tid = threadIdx.x, s = tid % W, t = tid / W;
  const unsigned tiles = p.S1 / W;
  const unsigned total = (unsigned)p.nitems * tiles;  // far below 2^32
  const FastDiv fd_tiles(tiles);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  unsigned phases = 0;  // bit st: parity to wait for on bars[st]
  int st = 0;
  unsigned u = blockIdx.x;
  if (tid == 0 && u < total) {
    fence_proxy_async_smem();
    const unsigned q0 = fd_tiles.div(u);
    tile_load_3d<L, W>(buf0, &mA, &bars[0], (int)(u - q0 * tiles) * W, (int)q0);
  }
  for (; u < total; u += gridDim.x) {
    const unsigned un = u + gridDim.x;
    if (tid == 0 && un < total) {
      fence_proxy_async_smem();
      const unsigned qn = fd_tiles.div(un);
      tile_load_3d<L, W>(buf0 + (st ^ 1) * L * W, &mA, &bars[st ^ 1], (int)(un - qn * tiles) * W, (int)qn);
    }
    const int item = (int)fd_tiles.div(u), tile = (int)(u - (unsigned)item * tiles);
    const ItemDesc &it = p.items[item];
    const int col = tile * W + s;
    double2 v[PTS], w[PTS];
    outer_twiddles<TC>(p.tw4M, col, t, w);  // global loads, before the wait
    const unsigned par = (phases >> st) & 1u;
    const bool ok = mbar_wait(&bars[st], par);
    phases ^= 1u << st;
    double2 *bf = buf0 + st * L * W;
#pragma unroll
    for (int i = 0; i < PTS; i++) v[i] = cmulc(bf[bidx<L>(t + i * TC, s)], w[i]);
    if (__syncthreads_or(!ok)) {  // a wait gave up: flag, drain, leave
      if (tid == 0) {
        atomicOr(it.flags, FLAG_TIMEOUT);
        mbar_drain(&bars[st], par);
        if (un < total) mbar_drain(&bars[st ^ 1], (phases >> (st ^ 1)) & 1u);
      }
      return;
    }
    block_fft<L, W, true>(v, t, s, bf, twS);
    double err = 0.0;
#pragma unroll
    for (int i = 0; i < PTS; i++) {
      const int n1 = t + i * TC;
      double2 z = cmul(v[i], pwS[n1]);
      double re = rint(z.x), im = rint(z.y);
      err = fmax(err, round_check(z, re, im));
      bf[bidx<L>(n1, s)] = make_double2(re, im);
    }
    atomic_max_err(it.err, err);
    __syncthreads();
    {
      // one 8-column group of one row per thread; consecutive lanes take
      // consecutive rows of a group (distinct banks in the swizzled layout)
      const int row = tid % L, gi = tid / L;
      double cre[8], cim[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        double2 z = bf[bidx<L>(row, 8 * gi + q)];
        cre[q] = z.x;
        cim[q] = z.y;
      }
      const unsigned n0 = (unsigned)row * (unsigned)p.S1 + (unsigned)tile * W + 8 * gi;
      store_rec(&it.rec[n0 >> 3], make_run(cre, it.b));
      store_rec(&it.rec[(n0 + p.M) >> 3], make_run(cim, it.b));
    }
    static_assert(PassTile<L>::NT == L * G, "one run pair per thread");
    __syncthreads();
    st ^= 1;
  }
}

// ------------------------------------------------------------------ rows
// Units: NR consecutive rows of the class's row space (items are contiguous
// in the slab).  Map: 3-d view (16 doubles, Lr/8 lines, rows).  Buffer A is
// refilled as soon as A's forward transform has left it, buffer B after the
// inverse transform (which runs in B's buffer).
constexpr int pow2_floor(int x) { return x >= 2 ? 2 * pow2_floor(x / 2) : 1; }

template <int L> struct RowTile {
  // rows per unit: a power of two (so units never straddle items, whose row
  // counts are powers of two) with about BC_ROW_POINTS points per operand
  static constexpr int NR = pow2_floor(BC_ROW_POINTS / L > 0 ? BC_ROW_POINTS / L : 1);
  static constexpr int NT = (L / PTS) * NR;
  static constexpr int LINES = L / 8;
  // TMA boxes hold at most 256 lines: split a row into equal boxes
  static constexpr int PARTS = (LINES + 255) / 256;
  static constexpr int BOX_LINES = LINES / PARTS;
  static_assert(BOX_LINES * PARTS == LINES && BOX_LINES % 8 == 0, "row split into whole swizzle atoms");
  static_assert(PARTS == 1 || NR == 1, "split rows come one per unit");
  static constexpr int MINB = NT <= 128 ? 3 : (NT <= 256 ? 2 : 1);
  static constexpr size_t TILE = (size_t)NR * L * 16;  // one operand's rows of a unit
  // radix-8 stage twiddles in shared memory (staged layout)
  static constexpr int TWN = StagedTw<L>::entries();
  // slots per operand: two (the next unit loads while one is transformed)
  // when four tiles fit the 227 KB a CTA may use, else one
  static constexpr int SLOTS = (4 * TILE + (size_t)TWN * 16 + 1024 <= 227 * 1024) ? 2 : 1;
  static constexpr size_t SMEM = 2 * SLOTS * TILE + (size_t)TWN * 16 + 1024;
};

// Barrier of one row's L/8 threads inside k2_rows: a named barrier when the
// row is whole warps, the warp when a warp holds whole rows, else the CTA.
template <int L> struct RowSyncOf {
  static constexpr int TC = L / PTS;
  using type = typename std::conditional<(TC % 32 == 0), GroupSync<TC>,
                                         typename std::conditional<(32 % TC == 0), GroupSync<32>, CtaSync>::type>::type;
  __device__ static type make(int row) {
    if constexpr (std::is_same<type, CtaSync>::value) return CtaSync{};
    else return type{1 + row};
  }
};

template <int L>
__device__ __forceinline__ void rows_load(double2 *dst, const CUtensorMap *map, uint64_t *bar, unsigned row0) {
  using R = RowTile<L>;
  mbar_expect_tx(bar, (unsigned)R::NR * L * 16);
  if (R::PARTS == 1) {
    tma_load_3d(dst, map, bar, 0, 0, (int)row0);
  } else {
#pragma unroll
    for (int h = 0; h < R::PARTS; h++) tma_load_3d(dst + h * R::BOX_LINES * 8, map, bar, 0, h * R::BOX_LINES, (int)row0);
  }
}

// Buffers: A and B each have SLOTS slots (two where they fit), so the rows
// of unit u + SLOTS*grid load while unit u is transformed.  A's spectrum
// stays in its own slot; B's slot is free after the product, A's after the
// inverse transform (which exchanges through A's slot).  Squaring uses the
// A slots only.
template <int L, bool SQ>
__global__ void __launch_bounds__(RowTile<L>::NT, RowTile<L>::MINB)
    k2_rows(ClassParams p, const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB) {
  pdl_wait();
  pdl_trigger();
  using R = RowTile<L>;
  constexpr int TC = L / PTS, NR = R::NR, NS = R::SLOTS;
  extern __shared__ unsigned char smraw[];
  __shared__ uint64_t bars[4];  // A slot q: bars[q]; B slot q: bars[2 + q]
  double2 *const bufA0 = align1024(smraw);  // A slot q at bufA0 + q*NR*L, B slot q at bufA0 + (NS+q)*NR*L
  double2 *twS = bufA0 + 2 * NS * NR * L;
  staged_tw_build<L>(twS, p.twLr);
  const int tid = threadIdx.x, rl = tid / TC, t = tid % TC;
  const unsigned rows_item = p.M / L;
  const unsigned total = (unsigned)p.nitems * rows_item / NR;  // far below 2^32
  const FastDiv fd_rows(rows_item);
  // row of the B slab for class row `row` (item i's B transform sits in its slot)
  auto brow = [&](unsigned row) -> unsigned {
    const unsigned item = fd_rows.div(row);
    return (unsigned)p.items[item].bslot * rows_item + (row - item * rows_item);
  };
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) mbar_init(&bars[k], 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned u = blockIdx.x;
  unsigned pend = 0;  // bit k: a copy issued on bars[k] that has not been seen to land
#pragma unroll
  for (int q = 0; q < NS; q++) {
    const unsigned uq = u + q * gridDim.x;
    if (uq < total) {
      pend |= (1u << q) | (SQ ? 0u : 1u << (2 + q));
      if (tid == 0) {
        fence_proxy_async_smem();
        rows_load<L>(bufA0 + q * NR * L, &mA, &bars[q], uq * NR);
        if (!SQ) rows_load<L>(bufA0 + (NS + q) * NR * L, &mB, &bars[2 + q], brow(uq * NR));
      }
    }
  }
  using RS = typename RowSyncOf<L>::type;
  const RS rsync = RowSyncOf<L>::make(rl);  // the threads of this row
  unsigned phases = 0;                      // bit k: parity to wait for on bars[k]
  bool bad = false;                         // some wait of this thread gave up
  auto wait_slot = [&](int k) {
    const bool ok = mbar_wait(&bars[k], (phases >> k) & 1u);
    if (ok) {
      phases ^= 1u << k;
      pend &= ~(1u << k);
    }
    bad |= !ok;
  };
  // after a wait gave up anywhere in the CTA: flag the item, issue nothing
  // more, let the copies still in flight land (thread 0 issued them all)
  auto give_up = [&](const ItemDesc &it) {
    if (tid == 0) {
      atomicOr(it.flags, FLAG_TIMEOUT);
#pragma unroll
      for (int k = 0; k < 4; k++)
        if ((pend >> k) & 1u) mbar_drain(&bars[k], (phases >> k) & 1u);
    }
  };
  for (int q = 0; u < total; u += gridDim.x, q = (q + 1 == NS) ? 0 : q + 1) {
    const unsigned un = u + NS * gridDim.x;  // the unit this slot loads next
    const unsigned grow = u * NR + rl;        // this thread's row in the class slab
    const unsigned item = fd_rows.div(grow);
    const ItemDesc &it = p.items[item];
    double2 *ra = it.bufA + (grow - item * rows_item) * (unsigned)L;
    double2 *smA = bufA0 + q * NR * L + rl * L;
    double2 *smB = bufA0 + (NS + q) * NR * L + rl * L;
    double2 v[PTS];
    wait_slot(q);
#pragma unroll
    for (int i = 0; i < PTS; i++) v[i] = smA[ridx(t + i * TC)];
    rsync();
    block_fft<L, 1, false, RS, true>(v, t, 0, smA, p.twLr, rsync, twS);
    if (SQ) {
#pragma unroll
      for (int i = 0; i < PTS; i++) v[i] = cmul(v[i], v[i]);
      rsync();  // the inverse overwrites entries other threads of the row may still read
    } else {
#pragma unroll
      for (int i = 0; i < PTS; i++) smA[ridx(t + i * TC)] = v[i];  // A's spectrum, read back by this thread only
      wait_slot(2 + q);
#pragma unroll
      for (int i = 0; i < PTS; i++) v[i] = smB[ridx(t + i * TC)];
      rsync();
      block_fft<L, 1, false, RS, true>(v, t, 0, smB, p.twLr, rsync, twS);
#pragma unroll
      for (int i = 0; i < PTS; i++) v[i] = cmul(smA[ridx(t + i * TC)], v[i]);
      // every row is done with this B slot and with its spectrum reads
      if (__syncthreads_or(bad)) {
        give_up(it);
        return;
      }
      if (un < total) {
        pend |= 1u << (2 + q);
        if (tid == 0) {
          fence_proxy_async_smem();
          rows_load<L>(bufA0 + (NS + q) * NR * L, &mB, &bars[2 + q], brow(un * NR));
        }
      }
    }
    block_fft<L, 1, true, RS, true>(v, t, 0, smA, p.twLr, rsync, twS);
#pragma unroll
    for (int i = 0; i < PTS; i++) ra[t + i * TC] = v[i];
    // every row is done with this A slot
    if (__syncthreads_or(bad)) {
      give_up(it);
      return;
    }
    if (un < total) {
      pend |= 1u << q;
      if (tid == 0) {
        fence_proxy_async_smem();
        rows_load<L>(bufA0 + q * NR * L, &mA, &bars[q], un * NR);
      }
    }
  }
}

// ------------------------------------------------------------------ outer forward (pack)
// Units: (item, operand, column tile).  The limb words behind each tile row
// (real and imaginary digit runs) are staged with cp.async one unit ahead;
// digits are cut from shared memory.
template <int L> struct PackTile {
  static constexpr int W = PassTile<L>::W;
  // words per staged row segment for widths up to 24 bits: the segment starts
  // one word below the first digit's word and must hold the 64-bit window of
  // the last digit (start offset < 64 bits, last window ends below 24W + 95)
  static constexpr int SEGW = (24 * W + 95) / 32 + 1;
  // staged segment: up to 3 extra words in front so 16-byte chunks align
  static constexpr int SEGW4 = (SEGW + 3 + 3) / 4 * 4;
  static constexpr int STAGE_WORDS = 2 * L * SEGW4;
  // dynamic shared memory: tile, two limb stages, stage twiddles, weights, slack
  static constexpr size_t SMEM = (size_t)L * W * 16 + 2 * (size_t)STAGE_WORDS * 4 + (size_t)tw_entries<L>() * 16 +
                                 (size_t)L * 16 + 1024;
  // the 64-bit window of the last digit (b <= 24, shift <= 3 words) stays inside
  static_assert(SEGW4 >= ((158 + 24 * (W - 1)) >> 5) + 2, "staged segment too short");
};

template <int L>
__global__ void __launch_bounds__(PassTile<L>::NT, PassTile<L>::MINB) k2_outer_fwd(ClassParams p) {
  pdl_trigger();  // the first pass of a class: launched normally, lets the next one start early
  using T = PassTile<L>;
  using K = PackTile<L>;
  constexpr int W = T::W, TC = L / PTS, NT = T::NT;
  extern __shared__ unsigned char smraw[];
  double2 *tile = align1024(smraw);
  uint32_t *stg = reinterpret_cast<uint32_t *>(tile + L * W);  // 2 stages of STAGE_WORDS
  double2 *twS = reinterpret_cast<double2 *>(stg + 2 * K::STAGE_WORDS);
  double2 *pwS = twS + tw_entries<L>();
  table_to_smem(twS, p.twL1, tw_entries<L>());
  table_to_smem(pwS, p.pw_fwd, L);
  const int tid = threadIdx.x, s = tid % W, t = tid / W;
  const int tiles = p.S1 / W;
  const unsigned nA = fwd_units_a(p, (unsigned)tiles);
  const unsigned total = nA + fwd_units_b(p, (unsigned)tiles);  // far below 2^32
  const FastDiv fd_tile((unsigned)tiles);
  // Row segment (n1, part) of tile tl starts one word below the word of digit
  // j0 = n1*S1 + tl*W + part*M.  S1 and M are multiples of 128, so that word is
  // n1*(S1 b/32) + part*(M b/32) + (tl*W*b >> 5), with the first two terms
  // multiples of 4: every segment of a tile has the same alignment `dl` below
  // a 16-byte boundary, and digit j0 + s sits at bit
  // 32*(1 + dl) + (tl*W*b & 31) + s*b of its staged segment.
  auto seg_shift = [&](int tl, int b, bool al16) -> int {
    return al16 ? (int)((((long long)tl * W * b >> 5) - 1) & 3) : 0;
  };
  auto stage_copy = [&](unsigned u, int st) {
    const FwdUnit f = fwd_unit(p, u, nA, fd_tile, (unsigned)tiles);
    const int tl = (int)f.rest, op = f.op;
    const ItemDesc &it = p.items[f.item];
    const uint32_t *X = op ? it.B : it.A;
    // word indices fit an int: operands and transforms stay below 2^29 words
    const int XL = (int)(op ? it.BL : it.AL);
    const int b = it.b;
    const bool al16 = op ? it.b16 : it.a16;
    const int RW = (int)((unsigned)p.S1 * (unsigned)b / 32), PW = (int)((unsigned)p.M * (unsigned)b / 32);
    const int wbase = ((tl * W * b) >> 5) - 1 - seg_shift(tl, b, al16);
    uint32_t *dst = stg + st * K::STAGE_WORDS;
    // the imaginary parts hold digits M and up: none when nd <= M
    const int parts = (op ? it.ndB : it.ndA) > (unsigned long long)p.M ? 2 : 1;
    if (al16) {
      constexpr int CH = K::SEGW4 / 4;
      const int NCH = parts * L * CH;
      for (int idx = tid; idx < NCH; idx += NT) {
        const int segi = idx / CH, k = idx - segi * CH;
        const int part = segi >= L, row = segi - (part ? L : 0);
        const int w = row * RW + (part ? PW : 0) + wbase + 4 * k;  // multiple of 4
        int nv = XL - w;
        nv = nv < 0 ? 0 : (nv > 4 ? 4 : nv);
        if (w < 0) nv = 0;
        cp_async16(dst + segi * K::SEGW4 + 4 * k, X + (nv ? w : 0), nv * 4);
      }
    } else {
      for (int idx = tid; idx < parts * (K::STAGE_WORDS / 2); idx += NT) {
        const int segi = idx / K::SEGW4, k = idx - segi * K::SEGW4;
        const int part = segi >= L, row = segi - (part ? L : 0);
        const int w = row * RW + (part ? PW : 0) + wbase + k;
        const bool in = w >= 0 && w < XL;
        cp_async4(dst + idx, X + (in ? w : 0), in ? 4 : 0);
      }
    }
  };
  unsigned u = blockIdx.x;
  int st = 0;
  if (u < total) stage_copy(u, 0);
  cp_async_commit();
  for (; u < total; u += gridDim.x) {
    const unsigned un = u + gridDim.x;
    if (un < total) stage_copy(un, st ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const FwdUnit f = fwd_unit(p, u, nA, fd_tile, (unsigned)tiles);
    const int tl = (int)f.rest, op = f.op;
    const ItemDesc &it = p.items[f.item];
    const unsigned nd = (unsigned)(op ? it.ndB : it.ndA);  // below 2^30
    double2 *gbuf = op ? it.bufB : it.bufA;
    const int b = it.b;
    const uint32_t *seg = stg + st * K::STAGE_WORDS;
    const int col = tl * W + s;
    const bool al16 = op ? it.b16 : it.a16;
    const unsigned rel = 32u * (1u + (unsigned)seg_shift(tl, b, al16)) + (unsigned)((tl * W * b) & 31) +
                         (unsigned)(s * b);  // bit of digit j0+s in its staged segment
    const unsigned wi = (rel - 1) >> 5, sh = (rel - 1) & 31;
    const unsigned mask = (1u << b) - 1;
    const bool imag = nd > (unsigned)p.M;  // any digit at M or above (else not staged)
    // digit j of the operand from its staged segment (0 beyond nd)
    auto digit = [&](int part, int n1) -> double {
      const unsigned j = (unsigned)n1 * (unsigned)p.S1 + col + (part ? (unsigned)p.M : 0u);
      const uint32_t *rw = seg + (part * L + n1) * K::SEGW4 + wi;
      // bits [sh, sh+32) of the 64-bit window: the bit below the digit, then
      // its b <= 24 bits
      const unsigned x = __funnelshift_r(rw[0], rw[1], sh);
      const int r = (int)((x >> 1) & mask);
      const int top = (j + 1 >= nd) ? 0 : (r >> (b - 1));
      return j < nd ? (double)(r - (top << b) + (int)(x & 1u)) : 0.0;
    };
    double2 v[PTS];
    if (imag) {
#pragma unroll
      for (int i = 0; i < PTS; i++) {
        const int n1 = t + i * TC;
        v[i] = cmul(make_double2(digit(0, n1), digit(1, n1)), pwS[n1]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < PTS; i++) {
        const int n1 = t + i * TC;
        const double d = digit(0, n1);
        const double2 w = pwS[n1];
        v[i] = make_double2(d * w.x, d * w.y);
      }
    }
    block_fft<L, W, false>(v, t, s, tile, twS);
    double2 w[PTS];
    outer_twiddles<TC>(p.tw4M, col, t, w);
#pragma unroll
    for (int i = 0; i < PTS; i++) gbuf[(unsigned)(t + i * TC) * (unsigned)p.S1 + col] = cmul(v[i], w[i]);
    __syncthreads();
    st ^= 1;
  }
  cp_async_wait<0>();
}

}  // namespace bc
