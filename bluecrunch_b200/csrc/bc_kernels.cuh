// bc_kernels.cuh — shared pieces of the exact FFT multiply (sm_100a): item
// and class descriptors, rounding check, the carry kernel and the one-CTA
// kernel for short transforms.
//
// A product class has complex length M = L1 * S1 (two levels, S1 = Lr) or
// M = L1 * L2 * Lr (three levels).  Point n of operand X holds the balanced
// digits n and n+M weighted by e^{i pi n/(2M)}.  Passes (one launch each,
// every launch covers all items of the class; the pass kernels are in
// bc_pipe.cuh):
//
//   k2_outer_fwd  digits -> pre-weight -> L1-point DFT down each column of the
//                 L1 x S1 matrix -> twiddle e^{-2 pi i s(4k1-1)/(4M)} (the
//                 column's weight factor folded in) -> buffer
//   k2_mid<L,0>   (3 levels) L2-point DFT down columns of each L2 x Lr block,
//                 twiddle e^{-2 pi i s k2/(L2 Lr)}
//   k2_rows       per row of Lr points: forward DFT of A and B, pointwise
//                 product (or square), inverse DFT — the spectrum never
//                 leaves the chip (rows of 1024 points: k2_rows_w1024, one
//                 warp per row, bc_rows_warp.cuh)
//   k2_mid<L,1>   (3 levels) inverse of k2_mid<L,0>
//   k2_outer_inv  conjugate twiddle -> inverse L1-point DFT -> un-weight and
//                 1/M -> round (max |x - round(x)| recorded) -> run records:
//                 8 consecutive coefficients -> (H, C), value H + C*2^{8b}
//   k_carry       decoupled-lookback scan of run carries -> output words
//
// k_small does all of it in one CTA for M <= 4096.
//
// Reference correspondence: the whole pipeline computes what _fft_mul
// computes (bigfloat/mul.c:108-174): the exact C = A*B mod 2^{32 CL}.
#pragma once
#include <cuda/atomic>

#include "bc_async.cuh"
#include "bc_device.cuh"

namespace bc {

enum : unsigned { FLAG_TIMEOUT = 1u, FLAG_TOPCARRY = 2u };

struct ItemDesc {
  const uint32_t *A;
  const uint32_t *B;
  uint32_t *C;
  unsigned long long AL, BL, CL;  // AL, BL already clamped to CL
  unsigned long long ndA, ndB;    // number of balanced digits
  double2 *bufA;
  double2 *bufB;                  // null when squaring
  RunRec *rec;                    // 2M/8 run records
  uint32_t *status;               // lookback tile status, zeroed before k_carry
  unsigned long long nwords;      // words written by k_carry (the rest are 0)
  unsigned long long nruns;       // runs needed to cover nwords
  unsigned long long tile0;       // first k_carry tile of this item (class-wide numbering)
  unsigned long long *err;        // max rounding error as double bits (atomicMax)
  unsigned int *flags;
  int b;
  int square;
  int a16, b16;                   // operand A / B starts on a 16-byte boundary
  int bslot;                      // slot of B's transform in the class's B slab (shared by items with the same B)
};

struct ClassParams {
  int M;
  int L1, S1;      // outer pass: L1-point DFTs with stride S1 = M/L1
  int L2, Lr;      // 3 levels: L2-point DFTs with stride Lr; 2 levels: L2 = 1, Lr = S1
  // Forward-pass units: the A transform of every item, then the B slab's
  // slots (nb of them; slot j is B of item bowner[j], null: item j).  Items
  // with the same B share one slot, so their B is packed and transformed
  // once.  fwd_ops restricts the outer forward pass to A (1) or B (2)
  // units; 0 covers both.
  int fwd_ops;
  int nb;
  const int *bowner;
  Tw2 tw4M;        // e^{-2 pi i m/(4M)}
  const double2 *pw_fwd;  // e^{+i pi n1/(2 L1)}
  const double2 *pw_inv;  // e^{-i pi n1/(2 L1)} / M
  const double2 *twL1, *twL2, *twLr;  // e^{-2 pi i m/L}
  const ItemDesc *items;
  int nitems;
  int sq;                 // every item of the class squares (one operand)
  unsigned int *counter;  // k_carry dynamic tile counter (zeroed before launch)
  unsigned long long carry_tiles;  // total k_carry tiles over the class
  // fused middle pass (three levels): per block (nitems * L1 of them) the
  // count of finished column items, then of finished row items; zeroed
  // before launch.  Null: the middle runs as separate passes.
  unsigned int *blkdone;
  double2 *slabA, *slabB;          // the class's A and B slabs (item i at slab + i*slab_elems)
  unsigned long long slab_elems;
};

// One unit of a forward pass: operand `op` of item `item` (for B, the owner
// of slot `slot`), and the unit's index `rest` inside that operand's
// per_op units.  Units [0, nA) are A's (item-major), the rest B's
// (slot-major).
struct FwdUnit {
  int item, op, slot;
  unsigned rest;
};
__device__ __forceinline__ FwdUnit fwd_unit(const ClassParams &p, unsigned u, unsigned nA, const FastDiv &fd_op,
                                            unsigned per_op) {
  FwdUnit f;
  if (u < nA) {
    const unsigned i = fd_op.div(u);
    f.item = (int)i;
    f.slot = (int)i;
    f.op = 0;
    f.rest = u - i * per_op;
  } else {
    const unsigned v = u - nA, j = fd_op.div(v);
    f.slot = (int)j;
    f.item = p.bowner ? p.bowner[j] : (int)j;
    f.op = 1;
    f.rest = v - j * per_op;
  }
  return f;
}
// A and B unit counts of a forward pass with per_op units per operand.
__device__ __forceinline__ unsigned fwd_units_a(const ClassParams &p, unsigned per_op) {
  return p.fwd_ops != 2 ? (unsigned)p.nitems * per_op : 0u;
}
__device__ __forceinline__ unsigned fwd_units_b(const ClassParams &p, unsigned per_op) {
  return (!p.sq && p.fwd_ops != 1) ? (unsigned)p.nb * per_op : 0u;
}

// e^{-2 pi i m/(4M)} for m = s*(4k-1) with s < S, k < 4M/(4S): m < 4M when
// k >= 1; for k = 0 it is the conjugate of m = s.
__device__ __forceinline__ double2 outer_tw(const Tw2 &T, int s, int k) {
  if (k == 0) { double2 w = tw2_get(T, (uint64_t)s); return make_double2(w.x, -w.y); }
  return tw2_get(T, (uint64_t)s * (uint64_t)(4 * k - 1));
}

// Rounding check of one point: max |x - round(x)| of its two coefficients,
// or 1.0 when a coefficient reaches 2^50 — beyond that the distance to the
// nearest integer stops measuring the error (doubles near 2^53 hold no
// fractions), so the product must be redone with narrower digits.
__device__ __forceinline__ double round_check(double2 z, double re, double im) {
  const double big = 1125899906842624.0;  // 2^50
  double e = fmax(fabs(z.x - re), fabs(z.y - im));
  return (fabs(re) >= big || fabs(im) >= big) ? 1.0 : e;
}

__device__ __forceinline__ void atomic_max_err(unsigned long long *p, double e) {
  // non-negative doubles order like their bit patterns
  unsigned long long bits = (unsigned long long)__double_as_longlong(e);
  for (int o = 16; o; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(~0u, bits, o);
    bits = t > bits ? t : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(p, bits);
}

// ------------------------------------------------------------------ runs
// 8 consecutive rounded coefficients c_u (exact integers held in doubles) ->
// H = sum (bits of the running carry) and C = final signed carry.
// h |= bits << off for off < 192 (selects instead of a runtime word index,
// so h stays in registers).
__host__ __device__ __forceinline__ void u192_or_bits(U192 &h, unsigned long long bits, int off) {
  const int wi = off >> 6, bi = off & 63;
  const unsigned long long lo = bits << bi, hi = bi ? bits >> (64 - bi) : 0ull;
  h.w[0] |= wi == 0 ? lo : 0ull;
  h.w[1] |= wi == 1 ? lo : (wi == 0 ? hi : 0ull);
  h.w[2] |= wi == 2 ? lo : (wi == 1 ? hi : 0ull);
}

__host__ __device__ __forceinline__ RunRec make_run(const double *c, int b) {
  if (b == 16) {
    // 8 x 16 bits fill two words exactly: constant shifts, no selects
    unsigned long long h0 = 0, h1 = 0;
    long long acc = 0;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      acc += (long long)c[u];
      const unsigned long long bits = (unsigned long long)acc & 0xffffull;
      if (u < 4) h0 |= bits << (16 * u);
      else h1 |= bits << (16 * (u - 4));
      acc >>= 16;
    }
    RunRec r;
    r.h0 = h0; r.h1 = h1; r.h2 = 0; r.c = acc;
    return r;
  }
  U192 h = {{0, 0, 0}};
  long long acc = 0;
  const unsigned long long mask = (1ull << b) - 1;
#pragma unroll
  for (int u = 0; u < 8; u++) {
    acc += (long long)c[u];
    u192_or_bits(h, (unsigned long long)acc & mask, b * u);
    acc >>= b;  // arithmetic: floor division
  }
  RunRec r;
  r.h0 = h.w[0]; r.h1 = h.w[1]; r.h2 = h.w[2]; r.c = acc;
  return r;
}

__device__ __forceinline__ void store_rec(RunRec *dst, const RunRec &r) {
  ulonglong2 *d = reinterpret_cast<ulonglong2 *>(dst);
  d[0] = make_ulonglong2(r.h0, r.h1);
  d[1] = make_ulonglong2(r.h2, (unsigned long long)r.c);
}

__device__ __forceinline__ RunRec load_rec(const RunRec *src) {
  const ulonglong2 *s = reinterpret_cast<const ulonglong2 *>(src);
  ulonglong2 a = s[0], b = s[1];
  RunRec r;
  r.h0 = a.x; r.h1 = a.y; r.h2 = b.x; r.c = (long long)b.y;
  return r;
}

// ------------------------------------------------------------------ scan helper
// Exclusive scan of transfer functions over a CTA of NT threads (earliest
// thread first).  sw needs 65 words.  Returns the exclusive prefix; *total
// receives the composition over the whole CTA.
template <int NT>
__device__ __forceinline__ uint32_t block_scan_fn(uint32_t f, uint32_t *sw, uint32_t *total) {
  static_assert(NT % 32 == 0 && NT <= 1024, "scan CTA size");
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = f;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t o = __shfl_up_sync(~0u, inc, d);
    if (lane >= d) inc = fn_compose(o, inc);
  }
  uint32_t ex = __shfl_up_sync(~0u, inc, 1);
  if (lane == 0) ex = FN_ID;
  if (lane == 31) sw[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t x = lane < NW ? sw[lane] : FN_ID;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t o = __shfl_up_sync(~0u, x, d);
      if (lane >= d) x = fn_compose(o, x);
    }
    uint32_t wx = __shfl_up_sync(~0u, x, 1);
    if (lane == 0) wx = FN_ID;
    if (lane < NW) sw[32 + lane] = wx;
    if (lane == 31) sw[64] = x;
  }
  __syncthreads();
  const uint32_t r = fn_compose(sw[32 + wid], ex);
  *total = sw[64];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------ carry
// Decoupled lookback over tiles of CARRY_NT runs.  Tile status word:
// 0 = not ready, (1<<30)|fn = aggregate, (2<<30)|(delta+1) = inclusive.
constexpr int CARRY_NT = 256;
constexpr int CARRY_RPT = 4;                            // runs per thread
constexpr int CARRY_TILE_RUNS = CARRY_NT * CARRY_RPT;   // runs per lookback tile
constexpr unsigned ST_AGG = 1u << 30, ST_INC = 2u << 30;
constexpr int LOOKBACK_SPINS = 1 << 22;

__device__ __forceinline__ U192 rec_h(const RunRec &r) { U192 h = {{r.h0, r.h1, r.h2}}; return h; }

// Words of run r (bits [r nbits, (r+1) nbits)) below nwords; a word that
// straddles into run r+1 takes its high bits from hn.
__device__ __forceinline__ void write_run_words(uint32_t *C, unsigned long long nwords, unsigned long long r,
                                                int nbits, const U192 &h, const U192 &hn) {
  const unsigned long long bit0 = r * (unsigned long long)nbits;
  unsigned long long w = (bit0 + 31) >> 5;
  const unsigned long long wend = (bit0 + nbits + 31) >> 5;
  for (; w < wend && w < nwords; w++) {
    const int off = (int)((w << 5) - bit0);
    uint32_t x = u192_bits32(h, off);
    if (off + 32 > nbits) x |= u192_bits32(hn, 0) << (nbits - off);
    C[w] = x;
  }
}

// 16-byte chunk c of a staged tile of run records lives at chunk position
// (c & ~7) | ((c ^ (c >> 3)) & 7): the 8 chunks of one thread's 4 records
// (8t .. 8t+7) land on 8 distinct bank groups across any 8 threads.
__device__ __forceinline__ int rec_chunk_pos(int c) { return (c & ~7) | ((c ^ (c >> 3)) & 7); }

// Corrected run values of a tile as three 64-bit planes (plane stride
// CARRY_TILE_RUNS + 1 words: entry CARRY_TILE_RUNS is the run after the
// tile's last one, for the word that straddles it).
constexpr int HC_STRIDE = CARRY_TILE_RUNS + 1;

// NB = 128: every item of the class has width 16 (runs of 128 bits), so the
// run arithmetic below is specialised at compile time; NB = 0: any width.
template <int NB>
__global__ void __launch_bounds__(CARRY_NT) k_carry(ClassParams p) {
  // records of the tile (32 KB), then reused for the corrected values
  __shared__ __align__(16) unsigned long long srec[CARRY_TILE_RUNS * 4];
  static_assert(3 * HC_STRIDE <= CARRY_TILE_RUNS * 4, "corrected values fit the record buffer");
  __shared__ uint32_t sw[65];
  __shared__ unsigned long long s_unit;
  __shared__ int s_delta;
  __shared__ long long s_cprev;
  const int tid = threadIdx.x;
  pdl_wait();
  pdl_trigger();
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(p.counter, 1u);
    __syncthreads();
    const unsigned long long unit = s_unit;
    if (unit >= p.carry_tiles) break;
    // find the item owning this tile (items are ordered by tile0)
    int lo = 0, hi = p.nitems - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (p.items[mid].tile0 <= unit) lo = mid; else hi = mid - 1;
    }
    const ItemDesc &it = p.items[lo];
    const unsigned long long tile = unit - it.tile0;
    const unsigned long long rt = tile * CARRY_TILE_RUNS;  // first run of the tile
    const unsigned long long nruns = it.nruns;
    const int nr = (int)min((unsigned long long)CARRY_TILE_RUNS, nruns - rt);  // runs of this tile
    const int nbits = NB ? NB : 8 * it.b;
    const unsigned long long nrec = (unsigned long long)(2 * p.M) / 8;
    // ---- stage the tile's records (coalesced 16-byte copies) and C_{rt-1}
    {
      const char *src = reinterpret_cast<const char *>(it.rec + rt);
      char *dst = reinterpret_cast<char *>(srec);
      const int nch = 2 * nr;
      for (int c = tid; c < 2 * CARRY_TILE_RUNS; c += CARRY_NT)
        cp_async16(dst + 16 * rec_chunk_pos(c), src + (c < nch ? 16 * c : 0), c < nch ? 16 : 0);
      cp_async_commit();
      if (tid == 0) s_cprev = rt > 0 ? load_rec(&it.rec[rt - 1]).c : 0;
      cp_async_wait<0>();
    }
    __syncthreads();
    // ---- this thread's CARRY_RPT consecutive runs
    const int k0 = tid * CARRY_RPT;
    U192 h[CARRY_RPT];
    long long c[CARRY_RPT];
    uint32_t f[CARRY_RPT];
    uint32_t F = FN_ID;
    long long cprev = s_cprev;
    if (k0 > 0 && k0 <= nr) {
      const int ch = rec_chunk_pos(2 * (k0 - 1) + 1);  // second chunk of record k0-1: (h2, c)
      cprev = (long long)srec[2 * ch + 1];
    }
#pragma unroll
    for (int q = 0; q < CARRY_RPT; q++) {
      const int k = k0 + q;
      f[q] = FN_ID;
      c[q] = 0;
      h[q].w[0] = h[q].w[1] = h[q].w[2] = 0;
      if (k < nr) {
        const int ca = rec_chunk_pos(2 * k), cb = rec_chunk_pos(2 * k + 1);
        h[q].w[0] = srec[2 * ca];
        h[q].w[1] = srec[2 * ca + 1];
        h[q].w[2] = srec[2 * cb];
        c[q] = (long long)srec[2 * cb + 1];
        f[q] = run_transfer(h[q], cprev, nbits);
        cprev = c[q];
        F = fn_compose(F, f[q]);
      }
    }
    uint32_t agg;
    const uint32_t ex = block_scan_fn<CARRY_NT>(F, sw, &agg);  // ends past a barrier: srec is free
    if (tid == 0) {
      // A tile whose composed map is constant knows its carry out before its
      // carry in: it publishes that at once, and a lookback that meets such an
      // aggregate can stop there.  Nearly every tile is constant, so waits are
      // one status read deep.
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> me(it.status[tile]);
      int din = 0;
      if (tile == 0) {
        me.store(ST_INC | (uint32_t)(fn_apply(agg, 0) + 1), cuda::memory_order_release);
      } else {
        if (fn_is_const(agg)) me.store(ST_INC | (uint32_t)(fn_apply(agg, 0) + 1), cuda::memory_order_release);
        else me.store(ST_AGG | agg, cuda::memory_order_release);
        uint32_t acc = FN_ID;  // maps of the tiles passed so far (nearest applied last)
        long long prev = (long long)tile - 1;
        int spins = 0;
        bool timed_out = false;
        for (;;) {
          cuda::atomic_ref<uint32_t, cuda::thread_scope_device> st(it.status[prev]);
          const uint32_t v = st.load(cuda::memory_order_acquire);
          if (v & ST_INC) {
            din = fn_apply(acc, (int)(v & 3u) - 1);
            break;
          } else if (v & ST_AGG) {
            const uint32_t fv = v & 0x3fu;
            if (fn_is_const(fv)) { din = fn_apply(acc, fn_apply(fv, 0)); break; }
            acc = fn_compose(fv, acc);
            prev--;
          } else {
            if (++spins > LOOKBACK_SPINS) { timed_out = true; break; }
            if (spins > 64) __nanosleep(32);
          }
        }
        if (timed_out) {
          atomicOr(it.flags, FLAG_TIMEOUT);
          din = 0;
        }
        if (!fn_is_const(agg)) me.store(ST_INC | (uint32_t)(fn_apply(agg, din) + 1), cuda::memory_order_release);
      }
      s_delta = din;
    }
    __syncthreads();
    // ---- carries into each run; corrected values to shared memory, or
    // (runs of 128 bits, every word of the tile inside the product, C on a
    // 16-byte boundary) each run's four words straight to C
    unsigned long long *hc = srec;
    const bool whole = nbits == 128 && (reinterpret_cast<uintptr_t>(it.C) & 15) == 0 &&
                       4ull * (rt + (unsigned long long)nr) <= it.nwords;
    int d = fn_apply(ex, s_delta);  // delta into run k0
#pragma unroll
    for (int q = 0; q < CARRY_RPT; q++) {
      const int k = k0 + q;
      if (k < nr) {
        u192_add_delta(h[q], d, nbits);
        d = fn_apply(f[q], d);
        if (whole) {
          *reinterpret_cast<uint4 *>(it.C + 4 * (rt + (unsigned long long)k)) =
              make_uint4((uint32_t)h[q].w[0], (uint32_t)(h[q].w[0] >> 32), (uint32_t)h[q].w[1],
                         (uint32_t)(h[q].w[1] >> 32));
        } else {
          hc[k] = h[q].w[0];
          hc[HC_STRIDE + k] = h[q].w[1];
          hc[2 * HC_STRIDE + k] = h[q].w[2];
        }
        if (k + 1 == nr) {
          // the run after the tile's last one, for a word that straddles it:
          // inside this item only when the item ends inside this tile
          U192 hn = {{0, 0, 0}};
          const unsigned long long r = rt + k;
          if (nr < CARRY_TILE_RUNS && r + 1 < nrec) {
            RunRec rn = load_rec(&it.rec[r + 1]);
            hn = rec_h(rn);
            (void)u192_add_s64(hn, c[q], nbits);
            u192_add_delta(hn, d, nbits);
          }
          hc[nr] = hn.w[0];
          hc[HC_STRIDE + nr] = hn.w[1];
          hc[2 * HC_STRIDE + nr] = hn.w[2];
          if (r + 1 == nrec && c[q] + d != 0) atomicOr(it.flags, FLAG_TOPCARRY);
        }
      }
    }
    // ---- words of the tile, one per thread per step (coalesced stores).
    // The tile starts on a word boundary (1024 runs of 8b bits).
    if (!whole) {  // uniform over the CTA
      __syncthreads();
      const unsigned long long w0 = rt * (unsigned long long)nbits / 32;
      const unsigned long long wend =
          min(it.nwords, (rt * (unsigned long long)nbits + (unsigned long long)nr * nbits + 31) / 32);
      const int nw = wend > w0 ? (int)(wend - w0) : 0;
      // run of word i: 32i / (8b) = 4i / b = (4i * ceil(2^20/b)) >> 20, exact
      // for 4i*b < 2^20 (here i < 6144 and b <= 24)
      const unsigned rb = ((1u << 20) + (unsigned)it.b - 1) / (unsigned)it.b;
      for (int i = tid; i < nw; i += CARRY_NT) {
        const int bit = 32 * i;
        const int k = (int)((4u * (unsigned)i * rb) >> 20), off = bit - k * nbits;
        U192 hk = {{hc[k], hc[HC_STRIDE + k], hc[2 * HC_STRIDE + k]}};
        uint32_t x = u192_bits32(hk, off);
        if (off + 32 > nbits) {
          U192 hn = {{hc[k + 1], hc[HC_STRIDE + k + 1], hc[2 * HC_STRIDE + k + 1]}};
          x |= u192_bits32(hn, 0) << (nbits - off);
        }
        it.C[w0 + i] = x;
      }
    }
    // zero any words beyond the product (CL > product length)
    if (tile == 0) {
      for (unsigned long long w = it.nwords + tid; w < it.CL; w += CARRY_NT) it.C[w] = 0;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ small
// Whole product in one CTA of M/8 threads (M <= 4096): pack, FFT, product,
// inverse, round, runs, in-CTA carry scan, words.
template <int M, bool SQ>
__global__ void __launch_bounds__(M / PTS, 1) k_small(ClassParams p) {
  extern __shared__ double2 sm[];
  constexpr int TC = M / PTS, NR = M / 8;  // NR real runs, NR imaginary runs
  static_assert(TC % 32 == 0, "k_small needs M >= 256");
  __shared__ uint32_t sw[65];
  const int t = threadIdx.x;
  RunRec *srec = reinterpret_cast<RunRec *>(sm);  // reused after the FFTs
  for (int item = blockIdx.x; item < p.nitems; item += gridDim.x) {
    const ItemDesc &it = p.items[item];
    double2 va[PTS], v[PTS];
#pragma unroll
    for (int i = 0; i < PTS; i++) {
      const int n = t + i * TC;
      double2 z = make_double2(digit_at(it.A, it.AL, it.b, n, it.ndA), digit_at(it.A, it.AL, it.b, n + M, it.ndA));
      va[i] = cmul(z, __ldg(&p.pw_fwd[n]));
    }
    block_fft<M, 1, false>(va, t, 0, sm, p.twL1);
    if (SQ) {
#pragma unroll
      for (int i = 0; i < PTS; i++) v[i] = cmul(va[i], va[i]);
    } else {
#pragma unroll
      for (int i = 0; i < PTS; i++) {
        const int n = t + i * TC;
        double2 z = make_double2(digit_at(it.B, it.BL, it.b, n, it.ndB), digit_at(it.B, it.BL, it.b, n + M, it.ndB));
        v[i] = cmul(z, __ldg(&p.pw_fwd[n]));
      }
      block_fft<M, 1, false>(v, t, 0, sm, p.twL1);
#pragma unroll
      for (int i = 0; i < PTS; i++) v[i] = cmul(va[i], v[i]);
    }
    block_fft<M, 1, true>(v, t, 0, sm, p.twL1);
    double err = 0.0;
#pragma unroll
    for (int i = 0; i < PTS; i++) {
      const int n = t + i * TC;
      double2 z = cmul(v[i], __ldg(&p.pw_inv[n]));
      double re = rint(z.x), im = rint(z.y);
      err = fmax(err, round_check(z, re, im));
      sm[sidx<M, 1>(n, 0)] = make_double2(re, im);
    }
    atomic_max_err(it.err, err);
    __syncthreads();
    double cre[8], cim[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      double2 z = sm[sidx<M, 1>(8 * t + u, 0)];
      cre[u] = z.x; cim[u] = z.y;
    }
    RunRec rre = make_run(cre, it.b), rim = make_run(cim, it.b);
    __syncthreads();
    srec[t] = rre;
    srec[NR + t] = rim;
    __syncthreads();
    const int nbits = 8 * it.b;
    // transfer functions
    U192 hre = rec_h(rre), him = rec_h(rim);
    const long long cprev_re = t ? srec[t - 1].c : 0;
    const long long cprev_im = srec[NR + t - 1].c;
    const uint32_t fre = run_transfer(hre, cprev_re, nbits);
    const uint32_t fim = run_transfer(him, cprev_im, nbits);
    uint32_t tot_re, tot_im;
    const uint32_t ex_re = block_scan_fn<TC>(fre, sw, &tot_re);
    const uint32_t ex_im = block_scan_fn<TC>(fim, sw, &tot_im);
    const int din_re = fn_apply(ex_re, 0);
    const int d_half = fn_apply(tot_re, 0);
    const int din_im = fn_apply(ex_im, d_half);
    u192_add_delta(hre, din_re, nbits);
    u192_add_delta(him, din_im, nbits);
    const int dout_im = fn_apply(fim, din_im);
    __syncthreads();
    srec[t].h0 = hre.w[0]; srec[t].h1 = hre.w[1]; srec[t].h2 = hre.w[2];
    srec[NR + t].h0 = him.w[0]; srec[NR + t].h1 = him.w[1]; srec[NR + t].h2 = him.w[2];
    __syncthreads();
    const U192 zero = {{0, 0, 0}};
    const U192 nre = rec_h(srec[t + 1 < 2 * NR ? t + 1 : t]);
    const U192 nim = (NR + t + 1 < 2 * NR) ? rec_h(srec[NR + t + 1]) : zero;
    write_run_words(it.C, it.nwords, (unsigned long long)t, nbits, hre, nre);
    write_run_words(it.C, it.nwords, (unsigned long long)(NR + t), nbits, him, nim);
    if (t == TC - 1 && rim.c + dout_im != 0) atomicOr(it.flags, FLAG_TOPCARRY);
    for (unsigned long long w = it.nwords + t; w < it.CL; w += TC) it.C[w] = 0;
    __syncthreads();
  }
}

}  // namespace bc
