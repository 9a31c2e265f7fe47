// bc_bsr.cuh — device kernels of the binary-splitting sum for e.
//
// The reference builds P(a,b), Q(a,b) with P/Q = sum_{j=a+1}^{b} 1/((a+1)(a+2)..j)
// and Q = (a+1)(a+2)..b by recursion on the host (main.c:63-109): leaves
// P = 1, Q = b, and P = P0*Q1 + P1, Q = Q0*Q1 at each node.  These integers
// do not depend on where the range is split, so the device version uses its
// own tree: leaves of up to 1024 consecutive terms computed one per warp
// (P(a,k+1) = P(a,k)*(k+1) + 1, Q(a,k+1) = Q(a,k)*(k+1)), then levels that
// pair neighbouring nodes, with both products of a level in one batched FFT
// multiply and the additions in k_add below.
#pragma once
#include <cuda/atomic>

#include "bc_kernels.cuh"

namespace bc {

// Wide leaves, one warp each: up to WLEAF_CAP limbs per value, lane l holding
// limbs [32l, 32l+32) in registers.  Per term k both values are multiplied
// by k (P also gets +1 at limb 0) lane by lane, and the carry out of a lane
// enters the next one (a second carry past a full lane ripples, bounded by
// 32 rounds).  A carry out of the top lane means the leaf was too wide for
// the capacity: flagged, never written past the buffer.
constexpr int WLEAF_LPL = 32;                    // limbs per lane
constexpr int WLEAF_CAP = 32 * WLEAF_LPL;        // limbs per value
constexpr int WLEAF_STRIDE = WLEAF_CAP + 2;      // limbs per stored value
constexpr int WLEAF_WARPS = 4;                   // warps per CTA

// x = x*k + add0 across the warp; returns 1 if a carry left the top lane.
__device__ __forceinline__ unsigned warp_mul_small(uint32_t (&x)[WLEAF_LPL], uint32_t k, uint32_t add0, int lane) {
  unsigned overflow = 0;
  uint32_t c = lane == 0 ? add0 : 0u;
#pragma unroll
  for (int q = 0; q < WLEAF_LPL; q++) {
    const unsigned long long v = (unsigned long long)x[q] * k + c;
    x[q] = (uint32_t)v;
    c = (uint32_t)(v >> 32);
  }
  uint32_t out = c;
  for (int round = 0; round < 32; round++) {
    if (lane == 31 && out) overflow = 1u;
    uint32_t cin = __shfl_up_sync(~0u, lane == 31 ? 0u : out, 1);
    if (lane == 0) cin = 0;
    if (!__any_sync(~0u, cin != 0)) break;
    uint32_t t = cin;
#pragma unroll
    for (int q = 0; q < WLEAF_LPL; q++) {
      const unsigned long long v = (unsigned long long)x[q] + t;
      x[q] = (uint32_t)v;
      t = (uint32_t)(v >> 32);
    }
    out = t;
  }
  return overflow;
}

// Leaf j covers terms (a + j*T, min(b, a + (j+1)*T)]; values go to
// out + (2j)*WLEAF_STRIDE (P) and out + (2j+1)*WLEAF_STRIDE (Q), lengths to
// len[2j], len[2j+1]; flags bit 0 on a capacity overflow.
__global__ void __launch_bounds__(32 * WLEAF_WARPS) k_bsr_leaves_wide(uint32_t a, uint32_t b, uint32_t T,
                                                                     uint32_t nleaf, uint32_t *out, uint32_t *len,
                                                                     unsigned *flags) {
  const int lane = threadIdx.x & 31;
  const uint32_t j = blockIdx.x * WLEAF_WARPS + (threadIdx.x >> 5);
  if (j >= nleaf) return;  // whole warps leave together
  const uint32_t a0 = a + j * T;
  const uint32_t b0 = min(b, a0 + T);
  uint32_t P[WLEAF_LPL], Q[WLEAF_LPL];
#pragma unroll
  for (int q = 0; q < WLEAF_LPL; q++) P[q] = Q[q] = 0;
  if (lane == 0) {
    P[0] = 1;
    Q[0] = a0 + 1;
  }
  unsigned ovf = 0;
  for (uint32_t k = a0 + 2; k <= b0; k++) {
    ovf |= warp_mul_small(P, k, 1u, lane);
    ovf |= warp_mul_small(Q, k, 0u, lane);
  }
  // lengths: highest nonzero limb + 1
  int hp = -1, hq = -1;
#pragma unroll
  for (int q = 0; q < WLEAF_LPL; q++) {
    if (P[q]) hp = lane * WLEAF_LPL + q;
    if (Q[q]) hq = lane * WLEAF_LPL + q;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    hp = max(hp, __shfl_xor_sync(~0u, hp, o));
    hq = max(hq, __shfl_xor_sync(~0u, hq, o));
  }
  uint32_t *oP = out + (size_t)(2 * j) * WLEAF_STRIDE, *oQ = oP + WLEAF_STRIDE;
#pragma unroll
  for (int q = 0; q < WLEAF_LPL; q++) {
    const int i = lane * WLEAF_LPL + q;
    if (i <= hp) oP[i] = P[q];
    if (i <= hq) oQ[i] = Q[q];
  }
  if (lane == 0) {
    len[2 * j] = (uint32_t)(hp + 1);
    len[2 * j + 1] = (uint32_t)(hq + 1);
  }
  if (__any_sync(~0u, ovf != 0) && lane == 0) atomicOr(flags, 1u);
}

// Significant length of each product C_i of CL_i limbs whose operands had
// nonzero top limbs: CL_i or CL_i - 1.
struct TrimDesc {
  const uint32_t *C;
  unsigned long long CL;
};
__global__ void k_trim(const TrimDesc *d, uint32_t n, unsigned long long *len) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long CL = d[i].CL;
  len[i] = CL - (CL > 1 && d[i].C[CL - 1] == 0 ? 1 : 0);
}

// R = X + Y for a batch of items: n = max(lx, ly) limbs of sum, then the
// carry out as limb n (len = n + carry).  An item has n / ADD_TILE + 1 tiles
// (the last one holds limb n) of ADD_TILE limbs; the carry
// into a tile is found by a decoupled lookback over the tiles of the item,
// with the carry maps {0,1} -> {0,1} kept in the {-1,0,1} map encoding of
// the multiply's carry scan (fn_make / fn_compose).
constexpr int ADD_NT = 256, ADD_PT = 8, ADD_TILE = ADD_NT * ADD_PT;

struct AddDesc {
  const uint32_t *x;
  const uint32_t *y;
  uint32_t *r;
  unsigned long long lx, ly, n;
  unsigned long long tile0;  // first tile of this item (batch-wide numbering)
};

struct AddParams {
  const AddDesc *items;
  int nitems;
  unsigned long long tiles;
  unsigned int *counter;       // zeroed before launch
  uint32_t *status;            // one word per tile, zeroed before launch
  unsigned long long *len;     // per item: n + carry out
  unsigned int *flags;         // bit 0: a lookback wait ran out
};

__global__ void __launch_bounds__(ADD_NT) k_add(AddParams p) {
  __shared__ uint32_t sw[65];
  __shared__ unsigned long long s_unit;
  __shared__ int s_cin;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(p.counter, 1u);
    __syncthreads();
    const unsigned long long unit = s_unit;
    if (unit >= p.tiles) break;
    int lo = 0, hi = p.nitems - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.items[mid].tile0 <= unit) lo = mid; else hi = mid - 1;
    }
    const AddDesc &it = p.items[lo];
    const unsigned long long tile = unit - it.tile0;
    const unsigned long long i0 = tile * ADD_TILE + (unsigned long long)tid * ADD_PT;
    uint32_t s[ADD_PT];
    unsigned c = 0;
    bool ones = true;
#pragma unroll
    for (int q = 0; q < ADD_PT; q++) {
      const unsigned long long i = i0 + q;
      const uint32_t xv = i < it.lx ? it.x[i] : 0u, yv = i < it.ly ? it.y[i] : 0u;
      const unsigned long long v = (unsigned long long)xv + yv + c;
      s[q] = (uint32_t)v;
      c = (unsigned)(v >> 32);
      if (i < it.n) ones = ones && s[q] == 0xffffffffu;
    }
    // carry out of this thread's limbs given its carry in: c, or c | ones
    const int c0 = (int)c, c1 = (int)(c | (ones ? 1u : 0u));
    const uint32_t f = fn_make(c0, c0, c1);
    uint32_t agg;
    const uint32_t ex = block_scan_fn<ADD_NT>(f, sw, &agg);
    if (tid == 0) {
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> me(p.status[it.tile0 + tile]);
      int cin = 0;
      if (tile == 0) {
        me.store(ST_INC | (uint32_t)(fn_apply(agg, 0) + 1), cuda::memory_order_release);
      } else {
        if (fn_is_const(agg)) me.store(ST_INC | (uint32_t)(fn_apply(agg, 0) + 1), cuda::memory_order_release);
        else me.store(ST_AGG | agg, cuda::memory_order_release);
        uint32_t acc = FN_ID;
        long long prev = (long long)tile - 1;
        int spins = 0;
        bool timed_out = false;
        for (;;) {
          cuda::atomic_ref<uint32_t, cuda::thread_scope_device> st(p.status[it.tile0 + prev]);
          const uint32_t v = st.load(cuda::memory_order_acquire);
          if (v & ST_INC) {
            cin = fn_apply(acc, (int)(v & 3u) - 1);
            break;
          } else if (v & ST_AGG) {
            const uint32_t fv = v & 0x3fu;
            if (fn_is_const(fv)) { cin = fn_apply(acc, fn_apply(fv, 0)); break; }
            acc = fn_compose(fv, acc);
            prev--;
          } else {
            if (++spins > LOOKBACK_SPINS) { timed_out = true; break; }
            if (spins > 64) __nanosleep(32);
          }
        }
        if (timed_out) {
          atomicOr(p.flags, 1u);
          cin = 0;
        }
        if (!fn_is_const(agg)) me.store(ST_INC | (uint32_t)(fn_apply(agg, cin) + 1), cuda::memory_order_release);
      }
      s_cin = cin;
    }
    __syncthreads();
    unsigned cc = (unsigned)fn_apply(ex, s_cin);  // carry into this thread's limbs
    uint32_t top = 0;
    bool has_top = false;
#pragma unroll
    for (int q = 0; q < ADD_PT; q++) {
      const unsigned long long i = i0 + q;
      const unsigned long long v = (unsigned long long)s[q] + cc;
      cc = (unsigned)(v >> 32);
      if (i < it.n) it.r[i] = (uint32_t)v;
      else if (i == it.n) { top = (uint32_t)v; has_top = true; }
    }
    // limb n (inside the item's last tile) is the carry out of limb n-1
    if (has_top) {
      it.r[it.n] = top;
      p.len[lo] = it.n + top;
    }
    __syncthreads();
  }
}

}  // namespace bc
