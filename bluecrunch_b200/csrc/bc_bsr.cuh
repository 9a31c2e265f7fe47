// bc_bsr.cuh — device kernels of the binary-splitting sum for e.
//
// The reference builds P(a,b), Q(a,b) with P/Q = sum_{j=a+1}^{b} 1/((a+1)(a+2)..j)
// and Q = (a+1)(a+2)..b by recursion on the host (main.c:63-109): leaves
// P = 1, Q = b, and P = P0*Q1 + P1, Q = Q0*Q1 at each node.  These integers
// do not depend on where the range is split, so the device version uses its
// own tree: leaves of up to LEAF_TERMS consecutive terms computed one per
// thread, then levels that pair neighbouring nodes, with both products of a
// level in one batched FFT multiply and the additions in k_add below.
#pragma once
#include <cuda/atomic>

#include "bc_kernels.cuh"

namespace bc {

constexpr int LEAF_TERMS = 64;
constexpr int LEAF_STRIDE = 66;  // limbs per leaf value: Q < 2^(32*64), P < 2Q
constexpr int LEAF_NT = 64;  // 2 x 66 limbs x 64 threads = 33 KB of static shared memory

// Leaf j covers terms (a + j*LEAF_TERMS, min(b, a + (j+1)*LEAF_TERMS)]:
// P = 1, Q = a0+1 for the first term, then P = P*k + 1, Q = Q*k for each
// further k (P(a,k+1) = P(a,k)*Q(k,k+1) + P(k,k+1)).  Limbs live in shared
// memory, limb i of thread t at i*LEAF_NT + t (no bank conflicts); outputs
// go to out + (2j)*LEAF_STRIDE (P) and out + (2j+1)*LEAF_STRIDE (Q), lengths
// to len[2j], len[2j+1].
__global__ void __launch_bounds__(LEAF_NT) k_bsr_leaves(uint32_t a, uint32_t b, uint32_t nleaf, uint32_t *out,
                                                        uint32_t *len) {
  __shared__ uint32_t sP[LEAF_STRIDE * LEAF_NT], sQ[LEAF_STRIDE * LEAF_NT];
  const int t = threadIdx.x;
  const uint32_t j = blockIdx.x * LEAF_NT + t;
  if (j >= nleaf) return;
  const uint32_t a0 = a + j * (uint32_t)LEAF_TERMS;
  const uint32_t b0 = min(b, a0 + (uint32_t)LEAF_TERMS);
  uint32_t *P = sP + t, *Q = sQ + t;  // element i at [i * LEAF_NT]
  int lp = 1, lq = 1;
  P[0] = 1;
  Q[0] = a0 + 1;
  for (uint32_t k = a0 + 2; k <= b0; k++) {
    unsigned long long c = 1;  // P*k + 1
    for (int i = 0; i < lp; i++) {
      const unsigned long long v = (unsigned long long)P[i * LEAF_NT] * k + c;
      P[i * LEAF_NT] = (uint32_t)v;
      c = v >> 32;
    }
    if (c) P[(lp++) * LEAF_NT] = (uint32_t)c;
    c = 0;  // Q*k
    for (int i = 0; i < lq; i++) {
      const unsigned long long v = (unsigned long long)Q[i * LEAF_NT] * k + c;
      Q[i * LEAF_NT] = (uint32_t)v;
      c = v >> 32;
    }
    if (c) Q[(lq++) * LEAF_NT] = (uint32_t)c;
  }
  uint32_t *oP = out + (size_t)(2 * j) * LEAF_STRIDE, *oQ = oP + LEAF_STRIDE;
  for (int i = 0; i < lp; i++) oP[i] = P[i * LEAF_NT];
  for (int i = 0; i < lq; i++) oQ[i] = Q[i * LEAF_NT];
  len[2 * j] = (uint32_t)lp;
  len[2 * j + 1] = (uint32_t)lq;
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
