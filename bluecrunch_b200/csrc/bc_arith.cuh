// bc_arith.cuh — sums, differences and comparisons of bigfloats held in
// device memory, for the Newton iteration of the reciprocal kept on the GPU.
//
// A windowed operand contributes its limbs to output limbs [lo, hi) of the
// result window (limb i of the result is x[i - lo] there, zero elsewhere), as
// the reference's _bigfloat_uadd / _bigfloat_usub read their operands through
// _bigfloat_word_at over the window [bot, top) (bigfloat/addsub.c:17-27,
// 65-181).  The carry (borrow) chain is resolved like the carry of k_add:
// each thread's limbs map a carry in of 0 or 1 to a carry out, a CTA scans the
// maps, and tiles chain by decoupled lookback with bounded waits.
#pragma once
#include <cuda/atomic>

#include "bc_bsr.cuh"

namespace bc {

struct WinOp {
  const uint32_t *x;
  long long lo, hi;  // output limbs [max(lo, 0), hi) read x[i - lo]
};

__device__ __forceinline__ uint32_t win_at(const WinOp &o, long long i) {
  return (i >= o.lo && i < o.hi) ? o.x[i - o.lo] : 0u;
}

struct AddSubParams {
  WinOp a, b;
  uint32_t *r;               // n limbs
  unsigned long long n;
  int sub;                   // 1: a - b (|a| >= |b| over the window), 0: a + b
  unsigned long long tiles;  // ceil(n / ADD_TILE)
  unsigned int *counter;     // zeroed before launch
  uint32_t *status;          // one word per tile, zeroed before launch
  unsigned int *cout;        // carry (borrow) out of limb n - 1
  unsigned int *flags;       // bit 0: a lookback wait ran out
};

__global__ void __launch_bounds__(ADD_NT) k_addsub_win(AddSubParams p) {
  __shared__ uint32_t sw[65];
  __shared__ unsigned long long s_unit;
  __shared__ int s_cin;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(p.counter, 1u);
    __syncthreads();
    const unsigned long long tile = s_unit;
    if (tile >= p.tiles) break;
    const long long i0 = (long long)(tile * ADD_TILE) + (long long)tid * ADD_PT;
    uint32_t s[ADD_PT];
    unsigned c = 0;
    bool run = true;  // add: all limbs 0xffffffff; sub: all limbs 0 (a carry in passes through)
#pragma unroll
    for (int q = 0; q < ADD_PT; q++) {
      const long long i = i0 + q;
      const uint32_t av = win_at(p.a, i), bv = win_at(p.b, i);
      if (p.sub) {
        const unsigned long long v = (unsigned long long)av - bv - c;
        s[q] = (uint32_t)v;
        c = (unsigned)((v >> 32) & 1u);
        if (i < (long long)p.n) run = run && s[q] == 0u;
      } else {
        const unsigned long long v = (unsigned long long)av + bv + c;
        s[q] = (uint32_t)v;
        c = (unsigned)(v >> 32);
        if (i < (long long)p.n) run = run && s[q] == 0xffffffffu;
      }
    }
    const int c0 = (int)c, c1 = (int)(c | (run ? 1u : 0u));
    uint32_t agg;
    const uint32_t ex = block_scan_fn<ADD_NT>(fn_make(c0, c0, c1), sw, &agg);
    if (tid == 0) {
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> me(p.status[tile]);
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
          cuda::atomic_ref<uint32_t, cuda::thread_scope_device> st(p.status[prev]);
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
    unsigned cc = (unsigned)fn_apply(ex, s_cin);  // carry (borrow) into this thread's limbs
#pragma unroll
    for (int q = 0; q < ADD_PT; q++) {
      const long long i = i0 + q;
      unsigned long long v;
      if (p.sub) {
        v = (unsigned long long)s[q] - cc;
        cc = (unsigned)((v >> 32) & 1u);
      } else {
        v = (unsigned long long)s[q] + cc;
        cc = (unsigned)(v >> 32);
      }
      if (i < (long long)p.n) p.r[i] = (uint32_t)v;
      if (i + 1 == (long long)p.n) *p.cout = cc;
    }
    __syncthreads();
  }
}

// *top = 1 + the highest i < n with x[i] != 0 (0 if none); *top zeroed
// before launch.
__global__ void k_top_nonzero(const uint32_t *x, unsigned long long n, unsigned long long *top) {
  unsigned long long best = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    if (x[i]) best = i + 1;
  for (int o = 16; o; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(~0u, best, o);
    best = t > best ? t : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(top, best);
}

// *hi = 1 + the highest i < n where the windowed operands differ (0 if
// they are equal over the window); *hi zeroed before launch.
__global__ void k_first_diff(WinOp a, WinOp b, unsigned long long n, unsigned long long *hi) {
  unsigned long long best = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    if (win_at(a, (long long)i) != win_at(b, (long long)i)) best = i + 1;
  for (int o = 16; o; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(~0u, best, o);
    best = t > best ? t : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(hi, best);
}

}  // namespace bc
