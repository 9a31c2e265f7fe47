// bc_radix.cuh — leaves of the binary-to-decimal conversion on the GPU.
//
// A leaf turns a fraction y (len limbs below the point, base 2^32) into k
// base-10^9 digits by k rounds of "multiply by 10^9, take the limb that
// crosses the point", on a window of limbs that drops the low limbs which can
// no longer reach the digit (the reference's convert_trunc,
// bigfloat/radix.c:41-91).  In absolute limb positions (limb len is an extra
// zero), round i works on [lo_i, hi_i): lo_1 = 0, hi_1 = len + 1, and
// lo_i = floor(alpha*(i-1)), hi_i = n + 1 for i >= 2, with alpha =
// log(10^9)/log(2^32) as the caller computes it.  Before the multiply the
// window's top limb is zero; the carry out of the window is dropped; the
// digit is limb n after the multiply and lands in s[k - i].
//
// One warp per leaf, RS limbs per lane in registers, laid out so that limb n
// is the last limb of lane 31 (lane l holds limbs base + l*RS ... base +
// (l+1)*RS - 1, base = n + 1 - 32*RS): the digit is then one fixed register,
// and the window's top limb, which enters each round after the first as
// zero, is that same register.  Limbs above n are not held: carries only move
// up, so they never reach limb n (in the first round the window reaches limb
// len >= n, but what it computes above n is dropped with the carry out).
// Each lane multiplies its limbs with a local carry chain; the carry out of a
// lane enters the next lane's lowest limb, and a carry out of that limb
// (astronomically rare) ripples further by a bounded loop.
#pragma once
#include <cstdint>

namespace bc {

constexpr int RS = 32;                   // limbs per lane
constexpr int RADIX_WINDOW = 32 * RS;    // limbs a leaf window may span
constexpr int RADIX_WARPS = 4;           // warps per CTA
constexpr uint32_t DEC_BASE = 1000000000u;

struct RadixLeaf {
  const uint32_t *y;   // device: len limbs of the fraction
  uint32_t *s;         // device: k digits
  uint32_t len, n, k, pad;
};

__global__ void __launch_bounds__(32 * RADIX_WARPS) k_radix_leaves(const RadixLeaf *leaves, int count, double alpha,
                                                                 unsigned *flags) {
  __shared__ uint32_t stage[RADIX_WARPS][RADIX_WINDOW + RADIX_WINDOW / 32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t *sm = stage[wib];
  const int warps = gridDim.x * RADIX_WARPS;
  for (int li = blockIdx.x * RADIX_WARPS + wib; li < count; li += warps) {
    const RadixLeaf lf = leaves[li];
    const uint32_t L = lf.len + 1;
    if (L > (uint32_t)RADIX_WINDOW || lf.n + 1 > (uint32_t)RADIX_WINDOW || lf.n + 1 > L + 1) {
      if (lane == 0) atomicOr(flags, 1u);
      continue;
    }
    // limb j sits at index j - base (base = n + 1 - RADIX_WINDOW <= 0): a
    // coalesced load into shared memory (one pad word per 32), then each lane
    // takes its RS consecutive indices
    const int base = (int)lf.n + 1 - RADIX_WINDOW;
    for (int t = lane; t < RADIX_WINDOW; t += 32) {
      const int j = t + base;
      sm[t + (t >> 5)] = (j >= 0 && j < (int)lf.len) ? lf.y[j] : 0u;
    }
    __syncwarp();
    uint32_t x[RS];
#pragma unroll
    for (int q = 0; q < RS; q++) {
      const int t = lane * RS + q;
      x[q] = sm[t + (t >> 5)];
    }
    __syncwarp();
    const int j0 = lane * RS + base;  // limb of x[0]
    for (uint32_t i = 1; i <= lf.k; i++) {
      const int lo = i == 1 ? 0 : (int)floor(alpha * (double)(i - 1));
      // rounds after the first: the window's top limb (limb n, the last
      // digit) enters as zero
      if (i > 1 && lane == 31) x[RS - 1] = 0;
      // multiply the window [lo, n] by 10^9
      uint32_t c = 0;
#pragma unroll
      for (int q = 0; q < RS; q++) {
        if (j0 + q >= lo) {
          const unsigned long long v = (unsigned long long)x[q] * DEC_BASE + c;
          x[q] = (uint32_t)v;
          c = (uint32_t)(v >> 32);
        }
      }
      // the carry out of lane l enters lane l+1 at its lowest limb, which is
      // inside the window whenever the carry is nonzero; lane 31's is dropped
      uint32_t cin = __shfl_up_sync(~0u, c, 1);
      if (lane == 0) cin = 0;
      {
        const unsigned long long v = (unsigned long long)x[0] + cin;
        x[0] = (uint32_t)v;
        uint32_t t = (uint32_t)(v >> 32);
        // rare: the lowest limb overflowed; ripple through the lane and on
        // into the next lanes (bounded: at most 32 rounds)
        for (int round = 0; round < 32 && __any_sync(~0u, t != 0); round++) {
#pragma unroll
          for (int q = 1; q < RS; q++) {
            const unsigned long long w = (unsigned long long)x[q] + t;
            x[q] = (uint32_t)w;
            t = (uint32_t)(w >> 32);
          }
          uint32_t up = __shfl_up_sync(~0u, t, 1);
          if (lane == 0) up = 0;
          const unsigned long long w = (unsigned long long)x[0] + up;
          x[0] = (uint32_t)w;
          t = (uint32_t)(w >> 32);
        }
      }
      // the digit: limb n, the last register of lane 31
      if (lane == 31) lf.s[lf.k - i] = x[RS - 1];
    }
  }
}

// ------------------------------------------------------------------ merges
// An internal node's digits from its children's (the reference's merge,
// bigfloat/radix.c:277-316): if the high part's lowest digit is 10^9 - 1 and
// the low part's top digit is 0, add 1 to the high part (base 10^9, carry
// past its top dropped); then the low kl digits are the low part's, or zero
// when the high part's lowest digit is 0 and the low part's top digit is
// 10^9 - 1; above them come the high part's digits from its second on.  No
// other carry can arise: the sum in the reference adds the low part into
// zeros.
struct MergeDesc {
  uint32_t *sh;        // kh digits of the high child (fixed in place)
  const uint32_t *sl;  // kl digits of the low child
  uint32_t *s;         // kh - 1 + kl digits of the node
  unsigned long long kh, kl;
  unsigned long long off;  // first copy unit of this node (batch-wide numbering)
};

// One thread per node: the +1 fix-up and the low-part decision (flag[i]).
__global__ void k_merge_fix(MergeDesc *d, int n, unsigned *flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  MergeDesc m = d[i];
  if (m.sh[0] == DEC_BASE - 1 && m.sl[m.kl - 1] == 0) {
    unsigned long long carry = 1;
    for (unsigned long long q = 0; q < m.kh && carry; q++) {
      const unsigned long long v = (unsigned long long)m.sh[q] + carry;
      carry = v / DEC_BASE;
      m.sh[q] = (uint32_t)(v % DEC_BASE);
    }
  }
  flag[i] = (m.sh[0] == 0 && m.sl[m.kl - 1] == DEC_BASE - 1) ? 1u : 0u;
}

// The copies, MERGE_UNIT digits per unit, units of all nodes in one grid.
constexpr int MERGE_UNIT = 4096;
__global__ void k_merge_copy(const MergeDesc *d, int n, unsigned long long units, const unsigned *flag) {
  for (unsigned long long u = blockIdx.x; u < units; u += gridDim.x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (d[mid].off <= u) lo = mid; else hi = mid - 1;
    }
    const MergeDesc &m = d[lo];
    const bool zero_low = flag[lo] != 0;
    const unsigned long long len = m.kh - 1 + m.kl;
    const unsigned long long i0 = (u - m.off) * MERGE_UNIT;
    for (unsigned long long i = i0 + threadIdx.x; i < i0 + MERGE_UNIT && i < len; i += blockDim.x)
      m.s[i] = i < m.kl ? (zero_low ? 0u : m.sl[i]) : m.sh[i - m.kl + 1];
  }
}

}  // namespace bc
