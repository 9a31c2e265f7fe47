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
// One warp per leaf: lane l holds limbs [l*RS, (l+1)*RS) in registers, each
// lane multiplies its limbs with a local carry chain, and the carry out of a
// lane enters the next lane (a carry of that carry past a full lane is
// astronomically rare and handled by a bounded ripple).
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
    // coalesced load into shared memory (one pad word per 32), then each
    // lane takes its RS consecutive limbs
    for (uint32_t j = lane; j < (uint32_t)RADIX_WINDOW; j += 32) sm[j + (j >> 5)] = j < lf.len ? lf.y[j] : 0u;
    __syncwarp();
    uint32_t x[RS];
#pragma unroll
    for (int q = 0; q < RS; q++) {
      const int j = lane * RS + q;
      x[q] = sm[j + (j >> 5)];
    }
    __syncwarp();
    const uint32_t j0 = (uint32_t)lane * RS;  // this lane's first limb
    const uint32_t owner = lf.n / RS, slot = lf.n % RS;
    for (uint32_t i = 1; i <= lf.k; i++) {
      const uint32_t lo = i == 1 ? 0u : (uint32_t)floor(alpha * (double)(i - 1));
      const uint32_t hi = i == 1 ? L : lf.n + 1;
      // multiply the window by 10^9 (its top limb enters as zero)
      uint32_t c = 0;
#pragma unroll
      for (int q = 0; q < RS; q++) {
        const uint32_t j = j0 + q;
        if (j >= lo && j < hi) {
          const uint32_t xin = j == hi - 1 ? 0u : x[q];
          const unsigned long long v = (unsigned long long)xin * DEC_BASE + c;
          x[q] = (uint32_t)v;
          c = (uint32_t)(v >> 32);
        }
      }
      // the window's top lane drops its carry; the others pass it up
      const bool top_lane = hi - 1 >= j0 && hi - 1 < j0 + RS;
      const bool above = j0 >= hi;
      uint32_t out = (top_lane || above) ? 0u : c;
      uint32_t cin = __shfl_up_sync(~0u, out, 1);
      if (lane == 0) cin = 0;
      // add the carry in at the lane's lowest window limb; a carry out of the
      // lane ripples to the next lane (bounded: at most 32 rounds)
      for (int round = 0; round < 32; round++) {
        uint32_t t = cin;
#pragma unroll
        for (int q = 0; q < RS; q++) {
          const uint32_t j = j0 + q;
          if (t && j >= lo && j < hi) {
            const unsigned long long v = (unsigned long long)x[q] + t;
            x[q] = (uint32_t)v;
            t = (uint32_t)(v >> 32);
          }
        }
        const uint32_t ov = (top_lane || above) ? 0u : t;
        if (!__any_sync(~0u, ov != 0)) break;
        cin = __shfl_up_sync(~0u, ov, 1);
        if (lane == 0) cin = 0;
      }
      // the digit: limb n
      uint32_t dgt = 0;
#pragma unroll
      for (int q = 0; q < RS; q++) dgt = (uint32_t)q == slot ? x[q] : dgt;
      dgt = __shfl_sync(~0u, dgt, (int)owner);
      if (lane == 0) lf.s[lf.k - i] = dgt;
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
