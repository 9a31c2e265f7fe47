// bc_school.cuh — many small exact products at once, schoolbook, one warp
// per product.
//
// The reference multiplies operands below its FFT threshold on the CPU with
// a basecase / Karatsuba product (bigfloat/mul.c:176-553, used below 100
// output limbs, mul.c:640-648).  A batch of such products (the lower levels
// of a level-ordered splitting tree or conversion tree hold thousands) is
// done here in integers, with no rounding to check:
//   1. the warp copies A and B (at most SCHOOL_MAX limbs each) into its
//      shared memory;
//   2. lane l forms the column sums S_k = sum_{i+j=k} A_i B_j for the
//      columns k = l, l+32, ... < CL as a 64-bit low part and a 32-bit high
//      part (at most SCHOOL_MAX products of < 2^64 each: S_k < 2^72);
//   3. lane 0 propagates the carries over the columns in order
//      (v = S_k + c, limb k = v mod 2^32, c = v >> 32 < 2^41) and the warp
//      stores the CL limbs (columns at and above AL + BL are zero).
#pragma once
#include <cstdint>

namespace bc {

constexpr int SCHOOL_MAX = 256;          // limbs per operand
constexpr int SCHOOL_CMAX = 2 * SCHOOL_MAX;  // output limbs
constexpr int SCHOOL_WARPS = 4;          // warps (products in flight) per CTA

struct SchoolDesc {
  unsigned long long a, b, c;  // word offsets of A, B in the input span and of C in the output span
  uint32_t AL, BL, CL;
  uint32_t pad;
};

__global__ void __launch_bounds__(32 * SCHOOL_WARPS) k_school(const SchoolDesc *__restrict__ d, unsigned n,
                                                              const uint32_t *__restrict__ in,
                                                              uint32_t *__restrict__ out) {
  __shared__ uint32_t sa[SCHOOL_WARPS][SCHOOL_MAX], sb[SCHOOL_WARPS][SCHOOL_MAX];
  __shared__ unsigned long long slo[SCHOOL_WARPS][SCHOOL_CMAX];
  __shared__ uint32_t shi[SCHOOL_WARPS][SCHOOL_CMAX];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned nw = gridDim.x * SCHOOL_WARPS;
  for (unsigned item = blockIdx.x * SCHOOL_WARPS + w; item < n; item += nw) {
    const SchoolDesc q = d[item];
    const int AL = (int)q.AL, BL = (int)q.BL, CL = (int)q.CL;
    for (int i = lane; i < AL; i += 32) sa[w][i] = in[q.a + i];
    for (int i = lane; i < BL; i += 32) sb[w][i] = in[q.b + i];
    __syncwarp();
    const int top = AL + BL - 1;  // columns 0 .. top-1 can be nonzero
    for (int k = lane; k < CL; k += 32) {
      unsigned long long lo = 0;
      uint32_t hi = 0;
      if (k < top) {
        const int i0 = k - (BL - 1) > 0 ? k - (BL - 1) : 0, i1 = k < AL - 1 ? k : AL - 1;
        for (int i = i0; i <= i1; i++) {
          const unsigned long long p = (unsigned long long)sa[w][i] * sb[w][k - i];
          lo += p;
          hi += lo < p ? 1u : 0u;
        }
      }
      slo[w][k] = lo;
      shi[w][k] = hi;
    }
    __syncwarp();
    if (lane == 0) {
      unsigned long long c = 0;  // carry into column k, below 2^41
      for (int k = 0; k < CL; k++) {
        const unsigned long long lo = slo[w][k] + c;
        const unsigned long long hi = (unsigned long long)shi[w][k] + (lo < c ? 1ull : 0ull);
        shi[w][k] = (uint32_t)lo;  // the limb, in place
        c = (lo >> 32) | (hi << 32);
      }
    }
    __syncwarp();
    for (int k = lane; k < CL; k += 32) out[q.c + k] = shi[w][k];
    __syncwarp();  // this warp's shared arrays are reused by its next product
  }
}

}  // namespace bc
