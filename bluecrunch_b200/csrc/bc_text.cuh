// bc_text.cuh — decimal text of base-10^9 limbs, rendered on the device.
//
// The reference prints a converted number limb by limb, most significant
// first, nine zero-padded decimal characters per limb (bigfloat/string.c:
// 93-111, through its limb formatter string.c:15-37).  Here one CTA renders
// TEXT_LIMBS consecutive output limbs: each thread writes its limbs' nine
// characters into shared memory, then the CTA stores the block's
// 9 * TEXT_LIMBS bytes as 16-byte words (9 * TEXT_LIMBS is a multiple of 16,
// so every block starts on a 16-byte boundary of the text).  The last,
// partial block stores bytes.
#pragma once
#include <cstdint>

namespace bc {

constexpr int TEXT_THREADS = 256;
constexpr int TEXT_LIMBS = 1024;  // per CTA; 9216 bytes of text
static_assert((9 * TEXT_LIMBS) % 16 == 0, "text blocks start on 16-byte boundaries");

// Output limb k (k = 0 .. n-1) is limbs[top - k]; its text is
// text[9k .. 9k + 8].  Each limb is below 10^9.
__global__ void __launch_bounds__(TEXT_THREADS) k_decimal_text(const uint32_t *__restrict__ limbs,
                                                               unsigned long long top, unsigned long long n,
                                                               char *__restrict__ text) {
  __shared__ __align__(16) char sm[9 * TEXT_LIMBS];
  const unsigned long long k0 = (unsigned long long)blockIdx.x * TEXT_LIMBS;
  if (k0 >= n) return;
  const int cnt = n - k0 < (unsigned long long)TEXT_LIMBS ? (int)(n - k0) : TEXT_LIMBS;
  for (int i = threadIdx.x; i < cnt; i += TEXT_THREADS) {
    uint32_t v = __ldg(&limbs[top - (k0 + (unsigned long long)i)]);
    char *s = sm + 9 * i;
#pragma unroll
    for (int d = 8; d >= 0; d--) {
      const uint32_t q = v / 10u;
      s[d] = (char)('0' + (v - 10u * q));
      v = q;
    }
  }
  __syncthreads();
  char *dst = text + 9 * k0;
  const int bytes = 9 * cnt;
  if (cnt == TEXT_LIMBS) {
    const uint4 *src4 = reinterpret_cast<const uint4 *>(sm);
    uint4 *dst4 = reinterpret_cast<uint4 *>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += TEXT_THREADS) dst4[i] = src4[i];
  } else {
    for (int i = threadIdx.x; i < bytes; i += TEXT_THREADS) dst[i] = sm[i];
  }
}

}  // namespace bc
