/* bc_oracle — CPU restatement of the reference's FFT multiply path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (bluecrunch_b200/) links,
 * loads or calls this library; only tests/, __graft_entry__.smoke() and the
 * CPU baseline leg of bench.py use it, and only as the checker.
 *
 * Each function cites the reference file:line it restates.  Pinned against
 * the reference's own known-answer tests (test/test_fft.c, test_int_to_fft.c,
 * test_fft_to_int.c, test_conversion.c) and against the compiled reference
 * (oracle/_ref) by tests/test_oracle.py.
 */
#ifndef BC_ORACLE_H
#define BC_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

/* bits per point from CL (bigfloat/mul.c:109-124); extended below 7 bits. */
int    bco_width(size_t CL);
/* smallest 2*2^k or 3*2^k >= n (fft/fft.c:22-41). */
size_t bco_fft_length(size_t n);

/* int_to_fft: bit-slice AL words into b-bit real parts, zero-pad to length
 * (fft/convert.c:45-80 with the generated int_to_fft{b}, gen.rb:111-160).
 * Returns the number of points written, ceil(32*AL/b). */
size_t bco_int_to_fft(double complex *V, size_t length, const uint32_t *A, size_t AL, int b);
/* fft_to_int: scale by 1/length, round with (uint64_t)(f+0.5), 64-bit carry,
 * emit b bits per point, stop after exactly AL words
 * (fft/convert.c:83-111 with fft_to_int{b}, gen.rb:162-208). */
void   bco_fft_to_int(const double complex *T, size_t length, uint32_t *A, size_t AL, int b);

/* Forward DIF transform, X_k = sum x_n e^{+2 pi i nk/N}, digit-reversed output
 * (fft/fft.c:43-96).  Inverse DIT from digit-reversed input, unscaled
 * (fft/fft.c:289-329).  N = 2^k or 3*2^k. */
void   bco_fft_forward(double complex *T, size_t n);
void   bco_fft_inverse(double complex *T, size_t n);
/* a[i] <- a[i]*b[i] (fft/pointwise.c:9-20). */
void   bco_pointwise(double complex *a, const double complex *b, size_t n);

/* The whole multiply: C = A*B mod 2^(32*CL) (bigfloat/mul.c:108-174).
 * Returns the width used.  Widths below 7 (CL > 4e6) are the documented
 * extension; the reference aborts there. */
int    bco_fft_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                   const uint32_t *BT, size_t BL);
/* Same, with the width forced (for error sweeps); returns max |x-round(x)|. */
double bco_fft_mul_width(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                         const uint32_t *BT, size_t BL, int b);

/* Exact schoolbook product, low CL words (bigfloat/mul.c:176-220). */
void   bco_basecase_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                        const uint32_t *BT, size_t BL);

/* Exact FP64-free product through a number-theoretic transform over the
 * prime 2^64-2^32+1 with 16-bit digits (own method; exact for
 * AL+BL <= 2^30 words).  Low CL words.  Returns 0, or -1 if too large. */
int    bco_ntt_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                   const uint32_t *BT, size_t BL);

/* A mod p for A = sum AT[i] 2^(32 i); p = 0x9f063b05 is the reference's
 * CHECKPRIME (bigfloat/mul.c:19-34); any prime < 2^32 works. */
uint32_t bco_checksum(const uint32_t *AT, size_t AL, uint32_t p);
/* 1 if C == A*B holds modulo each of nprimes built-in primes, else 0. */
int    bco_modcheck(const uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                    const uint32_t *BT, size_t BL, int nprimes);

#ifdef __cplusplus
}
#endif
#endif
