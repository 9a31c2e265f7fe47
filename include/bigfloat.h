/* bigfloat.h — arbitrary-precision float with base-2^32 limbs.
 *
 * Same type and prototypes as the reference's include/bigfloat.h:1-45 so that
 * callers written against it link unchanged.  value = +-sum coef[i] *
 * 2^(32*(i+exp)), little-endian limbs, len limbs in use.  Products of more
 * than two limbs go to the GPU through _fft_mul (include/mul.h) or, for whole
 * tree levels, bigfloat_mul_batch.
 */
#ifndef BIGFLOAT_H
#define BIGFLOAT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BIGFLOAT_EXTRA_PRECISION (2)

typedef struct {
  uint32_t *coef;  /* coefficients (limbs), little-endian */
  int64_t exp;     /* exponent in limbs */
  size_t len;      /* limbs in use */
  int sign;        /* 1: positive, 0: negative */
} _bigfloat_struct;

typedef _bigfloat_struct bigfloat_t[1];

/* management (reference bigfloat/{new,free,alloc,copy,set,zero}.c) */
void bigfloat_zero(bigfloat_t target);
int bigfloat_iszero(const bigfloat_t target);
void bigfloat_set(bigfloat_t target, uint32_t value);
void bigfloat_free(bigfloat_t target);
void bigfloat_new(bigfloat_t target);
void bigfloat_copy(bigfloat_t target, const bigfloat_t source);
void bigfloat_alloc(bigfloat_t target, size_t size);
void bigfloat_realloc(bigfloat_t target, size_t size);

/* arithmetic */
void bigfloat_neg(bigfloat_t target);
void bigfloat_floor(bigfloat_t target);
void bigfloat_add(bigfloat_t target, const bigfloat_t a, const bigfloat_t b, size_t p);
void bigfloat_sub(bigfloat_t target, const bigfloat_t a, const bigfloat_t b, size_t p);
void bigfloat_mul(bigfloat_t target, const bigfloat_t a, const bigfloat_t b, size_t p);
void bigfloat_mului(bigfloat_t a, uint32_t b);
void bigfloat_mulu(bigfloat_t target, const bigfloat_t a, uint32_t b);
void bigfloat_div(bigfloat_t target, const bigfloat_t a, const bigfloat_t b, size_t p);
void bigfloat_rcp(bigfloat_t target, const bigfloat_t a, size_t p);
void bigfloat_exp(bigfloat_t target, const bigfloat_t a, const uint64_t exp);
size_t bigfloat_radix_decimals(bigfloat_t target);

/* radix conversion 2^32 -> 10^9 */
void bigfloat_radix(bigfloat_t target, const bigfloat_t a);

/* output */
size_t bigfloat_to_string(char *string, const bigfloat_t value, size_t digits, int base);
void bigfloat_print(const char *name, const bigfloat_t value);
void bigfloat_print10(const char *name, const bigfloat_t value);

/* ---- additions of this implementation (no counterpart in the reference) */

/* One independent bigfloat_mul(t, a, b, p) per item, all products of the
 * batch in as few GPU launches as their transform shapes allow.  Results are
 * bit-identical to calling bigfloat_mul item by item.  Targets must be
 * distinct objects that alias no operand. */
typedef struct {
  _bigfloat_struct *target;
  const _bigfloat_struct *a;
  const _bigfloat_struct *b;
  size_t p;
} bigfloat_mul_item;
void bigfloat_mul_batch(bigfloat_mul_item *items, size_t n);

/* e to `digits` decimal digits; writes "2." + digits into e.txt and the hex
 * expansion into e-hex.txt in `outdir` (NULL = current directory).  mode 0:
 * the reference's recursive binary splitting, one product per GPU call;
 * mode 1: tree levels batched (bigfloat_mul_batch); mode 2: the whole tree
 * in device memory (bc_gpu_e_series). Returns 0 on success. */
int bluecrunch_e(size_t digits, int mode, const char *outdir);

/* Product counters since the last reset (for tests and benchmarks). */
typedef struct {
  size_t gpu_products, gpu_calls, small_products;
  double gpu_seconds;         /* wall time inside GPU calls (batch calls only for kernels) */
  double gpu_kernel_seconds;  /* GPU kernel time of the batch calls */
} bigfloat_mul_counters;
void bigfloat_get_counters(bigfloat_mul_counters *out);
void bigfloat_reset_counters(void);

#ifdef __cplusplus
}
#endif
#endif
