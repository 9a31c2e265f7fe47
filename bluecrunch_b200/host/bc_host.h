/* bc_host.h — internal declarations shared by the host C sources. */
#ifndef BC_HOST_H
#define BC_HOST_H
#include <stddef.h>
#include <stdint.h>

#include "bigfloat.h"

/* Below this many output limbs a product stays on the host, as the
 * reference's bigfloat_mul dispatch does (KARATZUBA_THRESH,
 * bigfloat/mul.c:14,645-648). */
#define BC_SMALL_PRODUCT_LIMBS 100

typedef struct {
  const uint32_t *T;
  size_t L;
  int64_t exp;
} bc_operand;

typedef struct {
  uint32_t *C;
  size_t CL;
  const uint32_t *A;
  size_t AL;
  const uint32_t *B;
  size_t BL;
} bc_gpu_item;

void *bc_xmalloc(size_t n);
/* memcpy / memset to zero, split over the OpenMP threads when large. */
void bc_par_memcpy(void *dst, const void *src, size_t n);
void bc_par_memzero(void *dst, size_t n);
void *bc_xrealloc(void *p, size_t n);
void bc_mul_operands(const _bigfloat_struct *a, const _bigfloat_struct *b, size_t p, bc_operand *oa, bc_operand *ob);
/* Initialise the GPU engine once (aborts with a message if there is none). */
void bc_host_ensure_gpu(void);
/* All items on the GPU in one batch; aborts with a message on failure. */
void bc_host_gpu_batch(bc_gpu_item *items, size_t n);
/* The batch's small products on the GPU in one launch (no aliasing). */
void bc_host_gpu_small_batch(bc_gpu_item *items, size_t n);
/* Below this many small products a batch computes them on host threads. */
#ifndef BC_SMALL_GPU_MIN
#define BC_SMALL_GPU_MIN 256
#endif
/* Product of small operands on the host (schoolbook), CT may alias. */
void bc_small_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL, const uint32_t *BT, size_t BL);
/* The BC_VERIFY check: 0 when C = A*B modulo two 32-bit primes (or when
 * CL < AL+BL), else the prime that failed. */
uint64_t bc_host_product_check(const uint32_t *C, size_t CL, const uint32_t *A, size_t AL, const uint32_t *B,
                               size_t BL);

/* A binary-to-decimal conversion whose base-10^9 digits stay in device
 * memory (bigfloat_radix_device): dev holds limbs [0, len) or, when the top
 * limb was split, [0, len - 1) with the value's top limb in `top`;
 * value = sum limb[i] 10^(9(i + exp)). */
typedef struct {
  uint32_t *dev;
  size_t len;
  int64_t exp;
  uint32_t top;
} bc_dec_device;
int bigfloat_radix_device(bc_dec_device *d, const bigfloat_t a);
int bc_dec_device_write(const bc_dec_device *d, size_t digits, int fd);
void bc_dec_device_free(bc_dec_device *d);

#endif
