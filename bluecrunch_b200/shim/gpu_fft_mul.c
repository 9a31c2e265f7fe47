/* gpu_fft_mul.c — the reference-side binding of the B200 multiply.
 *
 * A bluecrunch build that keeps its own host code (bigfloat/*.c, main.c,
 * util/) adds this one file and links libbcgpu.so: this definition of
 * _fft_mul (include/mul.h:3) replaces the CPU one of bigfloat/mul.c:108-174.
 * Same contract: exactly CL limbs of A*B mod 2^(32 CL), CT may alias AT or
 * BT, returns the digit width; a failure aborts with a message, as the
 * reference aborts on widths it cannot pack (fft/convert.c:66-68).
 *
 * The engine is initialised on the first call (once, thread-safe: the
 * reference calls _fft_mul from Cilk-spawned branches, main.c:86-89 and
 * bigfloat/radix.c:268-271); bc_gpu_mul itself serialises callers.
 * oracle/Makefile's gpu-relink target builds the reference's CLI this way
 * (the reference's mul.o keeps its _fft_mul as a weak symbol).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bc_gpu.h"

static pthread_once_t engine_once = PTHREAD_ONCE_INIT;
static int engine_status = BC_ERR_NOT_INIT;

static void engine_start(void) {
  engine_status = bc_gpu_init(NULL); /* $BC_TUNE_FILE selects the width table */
}

int _fft_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  pthread_once(&engine_once, engine_start);
  if (engine_status != BC_OK) {
    fprintf(stderr, "_fft_mul: bc_gpu_init: %s\n", bc_gpu_strerror(engine_status));
    abort();
  }
  bc_mul_stats st;
  const int rc = bc_gpu_mul(CT, CL, AT, AL, BT, BL, &st);
  if (rc != BC_OK) {
    fprintf(stderr, "_fft_mul: %s\n", bc_gpu_strerror(rc));
    abort();
  }
  return st.width;
}
