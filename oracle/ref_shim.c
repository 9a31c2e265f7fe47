/* Glue that lets the unmodified reference sources build and run here.
 * Test infrastructure: only tests/, smoke() and bench.py's CPU legs use it.
 *
 * 1. Cilk runtime queries (main.c:175-177, test/*.c) answered for the serial
 *    or OpenMP build.
 * 2. fft_forward: the reference's version (fft/fft.c:395-414) runs an
 *    unfinished Bailey four-step debug block for power-of-two lengths > 30
 *    (fft/fft.c:397-410) that prints the arrays and aborts on a 1e-15 assert.
 *    fft/fft.c is compiled with -Dfft_forward=bcref_unfinished_fft_forward so
 *    that definition is set aside, and this one keeps the rest of the
 *    function: cached-table path when the length has a table, uncached
 *    cos/sin path otherwise (fft/fft.c:411-413).
 * 3. bcref_main wraps the reference main() (compiled as bcref_main) in an
 *    OpenMP parallel region so spawned tasks have workers; bcref_fft_mul_par
 *    does the same for one _fft_mul call (bench CPU leg).
 */
#include <complex.h>
#include <stddef.h>
#include <stdint.h>
#ifdef BC_REF_OPENMP
#include <omp.h>
#endif

size_t table_select(size_t length);
extern int twiddle_table_size;
void _fft_forward(complex double *T, size_t length);
void _fft_forward_uncached(complex double *T, size_t length);
int _fft_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL);

int __cilkrts_get_nworkers(void) {
#ifdef BC_REF_OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int __cilkrts_set_param(const char *name, const char *value) {
  (void)name; (void)value;
  return 0;
}

void fft_forward(complex double *T, size_t length) {
  if (table_select(length) < (size_t)twiddle_table_size) {
    _fft_forward(T, length);
  } else {
    _fft_forward_uncached(T, length);
  }
}

int bcref_fft_mul_par(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  int r = 0;
#ifdef BC_REF_OPENMP
#pragma omp parallel
#pragma omp single
#endif
  r = _fft_mul(CT, CL, AT, AL, BT, BL);
  return r;
}

int bcref_threads(void) { return __cilkrts_get_nworkers(); }
