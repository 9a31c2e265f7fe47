/* newton.c — reciprocal and division by Newton's iteration.
 *
 * Same iteration as the reference (bigfloat/rcp.c:15-101, bigfloat/div.c:14-27)
 * so every intermediate value, and therefore e's digits, is the same:
 *   r <- r - (r*x - 1)*r, precision p -> p/2+1 per level (1 -> 0, 2 -> 1);
 *   at p == 0 a two-limb seed from a double built from the top three limbs
 *   (the reference scales by UINT32_MAX, not 2^32; kept, the iteration
 *   corrects it).
 * Each level's two products depend on each other, so they are single GPU
 * products; the large ones are where one-product latency matters.
 */
#include <stdio.h>
#include <stdlib.h>

#include "bc_host.h"
#include "bigfloat.h"

static void seed(bigfloat_t t, const bigfloat_t a) {
  int64_t e = a->exp;
  size_t L = a->len;
  const uint32_t *T = a->coef;
  if (L > 3) {
    size_t chop = L - 3;
    L = 3;
    e += (int64_t)chop;
    T += chop;
  }
  double v = T[0];
  if (L >= 2) v += (double)T[1] * (double)UINT32_MAX;
  if (L >= 3) v += (double)T[2] * (double)UINT32_MAX * (double)UINT32_MAX;
  v = 1. / v;
  e = -e;
  while (v < (double)UINT32_MAX) {
    v *= (double)UINT32_MAX;
    e--;
  }
  uint64_t v64 = (uint64_t)v;
  bigfloat_alloc(t, 2);
  t->sign = a->sign;
  t->coef[0] = (uint32_t)(v64 % UINT32_MAX);
  t->coef[1] = (uint32_t)(v64 / UINT32_MAX);
  t->exp = e;
}

void bigfloat_rcp(bigfloat_t t, const bigfloat_t a, size_t p) {
  if (a->len == 0) {
    fprintf(stderr, "Divide by Zero\n");
    abort();
  }
  if (p == 0) {
    seed(t, a);
    return;
  }
  size_t s = p / 2 + 1;
  if (p == 1) s = 0;
  if (p == 2) s = 1;
  bigfloat_t r, one, ax, err, corr;
  bigfloat_new(r);
  bigfloat_new(one);
  bigfloat_new(ax);
  bigfloat_new(err);
  bigfloat_new(corr);
  bigfloat_rcp(r, a, s);
  bigfloat_set(one, 1);
  bigfloat_mul(ax, a, r, p);       /* r*x */
  bigfloat_sub(err, ax, one, p);   /* r*x - 1 */
  bigfloat_mul(corr, err, r, p);   /* (r*x - 1)*r */
  bigfloat_sub(t, r, corr, p);     /* r - (r*x - 1)*r */
  bigfloat_free(r);
  bigfloat_free(one);
  bigfloat_free(ax);
  bigfloat_free(err);
  bigfloat_free(corr);
}

void bigfloat_div(bigfloat_t t, const bigfloat_t a, const bigfloat_t b, size_t p) {
  bigfloat_t r;
  bigfloat_new(r);
  if (p == 0) p = a->len + b->len;
  bigfloat_rcp(r, b, p);
  bigfloat_mul(t, a, r, p);
  bigfloat_free(r);
}
