/* newton.c — reciprocal and division by Newton's iteration.
 *
 * Same iteration as the reference (bigfloat/rcp.c:15-101, bigfloat/div.c:14-27)
 * so every intermediate value, and therefore e's digits, is the same:
 *   r <- r - (r*x - 1)*r, precision p -> p/2+1 per level (1 -> 0, 2 -> 1);
 *   at p == 0 a two-limb seed from a double built from the top three limbs
 *   (the reference scales by UINT32_MAX, not 2^32; kept, the iteration
 *   corrects it).
 * Each level's two products depend on each other, so they are single
 * products.  Levels below 2^16 limbs run here (each product one GPU call, or
 * the host's exact schoolbook below 100 limbs); from 2^16 limbs up, the
 * levels and the quotient run in device memory (bc_gpu_newton) with the same
 * semantics for every product, sum and difference, so only the operands and
 * the result cross the bus.
 */
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "bc_gpu.h"
#include "bc_host.h"
#include "bigfloat.h"

/* $BC_STATS: per-level times of the large levels (products and subtractions). */
static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

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

/* Precision of the level below p (bigfloat/rcp.c:73-80). */
static size_t rcp_inner(size_t p) { return p == 1 ? 0 : (p == 2 ? 1 : p / 2 + 1); }

/* Levels of BC_DEVICE_NEWTON limbs and more run in device memory
 * (bc_gpu_newton): the host computes the reciprocal at the first level below
 * that, the device the levels above it and, for a division, the quotient.
 * $BC_NEWTON_HOST keeps every level on the host.  Returns 1 when done. */
#define BC_DEVICE_NEWTON ((size_t)1 << 16)
static int newton_device(bigfloat_t t, const bigfloat_t num, const bigfloat_t den, size_t p, size_t pdiv) {
  if (p < BC_DEVICE_NEWTON || getenv("BC_NEWTON_HOST")) return 0;
  size_t lv[64];
  int n = 0;
  size_t q = p;
  while (q >= BC_DEVICE_NEWTON && n < 64) {
    lv[n++] = q;
    q = rcp_inner(q);
  }
  /* lv[0] = p > lv[1] > ... > lv[n-1] >= BC_DEVICE_NEWTON > q */
  bigfloat_t r0;
  bigfloat_new(r0);
  bigfloat_rcp(r0, den, q);
  size_t up[64];
  for (int k = 0; k < n; k++) up[k] = lv[n - 1 - k];
  bc_bignum d = {den->coef, den->len, den->exp, den->sign}, r = {r0->coef, r0->len, r0->exp, r0->sign};
  bc_bignum a = {num ? num->coef : NULL, num ? num->len : 0, num ? num->exp : 0, num ? num->sign : 1};
  bc_bignum_out out;
  bc_host_ensure_gpu();
  const int rc = bc_gpu_newton(&d, &r, up, n, num ? &a : NULL, pdiv, &out);
  bigfloat_free(r0);
  if (rc != BC_OK) {
    fprintf(stderr, "bluecrunch: Newton iteration on the GPU failed: %s\n", bc_gpu_strerror(rc));
    abort();
  }
  free(t->coef);
  t->coef = out.coef;
  t->len = out.len;
  t->exp = out.exp;
  t->sign = out.sign;
  return 1;
}

void bigfloat_rcp(bigfloat_t t, const bigfloat_t a, size_t p) {
  if (a->len == 0) {
    fprintf(stderr, "Divide by Zero\n");
    abort();
  }
  if (newton_device(t, NULL, a, p, 0)) return;
  if (p == 0) {
    seed(t, a);
    return;
  }
  const size_t s = rcp_inner(p);
  bigfloat_t r, one, ax, err, corr;
  bigfloat_new(r);
  bigfloat_new(one);
  bigfloat_new(ax);
  bigfloat_new(err);
  bigfloat_new(corr);
  bigfloat_rcp(r, a, s);
  bigfloat_set(one, 1);
  const int stats = p >= 1000000 && getenv("BC_STATS") != NULL;
  double t0 = stats ? now_s() : 0, t1 = 0, t2 = 0, t3 = 0;
  bigfloat_mul(ax, a, r, p);       /* r*x */
  if (stats) t1 = now_s();
  bigfloat_sub(err, ax, one, p);   /* r*x - 1 */
  if (stats) t2 = now_s();
  bigfloat_mul(corr, err, r, p);   /* (r*x - 1)*r */
  if (stats) t3 = now_s();
  bigfloat_sub(t, r, corr, p);     /* r - (r*x - 1)*r */
  if (stats)
    printf("    rcp level p=%zu: r*x %.3f s (%zu x %zu limbs), -1 %.3f s, *r %.3f s (%zu x %zu), r-corr %.3f s\n", p,
           t1 - t0, a->len, r->len, t2 - t1, t3 - t2, err->len, r->len, now_s() - t3);
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
  if (b->len && newton_device(t, a, b, p, p)) {
    bigfloat_free(r);
    return;
  }
  bigfloat_rcp(r, b, p);
  const double t0 = now_s();
  bigfloat_mul(t, a, r, p);
  if (p >= 1000000 && getenv("BC_STATS")) printf("    div: a*rcp %.3f s\n", now_s() - t0);
  bigfloat_free(r);
}
