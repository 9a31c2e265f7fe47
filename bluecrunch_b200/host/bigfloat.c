/* bigfloat.c — bigfloat_t management, addition, subtraction, multiply
 * dispatch and scalar multiplies.
 *
 * Values and lengths follow the reference bit for bit (every product is
 * exact, so e's digits depend only on these host-side rules):
 *   - precision p means p+2 limbs kept, low limbs chopped
 *     (bigfloat/addsub.c:83-86,140-143, bigfloat/mul.c:573-602);
 *   - a product has AL+BL limbs, then one top zero limb is trimmed and, above
 *     1000 limbs, all top zero limbs (bigfloat/mul.c:667-675);
 *   - subtraction strips top zero limbs (bigfloat/addsub.c:165-173).
 * Memory handling is this file's own: results are built in fresh buffers and
 * swapped in, so aliasing of target and operands is always safe.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bigfloat.h"
#include "bc_host.h"
#include "mul.h"

/* ---------------------------------------------------------------- lifecycle
 * bigfloat/new.c, free.c, alloc.c, copy.c, set.c, zero.c, neg.c, floor.c */

void bigfloat_new(bigfloat_t t) {
  t->sign = 1;
  t->exp = 0;
  t->len = 0;
  t->coef = NULL;
}

void bigfloat_free(bigfloat_t t) {
  free(t->coef);
  t->coef = NULL;
}

void bigfloat_alloc(bigfloat_t t, size_t size) {
  bigfloat_free(t);
  t->exp = 0;
  t->sign = 1;
  t->len = size;
  t->coef = (uint32_t *)bc_xmalloc(size * sizeof(uint32_t));
}

void bigfloat_realloc(bigfloat_t t, size_t size) {
  size_t old = t->len;
  t->coef = (uint32_t *)bc_xrealloc(t->coef, size * sizeof(uint32_t));
  t->len = size;
  if (size > old) memset(t->coef + old, 0, (size - old) * sizeof(uint32_t));
}

void bigfloat_copy(bigfloat_t t, const bigfloat_t s) {
  uint32_t *c = (uint32_t *)bc_xmalloc(s->len * sizeof(uint32_t));
  if (s->len) memcpy(c, s->coef, s->len * sizeof(uint32_t));
  free(t->coef);
  t->coef = c;
  t->exp = s->exp;
  t->sign = s->sign;
  t->len = s->len;
}

void bigfloat_zero(bigfloat_t t) {
  free(t->coef);
  t->coef = NULL;
  t->exp = 0;
  t->len = 0;
  t->sign = 1;
}

int bigfloat_iszero(const bigfloat_t t) { return t->len == 0; }

void bigfloat_set(bigfloat_t t, uint32_t value) {
  if (value == 0) {
    bigfloat_zero(t);
    return;
  }
  bigfloat_alloc(t, 1);
  t->coef[0] = value;
}

void bigfloat_neg(bigfloat_t t) {
  if (!bigfloat_iszero(t)) t->sign = !t->sign;
}

void bigfloat_floor(bigfloat_t t) {
  if (!t->coef || t->exp >= 0) return;
  size_t shift = (size_t)(-t->exp);
  t->len -= shift;
  t->exp = 0;
  memmove(t->coef, t->coef + shift, t->len * sizeof(uint32_t));
  t->coef = (uint32_t *)bc_xrealloc(t->coef, t->len * sizeof(uint32_t));
}

void bigfloat_print(const char *name, const bigfloat_t v) {
  printf("%s = bigfloat_t {exp = %ld, len = %ld, sign = %d, coef = ", name, (long)v->exp, (long)v->len, v->sign);
  if (!v->coef) {
    printf("NULL");
  } else {
    printf("{ ");
    for (size_t i = 0; i < v->len; i++) printf(i + 1 < v->len ? "0x%08x, " : "0x%08x", v->coef[i]);
    printf(" }");
  }
  printf("}\n");
}

void bigfloat_print10(const char *name, const bigfloat_t v) {
  printf("%s = bigfloat_t {exp = %ld, len = %ld, sign = %d, coef = ", name, (long)v->exp, (long)v->len, v->sign);
  if (!v->coef) {
    printf("NULL");
  } else {
    printf("{ ");
    for (size_t i = 0; i < v->len; i++) printf(i + 1 < v->len ? "%d, " : "%d", v->coef[i]);
    printf(" }");
  }
  printf("}\n");
}

/* ---------------------------------------------------------------- add / sub */

/* Limb of x at magnitude m (0 outside), bigfloat/addsub.c:17-27. */
static inline uint32_t limb_at(const _bigfloat_struct *x, int64_t m) {
  if (m < x->exp || m >= x->exp + (int64_t)x->len) return 0;
  return x->coef[m - x->exp];
}

/* Compare |a| and |b|: 1, -1 or 0 (bigfloat/addsub.c:33-63). */
static int ucmp(const _bigfloat_struct *a, const _bigfloat_struct *b) {
  int64_t ta = a->exp + (int64_t)a->len, tb = b->exp + (int64_t)b->len;
  if (ta != tb) return ta > tb ? 1 : -1;
  for (int64_t m = ta; m >= a->exp || m >= b->exp; m--) {
    uint32_t x = limb_at(a, m), y = limb_at(b, m);
    if (x != y) return x > y ? 1 : -1;
  }
  return 0;
}

/* The window [bot, top) kept for a sum or difference at precision p
 * (bigfloat/addsub.c:65-90 and 123-145): everything when p == 0, else the top
 * p+2 limbs.  Returns the exponent the reference assigns (top - p, with p the
 * window length when untruncated). */
static int64_t window(const _bigfloat_struct *a, const _bigfloat_struct *b, size_t p, int64_t *bot, int64_t *top) {
  int64_t ta = a->exp + (int64_t)a->len, tb = b->exp + (int64_t)b->len;
  *top = ta > tb ? ta : tb;
  *bot = a->exp < b->exp ? a->exp : b->exp;
  int64_t tl = *top - *bot;
  if (p == 0) p = (size_t)tl;
  else p += BIGFLOAT_EXTRA_PRECISION;
  if (tl > (int64_t)p) *bot = *top - (int64_t)p;
  return *top - (int64_t)p;
}

/* memcpy / memset of large arrays split over the OpenMP threads. */
void bc_par_memcpy(void *dst, const void *src, size_t n) {
  if (n < ((size_t)4 << 20)) {
    memcpy(dst, src, n);
    return;
  }
  const long nch = 64;
  const size_t chunk = (n + (size_t)nch - 1) / (size_t)nch;
#pragma omp parallel for schedule(static)
  for (long h = 0; h < nch; h++) {
    const size_t s0 = (size_t)h * chunk;
    if (s0 < n) memcpy((char *)dst + s0, (const char *)src + s0, s0 + chunk < n ? chunk : n - s0);
  }
}

void bc_par_memzero(void *dst, size_t n) {
  if (n < ((size_t)4 << 20)) {
    memset(dst, 0, n);
    return;
  }
  const long nch = 64;
  const size_t chunk = (n + (size_t)nch - 1) / (size_t)nch;
#pragma omp parallel for schedule(static)
  for (long h = 0; h < nch; h++) {
    const size_t s0 = (size_t)h * chunk;
    if (s0 < n) memset((char *)dst + s0, 0, s0 + chunk < n ? chunk : n - s0);
  }
}

/* Sums and differences of more than PAR_LIMBS limbs run in parallel chunks:
 * each chunk first with carry (borrow) in 0, recording its carry out and
 * whether its result is all ones (all zeros), then the carries into the
 * chunks follow in order (a chunk passes an incoming carry on only when its
 * result is all ones), and each chunk that receives one adds it.  Same
 * limbs as the serial loop.
 *
 * Inside a chunk the window is cut where an operand starts or ends, so each
 * piece runs a plain loop over the operands present there (an absent
 * operand contributes zeros) without a bounds test per limb. */
#define PAR_LIMBS ((size_t)1 << 20)

/* Output limb i of the window is limb i - off of x, for i in [lo, hi). */
typedef struct {
  const uint32_t *coef;
  int64_t off;
  size_t lo, hi;
} opview;

static opview view_of(const _bigfloat_struct *x, int64_t bot, size_t n) {
  opview v;
  const int64_t lo = x->exp - bot, hi = lo + (int64_t)x->len;
  v.coef = x->coef;
  v.off = lo;
  v.lo = lo < 0 ? 0 : (lo > (int64_t)n ? n : (size_t)lo);
  v.hi = hi < 0 ? 0 : (hi > (int64_t)n ? n : (size_t)hi);
  if (v.hi < v.lo) v.hi = v.lo;
  return v;
}

/* c[k] = A[k] + B[k] + cy over k < m (a null operand is zero); returns the
 * carry out, ANDs the limbs into *all. */
static uint64_t add_piece(uint32_t *c, const uint32_t *A, const uint32_t *B, size_t m, uint64_t cy, uint32_t *all) {
  uint32_t al = *all;
  if (A && B) {
    for (size_t k = 0; k < m; k++) {
      const uint64_t w = (uint64_t)A[k] + B[k] + cy;
      c[k] = (uint32_t)w;
      cy = w >> 32;
      al &= c[k];
    }
  } else if (A || B) {
    const uint32_t *X = A ? A : B;
    for (size_t k = 0; k < m; k++) {
      const uint64_t w = (uint64_t)X[k] + cy;
      c[k] = (uint32_t)w;
      cy = w >> 32;
      al &= c[k];
    }
  } else {
    for (size_t k = 0; k < m; k++) {
      c[k] = (uint32_t)cy;
      al &= c[k];
      cy = 0;
    }
  }
  *all = al;
  return cy;
}

/* c[k] = A[k] - B[k] - br over k < m; returns the borrow out, ORs the limbs
 * into *any. */
static uint64_t sub_piece(uint32_t *c, const uint32_t *A, const uint32_t *B, size_t m, uint64_t br, uint32_t *any) {
  uint32_t an = *any;
  if (A && B) {
    for (size_t k = 0; k < m; k++) {
      const uint64_t w = (uint64_t)A[k] - B[k] - br;
      c[k] = (uint32_t)w;
      br = (w >> 32) & 1;
      an |= c[k];
    }
  } else if (A) {
    for (size_t k = 0; k < m; k++) {
      const uint64_t w = (uint64_t)A[k] - br;
      c[k] = (uint32_t)w;
      br = (w >> 32) & 1;
      an |= c[k];
    }
  } else if (B) {
    for (size_t k = 0; k < m; k++) {
      const uint64_t w = (uint64_t)0 - B[k] - br;
      c[k] = (uint32_t)w;
      br = (w >> 32) & 1;
      an |= c[k];
    }
  } else {
    for (size_t k = 0; k < m; k++) {
      c[k] = br ? 0xffffffffu : 0u;
      an |= c[k];
    }
  }
  *any = an;
  return br;
}

/* Limbs [s0, s1) of the window, cut at the operands' ends; `sub` selects
 * a - b, else a + b.  Returns the carry (borrow) out; *acc collects the AND
 * (sum) or OR (difference) of the limbs. */
static uint64_t run_chunk(uint32_t *c, const opview *a, const opview *b, size_t s0, size_t s1, uint64_t cin, int sub,
                          uint32_t *acc) {
  size_t cut[6] = {s0, a->lo, a->hi, b->lo, b->hi, s1};
  for (int i = 1; i < 6; i++)  /* insertion sort of six cut points */
    for (int j = i; j > 0 && cut[j - 1] > cut[j]; j--) {
      const size_t t = cut[j];
      cut[j] = cut[j - 1];
      cut[j - 1] = t;
    }
  uint64_t cy = cin;
  for (int i = 0; i < 5; i++) {
    size_t u = cut[i] < s0 ? s0 : cut[i], v = cut[i + 1] > s1 ? s1 : cut[i + 1];
    if (u >= v) continue;
    const uint32_t *A = (u >= a->lo && u < a->hi) ? a->coef + (int64_t)u - a->off : NULL;
    const uint32_t *B = (u >= b->lo && u < b->hi) ? b->coef + (int64_t)u - b->off : NULL;
    cy = sub ? sub_piece(c + u, A, B, v - u, cy, acc) : add_piece(c + u, A, B, v - u, cy, acc);
  }
  return cy;
}

static void uadd(bigfloat_t t, const _bigfloat_struct *a, const _bigfloat_struct *b, size_t p) {
  int64_t bot, top;
  int64_t e = window(a, b, p, &bot, &top);
  size_t n = (size_t)(top - bot);
  uint32_t *c = (uint32_t *)bc_xmalloc((n + 1) * sizeof(uint32_t));
  const opview va = view_of(a, bot, n), vb = view_of(b, bot, n);
  uint64_t carry = 0;
  if (n < PAR_LIMBS) {
    uint32_t all = 0xffffffffu;
    carry = run_chunk(c, &va, &vb, 0, n, 0, 0, &all);
  } else {
    const long nch = 256;
    const size_t chunk = (n + (size_t)nch - 1) / (size_t)nch;
    unsigned char co[256], ones[256], ci[257];
#pragma omp parallel for schedule(static)
    for (long h = 0; h < nch; h++) {
      const size_t s0 = (size_t)h * chunk < n ? (size_t)h * chunk : n, s1 = s0 + chunk < n ? s0 + chunk : n;
      uint32_t all = 0xffffffffu;
      co[h] = (unsigned char)run_chunk(c, &va, &vb, s0, s1, 0, 0, &all);
      ones[h] = s0 < s1 && all == 0xffffffffu;
    }
    ci[0] = 0;
    for (long h = 0; h < nch; h++) ci[h + 1] = co[h] | (ones[h] & ci[h]);
#pragma omp parallel for schedule(static)
    for (long h = 0; h < nch; h++) {
      if (!ci[h]) continue;
      const size_t s0 = (size_t)h * chunk, s1 = s0 + chunk < n ? s0 + chunk : n;
      for (size_t i = s0; i < s1; i++)
        if (++c[i] != 0) break;
    }
    carry = ci[nch];
  }
  if (carry) c[n++] = 1;
  int sign = a->sign;
  free(t->coef);
  t->coef = c;
  t->sign = sign;
  t->exp = e;
  t->len = n;
}

/* |a| >= |b| assumed (callers order the operands). */
static void usub(bigfloat_t t, const _bigfloat_struct *a, const _bigfloat_struct *b, size_t p) {
  int64_t bot, top;
  int64_t e = window(a, b, p, &bot, &top);
  size_t n = (size_t)(top - bot);
  uint32_t *c = (uint32_t *)bc_xmalloc((n + 1) * sizeof(uint32_t));
  const opview va = view_of(a, bot, n), vb = view_of(b, bot, n);
  if (n < PAR_LIMBS) {
    uint32_t any = 0;
    (void)run_chunk(c, &va, &vb, 0, n, 0, 1, &any);
  } else {
    const long nch = 256;
    const size_t chunk = (n + (size_t)nch - 1) / (size_t)nch;
    unsigned char bo[256], zeros[256], bi[257];
#pragma omp parallel for schedule(static)
    for (long h = 0; h < nch; h++) {
      const size_t s0 = (size_t)h * chunk < n ? (size_t)h * chunk : n, s1 = s0 + chunk < n ? s0 + chunk : n;
      uint32_t any = 0;
      bo[h] = (unsigned char)run_chunk(c, &va, &vb, s0, s1, 0, 1, &any);
      zeros[h] = s0 < s1 && any == 0;
    }
    bi[0] = 0;
    for (long h = 0; h < nch; h++) bi[h + 1] = bo[h] | (zeros[h] & bi[h]);
#pragma omp parallel for schedule(static)
    for (long h = 0; h < nch; h++) {
      if (!bi[h]) continue;
      const size_t s0 = (size_t)h * chunk, s1 = s0 + chunk < n ? s0 + chunk : n;
      for (size_t i = s0; i < s1; i++)
        if (c[i]-- != 0) break;
    }
  }
  while (n > 0 && c[n - 1] == 0) n--;
  int sign = a->sign;
  free(t->coef);
  t->coef = c;
  t->sign = sign;
  t->exp = e;
  t->len = n;
  if (n == 0) bigfloat_zero(t);
}

/* bigfloat/addsub.c:183-210 */
void bigfloat_add(bigfloat_t t, const bigfloat_t a, const bigfloat_t b, size_t p) {
  if (a->sign == b->sign) {
    uadd(t, a, b, p);
  } else if (ucmp(a, b) > 0) {
    usub(t, a, b, p);
  } else {
    usub(t, b, a, p);
    bigfloat_neg(t);
  }
}

/* bigfloat/addsub.c:212-237 */
void bigfloat_sub(bigfloat_t t, const bigfloat_t a, const bigfloat_t b, size_t p) {
  if (a->sign != b->sign) {
    uadd(t, a, b, p);
  } else if (ucmp(a, b) > 0) {
    usub(t, a, b, p);
  } else {
    usub(t, b, a, p);
    bigfloat_neg(t);
  }
}

/* ---------------------------------------------------------------- multiply */

/* Product length and trimming rule of bigfloat/mul.c:664-675. */
static void trim_product(bigfloat_t t) {
  if (t->coef[t->len - 1] == 0) t->len--;
  if (t->len > 1000)
    while (t->coef[t->len - 1] == 0) t->len--;
}

/* Operands after the precision chop of bigfloat/mul.c:573-602. */
void bc_mul_operands(const _bigfloat_struct *a, const _bigfloat_struct *b, size_t p, bc_operand *oa, bc_operand *ob) {
  if (p == 0) p = a->len + b->len;
  else p += BIGFLOAT_EXTRA_PRECISION;
  oa->T = a->coef; oa->L = a->len; oa->exp = a->exp;
  ob->T = b->coef; ob->L = b->len; ob->exp = b->exp;
  if (oa->L > p) { size_t chop = oa->L - p; oa->L = p; oa->exp += (int64_t)chop; oa->T += chop; }
  if (ob->L > p) { size_t chop = ob->L - p; ob->L = p; ob->exp += (int64_t)chop; ob->T += chop; }
}

/* bigfloat/mul.c:555-676: exact product of the chopped operands.  CL == 2 and
 * CL < 100 stay on the host (the reference's fast path and Karatzuba range);
 * everything else is one GPU product. */
void bigfloat_mul(bigfloat_t t, const bigfloat_t a, const bigfloat_t b, size_t p) {
  if (bigfloat_iszero(a) || bigfloat_iszero(b)) {
    bigfloat_zero(t);
    return;
  }
  bc_operand oa, ob;
  bc_mul_operands(a, b, p, &oa, &ob);
  const size_t CL = oa.L + ob.L;
  const int sign = a->sign == b->sign;
  const int64_t exp = oa.exp + ob.exp;
  uint32_t *c = (uint32_t *)bc_xmalloc(CL * sizeof(uint32_t));
  if (CL == 2) {
    uint64_t r = (uint64_t)oa.T[0] * ob.T[0];
    c[0] = (uint32_t)r;
    c[1] = (uint32_t)(r >> 32);
  } else if (CL < BC_SMALL_PRODUCT_LIMBS) {
    bc_small_mul(c, CL, oa.T, oa.L, ob.T, ob.L);
  } else {
    _fft_mul(c, CL, (uint32_t *)oa.T, oa.L, (uint32_t *)ob.T, ob.L);
  }
  free(t->coef);
  t->coef = c;
  t->sign = sign;
  t->exp = exp;
  t->len = CL;
  trim_product(t);
}

/* Batch of bigfloat_mul: small products on the host, the rest in one
 * bc_gpu_mul_batch call.  Each result is what bigfloat_mul would produce. */
void bigfloat_mul_batch(bigfloat_mul_item *items, size_t n) {
  /* 1: operands, targets and which products go to the GPU (serial: cheap) */
  bc_gpu_item *g = (bc_gpu_item *)bc_xmalloc((n ? n : 1) * sizeof(bc_gpu_item));
  bc_operand *ops = (bc_operand *)bc_xmalloc((n ? 2 * n : 2) * sizeof(bc_operand));
  char *kind = (char *)bc_xmalloc(n ? n : 1);  /* 0 zero, 1 host, 2 gpu, 3 gpu small */
  size_t ng = 0, ns = 0;
  for (size_t i = 0; i < n; i++) {
    _bigfloat_struct *t = items[i].target;
    const _bigfloat_struct *a = items[i].a, *b = items[i].b;
    if (bigfloat_iszero(a) || bigfloat_iszero(b)) {
      bigfloat_zero(t);
      kind[i] = 0;
      continue;
    }
    bc_operand *oa = &ops[2 * i], *ob = &ops[2 * i + 1];
    bc_mul_operands(a, b, items[i].p, oa, ob);
    const size_t CL = oa->L + ob->L;
    uint32_t *c = (uint32_t *)bc_xmalloc(CL * sizeof(uint32_t));
    kind[i] = (CL == 2 || CL < BC_SMALL_PRODUCT_LIMBS) ? 1 : 2;
    if (kind[i] == 1 && CL > 2) ns++;
    if (kind[i] == 2) {
      g[ng].C = c; g[ng].CL = CL; g[ng].A = oa->T; g[ng].AL = oa->L; g[ng].B = ob->T; g[ng].BL = ob->L;
      ng++;
    }
    free(t->coef);
    t->coef = c;
    t->sign = a->sign == b->sign;
    t->exp = oa->exp + ob->exp;
    t->len = CL;
  }
  /* 2: GPU products in one batch while host threads do the small ones; many
   * small ones (the lower levels of a level-ordered tree) go to the GPU as
   * one more batch (schoolbook, one launch) */
  bc_gpu_item *sg = NULL;
  if (ns >= BC_SMALL_GPU_MIN) {
    sg = (bc_gpu_item *)bc_xmalloc(ns * sizeof(bc_gpu_item));
    ns = 0;
    for (size_t i = 0; i < n; i++) {
      if (kind[i] != 1 || items[i].target->len == 2) continue;
      const bc_operand *oa = &ops[2 * i], *ob = &ops[2 * i + 1];
      _bigfloat_struct *t = items[i].target;
      sg[ns].C = t->coef; sg[ns].CL = t->len; sg[ns].A = oa->T; sg[ns].AL = oa->L; sg[ns].B = ob->T; sg[ns].BL = ob->L;
      ns++;
      kind[i] = 3;
    }
  }
  long nn = (long)n;
#pragma omp parallel
  {
#pragma omp single nowait
    {
      if (ng) bc_host_gpu_batch(g, ng);
      if (sg) bc_host_gpu_small_batch(sg, ns);
    }
#pragma omp for schedule(dynamic, 256)
    for (long i = 0; i < nn; i++) {
      if (kind[i] != 1) continue;
      _bigfloat_struct *t = items[i].target;
      const bc_operand *oa = &ops[2 * i], *ob = &ops[2 * i + 1];
      if (t->len == 2) {
        uint64_t r = (uint64_t)oa->T[0] * ob->T[0];
        t->coef[0] = (uint32_t)r;
        t->coef[1] = (uint32_t)(r >> 32);
      } else {
        bc_small_mul(t->coef, t->len, oa->T, oa->L, ob->T, ob->L);
      }
    }
  }
  for (size_t i = 0; i < n; i++)
    if (kind[i]) trim_product(items[i].target);
  free(kind);
  free(ops);
  free(g);
  free(sg);
}

/* bigfloat/mul.c:64-80: a *= b in place over a->len limbs, the top limb
 * cleared first and the final carry dropped. */
void bigfloat_mului(bigfloat_t a, uint32_t b) {
  a->coef[a->len - 1] = 0;
  uint64_t carry = 0;
  for (size_t i = 0; i < a->len; i++) {
    uint64_t v = (uint64_t)a->coef[i] * b + carry;
    a->coef[i] = (uint32_t)v;
    carry = v >> 32;
  }
}

/* bigfloat/mul.c:83-102: target->len limbs of a*b (target allocated by the
 * caller, final carry dropped). */
void bigfloat_mulu(bigfloat_t t, const bigfloat_t a, uint32_t b) {
  uint64_t carry = 0;
  for (size_t i = 0; i < t->len; i++) {
    uint64_t v = carry;
    if (i < a->len) v += (uint64_t)a->coef[i] * b;
    t->coef[i] = (uint32_t)v;
    carry = v >> 32;
  }
}

/* bigfloat/exp.c:13-29: square and multiply, in place, no truncation. */
void bigfloat_exp(bigfloat_t t, const bigfloat_t a, uint64_t e) {
  bigfloat_t cp;
  bigfloat_new(cp);
  bigfloat_copy(cp, a);
  bigfloat_set(t, 1);
  while (e > 0) {
    if (e % 2 == 1) bigfloat_mul(t, t, cp, 0);
    bigfloat_mul(cp, cp, cp, 0);
    e /= 2;
  }
  bigfloat_free(cp);
}
