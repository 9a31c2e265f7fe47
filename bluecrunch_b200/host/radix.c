/* radix.c — binary (2^32) to decimal (10^9) conversion of a fraction, and
 * string output.
 *
 * The conversion is the reference's subquadratic, division-free scheme after
 * Bouvier and Zimmermann (bigfloat/radix.c:20-360): a tree that splits k
 * output digits into kh = (k+1)/2 high and kl = k-kh+1 low digits, the low
 * half obtained from y * 10^(9(k-kl)) mod 2^(32n) (one product per node),
 * leaves of at most KT digits by repeated multiplication by 10^9, and two
 * fix-ups where the halves meet.  Every step that touches values is the same
 * as the reference's, so the digits are identical.
 *
 * Three drivers, all producing the same digits: convert_rec_percall()
 * recurses like the reference (one GPU product per node, BC_RADIX_PERCALL);
 * convert_levels() walks the same tree level by level, multiplies a whole
 * level in one bigfloat_mul_batch, converts all leaves on the GPU in one
 * launch (bc_gpu_radix_leaves) and combines each level in parallel on the
 * host (BC_RADIX_LEVELS); convert_tree(), the default, plans the tree here
 * and runs all of it in device memory (bc_gpu_radix_tree).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "bc_gpu.h"
#include "bc_host.h"
#include "bench.h"
#include "bigfloat.h"

#define OLDBASE (4294967296.0)
#define NEWBASE (1000000000u)
#define LOGR (log(OLDBASE) / log((double)NEWBASE))
#define ALPHA (log((double)NEWBASE) / log(OLDBASE))
#define KT (1000)
#define TABLE_SLOTS 128

/* bigfloat/radix.c:20-39 */
size_t bigfloat_radix_decimals(bigfloat_t t) {
  double approx = 0.0;
  if (t->len >= 3) approx += (double)t->coef[t->len - 3];
  if (t->len >= 2) approx += (double)t->coef[t->len - 2] * OLDBASE;
  approx += (double)t->coef[t->len - 1] * OLDBASE * OLDBASE;
  double digits = log(approx) / log((double)NEWBASE);
  double additional = ((double)t->len - 3.0) * log(OLDBASE) / log((double)NEWBASE);
  return (size_t)ceil(digits + additional + 1e-10);
}

/* ---------------------------------------------------------------- leaves */

/* bigfloat/radix.c:41-91: k base-10^9 digits of the fraction y0 (n limbs
 * below the point) by k rounds of t <- t*10^9, taking the limb that crosses
 * the point and dropping limbs that can no longer matter. */
static void convert_trunc(bigfloat_t s, const _bigfloat_struct *y0, size_t k, size_t n) {
  const double alpha = ALPHA;
  const size_t L = y0->len + 1;
  uint32_t *base = (uint32_t *)bc_xmalloc(L * sizeof(uint32_t));
  memcpy(base, y0->coef, y0->len * sizeof(uint32_t));
  base[L - 1] = 0;
  uint32_t *tc = base;
  size_t tl = L;
  for (size_t i = 1; i <= k; i++) {
    /* bigfloat_mului: clear the top limb, multiply, drop the carry */
    tc[tl - 1] = 0;
    uint64_t carry = 0;
    for (size_t j = 0; j < tl; j++) {
      uint64_t v = (uint64_t)tc[j] * NEWBASE + carry;
      tc[j] = (uint32_t)v;
      carry = v >> 32;
    }
    size_t ni_1 = (size_t)((double)n - floor(alpha * (double)(i - 1)));
    size_t ni = (size_t)((double)n - floor(alpha * (double)i));
    s->coef[k - i] = tc[ni_1];
    tl = ni_1;
    tc += (ni_1 - ni);
    tl -= (ni_1 - ni);
    tl += 1;
    tc[tl - 1] = 0;
  }
  s->len = k;
  free(base);
}

/* ---------------------------------------------------------------- table of 10^(9e) */

typedef struct {
  size_t exps[TABLE_SLOTS];
  bigfloat_t val[TABLE_SLOTS];
  int n;
} pow_table;

static int table_find(const pow_table *tb, size_t e) {
  for (int i = 0; i < TABLE_SLOTS; i++)
    if (tb->exps[i] == e) return i;
  return -1;
}

static void table_insert(pow_table *tb, size_t e) {
  for (int i = 0; i < TABLE_SLOTS; i++) {
    if (tb->exps[i] == e) return;
    if (tb->exps[i] == 0) {
      tb->exps[i] = e;
      return;
    }
  }
}

/* bigfloat/radix.c:136-154: every internal node needs 10^(9(k-kl)). */
static void table_collect(pow_table *tb, size_t k) {
  if (k < KT) return;
  size_t kh = (k + 1) / 2, kl = k - kh + 1;
  table_collect(tb, kh);
  if (kl != kh) table_collect(tb, kl);
  table_insert(tb, k - kl);
}

static int cmp_size(const void *x, const void *y) {
  size_t a = *(const size_t *)x, b = *(const size_t *)y;
  return a < b ? -1 : (a > b);
}

/* bigfloat/radix.c:156-205 builds the entries in increasing order from the
 * smallest (a power) by one multiply by 10^9 or one squaring (plus one
 * multiply by 10^9).  The values are exact integers, so any exact order gives
 * the same table; this keeps the reference's steps. */
static void table_build(pow_table *tb, size_t k) {
  memset(tb->exps, 0, sizeof tb->exps);
  tb->n = 0;
  if (k < KT) return;
  table_collect(tb, k);
  int n = 0;
  while (n < TABLE_SLOTS && tb->exps[n]) n++;
  /* the reference sorts all but the last entry (bigfloat/radix.c:125-134);
   * the last inserted is the root's, the largest, so a full sort is equal */
  qsort(tb->exps, (size_t)n, sizeof(size_t), cmp_size);
  tb->n = n;
  for (int i = 0; i < n; i++) bigfloat_new(tb->val[i]);
  bigfloat_t base;
  bigfloat_new(base);
  bigfloat_set(base, NEWBASE);
  bigfloat_exp(tb->val[0], base, tb->exps[0]);
  bigfloat_free(base);
  for (int i = 1; i < n; i++) {
    size_t e = tb->exps[i];
    int j = table_find(tb, e - 1);
    if (j >= 0 && j < i) {
      bigfloat_alloc(tb->val[i], tb->val[j]->len + 1);
      bigfloat_mulu(tb->val[i], tb->val[j], NEWBASE);
      continue;
    }
    j = table_find(tb, e / 2);
    if (j >= 0 && j < i) {
      bigfloat_mul(tb->val[i], tb->val[j], tb->val[j], 0);
      if (e & 1) {
        bigfloat_realloc(tb->val[i], tb->val[i]->len + 1);
        bigfloat_mului(tb->val[i], NEWBASE);
      }
      continue;
    }
    fprintf(stderr, "radix table: no predecessor for 10^(9*%zu)\n", e);
    abort();
  }
}

/* The same table as a plan for the device: exponents, entry 0's value, and
 * for every later entry the step table_build would take (op 1: times 10^9
 * from entry e-1; op 2: square of entry e/2; op 3: that square times 10^9). */
static void table_plan(pow_table *tb, size_t k, bc_radix_pow_step *steps) {
  memset(tb->exps, 0, sizeof tb->exps);
  tb->n = 0;
  if (k < KT) return;
  table_collect(tb, k);
  int n = 0;
  while (n < TABLE_SLOTS && tb->exps[n]) n++;
  qsort(tb->exps, (size_t)n, sizeof(size_t), cmp_size);
  tb->n = n;
  for (int i = 0; i < n; i++) bigfloat_new(tb->val[i]);
  bigfloat_t base;
  bigfloat_new(base);
  bigfloat_set(base, NEWBASE);
  bigfloat_exp(tb->val[0], base, tb->exps[0]);
  bigfloat_free(base);
  steps[0].src = 0;
  steps[0].op = 0;
  for (int i = 1; i < n; i++) {
    size_t e = tb->exps[i];
    int j = table_find(tb, e - 1);
    if (j >= 0 && j < i) {
      steps[i].src = j;
      steps[i].op = 1;
      continue;
    }
    j = table_find(tb, e / 2);
    if (j >= 0 && j < i) {
      steps[i].src = j;
      steps[i].op = (e & 1) ? 3 : 2;
      continue;
    }
    fprintf(stderr, "radix table: no predecessor for 10^(9*%zu)\n", e);
    abort();
  }
}

static void table_free(pow_table *tb) {
  for (int i = 0; i < tb->n; i++) bigfloat_free(tb->val[i]);
  tb->n = 0;
  memset(tb->exps, 0, sizeof tb->exps);
}

/* ---------------------------------------------------------------- split and merge */

static void split_sizes(size_t k, size_t g, size_t *kh, size_t *kl, size_t *nh, size_t *nl) {
  *kh = (k + 1) / 2;
  *kl = k - *kh + 1;
  /* smallest limb counts with 4 g 10^(9 k*) < 2^(32 n*) (bigfloat/radix.c:238-243) */
  *nh = (size_t)floor((double)(*kh * log((double)NEWBASE) + log(4.) + log((double)g)) / log(OLDBASE) + 1);
  *nl = (size_t)floor((double)(*kl * log((double)NEWBASE) + log(4.) + log((double)g)) / log(OLDBASE) + 1);
}

/* yh = top limbs of y (bigfloat/radix.c:245-249). */
static void take_high(bigfloat_t yh, const _bigfloat_struct *y, size_t n, size_t nh) {
  bigfloat_alloc(yh, y->len - (n - nh));
  bc_par_memcpy(yh->coef, y->coef + (n - nh), yh->len * sizeof(uint32_t));
}

/* s = floor(sh/b) * b^kl + sl with the two edge fix-ups
 * (bigfloat/radix.c:277-316). */
static void merge(bigfloat_t s, bigfloat_t sh, const bigfloat_t sl, size_t kl) {
  if (sh->coef[0] == NEWBASE - 1 && sl->coef[sl->len - 1] == 0) {
    uint32_t carry = 1;
    for (size_t i = 0; i < sh->len && carry; i++) {
      uint64_t sum = (uint64_t)sh->coef[i] + carry;
      carry = (uint32_t)(sum / NEWBASE);
      sh->coef[i] = (uint32_t)(sum % NEWBASE);
    }
  }
  int sl_zero = sh->coef[0] == 0 && sl->coef[sl->len - 1] == NEWBASE - 1;
  bigfloat_alloc(s, sh->len - 1 + kl);
  bc_par_memzero(s->coef, kl * sizeof(uint32_t));
  bc_par_memcpy(s->coef + kl, sh->coef + 1, (sh->len - 1) * sizeof(uint32_t));
  if (!sl_zero) bigfloat_add(s, s, sl, 0);
}

/* yl view: low n limbs of y * 10^(9(k-kl)), then the top nl of those
 * (bigfloat/radix.c:251-261).  `prod` owns the limbs; yl points into it. */
static void low_view(_bigfloat_struct *yl, const bigfloat_t prod, size_t n, size_t nl) {
  yl->coef = prod->coef + (n - nl);
  yl->len = nl;
  yl->exp = prod->exp;
  yl->sign = prod->sign;
}

/* ---------------------------------------------------------------- recursive driver */

static pow_table g_tab;

static void convert_rec_percall(bigfloat_t s, size_t k, const _bigfloat_struct *y, size_t n, size_t g) {
  if (k <= KT) {
    bigfloat_alloc(s, k);
    convert_trunc(s, y, k, n);
    return;
  }
  size_t kh, kl, nh, nl;
  split_sizes(k, g, &kh, &kl, &nh, &nl);
  bigfloat_t yh, prod, sh, sl;
  bigfloat_new(yh);
  bigfloat_new(prod);
  bigfloat_new(sh);
  bigfloat_new(sl);
  take_high(yh, y, n, nh);
  bigfloat_mul(prod, y, g_tab.val[table_find(&g_tab, k - kl)], 0);
  if (prod->len < n) bigfloat_realloc(prod, n); /* trimmed top zeros come back as zeros */
  _bigfloat_struct yl;
  low_view(&yl, prod, n, nl);
  convert_rec_percall(sh, kh, yh, nh, g);
  convert_rec_percall(sl, kl, &yl, nl, g);
  merge(s, sh, sl, kl);
  bigfloat_free(sh);
  bigfloat_free(sl);
  bigfloat_free(yh);
  bigfloat_free(prod);
}

/* ---------------------------------------------------------------- level driver */

typedef struct node {
  size_t k, n;
  int parent;        /* index in the previous level, -1 for the root */
  int is_high;       /* 1: sh of the parent, 0: sl */
  _bigfloat_struct y;      /* input (view or owned) */
  _bigfloat_struct owner;  /* owns y's limbs */
  _bigfloat_struct s;      /* output digits */
  size_t kl;               /* for internal nodes */
  int child_h, child_l;    /* indices in the next level */
} node;

static double wall_now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void convert_levels(bigfloat_t target, size_t k0, const _bigfloat_struct *y0, size_t n0, size_t g) {
  double t0 = wall_now(), t_split = 0, t_leaf = 0, t_merge = 0;
  node **lv = NULL;
  size_t *cnt = NULL;
  int nlv = 0;
  lv = (node **)bc_xmalloc(sizeof(node *));
  cnt = (size_t *)bc_xmalloc(sizeof(size_t));
  lv[0] = (node *)calloc(1, sizeof(node));
  cnt[0] = 1;
  lv[0][0].k = k0;
  lv[0][0].n = n0;
  lv[0][0].parent = -1;
  lv[0][0].y = *y0;
  bigfloat_new(&lv[0][0].owner);
  bigfloat_new(&lv[0][0].s);
  nlv = 1;
  /* top-down: split every internal node, one product batch per level */
  for (;;) {
    node *L = lv[nlv - 1];
    size_t m = cnt[nlv - 1], ninternal = 0;
    for (size_t i = 0; i < m; i++) ninternal += L[i].k > KT;
    if (!ninternal) break;
    node *N = (node *)calloc(2 * ninternal, sizeof(node));
    bigfloat_mul_item *items = (bigfloat_mul_item *)bc_xmalloc(ninternal * sizeof(bigfloat_mul_item));
    size_t c = 0, q = 0;
    for (size_t i = 0; i < m; i++) {
      node *x = &L[i];
      if (x->k <= KT) continue;
      size_t kh, kl, nh, nl;
      split_sizes(x->k, g, &kh, &kl, &nh, &nl);
      x->kl = kl;
      node *h = &N[c], *l = &N[c + 1];
      x->child_h = (int)c;
      x->child_l = (int)c + 1;
      c += 2;
      h->k = kh; h->n = nh; h->parent = (int)i; h->is_high = 1;
      l->k = kl; l->n = nl; l->parent = (int)i; l->is_high = 0;
      bigfloat_new(&h->owner); bigfloat_new(&l->owner);
      bigfloat_new(&h->s); bigfloat_new(&l->s);
      take_high(&h->owner, &x->y, x->n, nh);
      h->y = h->owner;
      items[q].target = &l->owner;
      items[q].a = &x->y;
      items[q].b = g_tab.val[table_find(&g_tab, x->k - kl)];
      items[q].p = 0;
      q++;
    }
    bigfloat_mul_batch(items, q);
    free(items);
    for (size_t i = 0; i < m; i++) {
      node *x = &L[i];
      if (x->k <= KT) continue;
      node *l = &N[x->child_l];
      if (l->owner.len < x->n) bigfloat_realloc(&l->owner, x->n);
      low_view(&l->y, &l->owner, x->n, l->n);
      bigfloat_free(&x->owner); /* an internal node's input is no longer needed */
    }
    lv = (node **)bc_xrealloc(lv, (size_t)(nlv + 1) * sizeof(node *));
    cnt = (size_t *)bc_xrealloc(cnt, (size_t)(nlv + 1) * sizeof(size_t));
    lv[nlv] = N;
    cnt[nlv] = c;
    nlv++;
  }
  t_split = wall_now() - t0;
  t0 = wall_now();
  /* leaves, all levels at once, in one GPU launch (convert_trunc's rounds
   * per leaf, bc_gpu_radix_leaves) */
  {
    size_t nleaf = 0;
    for (int d = 0; d < nlv; d++)
      for (size_t i = 0; i < cnt[d]; i++) nleaf += lv[d][i].k <= KT;
    bc_radix_leaf *rl = (bc_radix_leaf *)bc_xmalloc((nleaf ? nleaf : 1) * sizeof(bc_radix_leaf));
    size_t q = 0;
    for (int d = 0; d < nlv; d++)
      for (size_t i = 0; i < cnt[d]; i++) {
        node *x = &lv[d][i];
        if (x->k > KT) continue;
        bigfloat_alloc(&x->s, x->k);
        x->s.len = x->k;
        rl[q].y = x->y.coef;
        rl[q].len = x->y.len;
        rl[q].n = x->n;
        rl[q].k = x->k;
        rl[q].s = x->s.coef;
        q++;
      }
    bc_host_ensure_gpu();
    int rc = bc_gpu_radix_leaves(rl, q, ALPHA);
    if (rc != BC_OK) {
      fprintf(stderr, "bigfloat_radix: GPU conversion of %zu leaves failed: %s\n", q, bc_gpu_strerror(rc));
      abort();
    }
    free(rl);
  }
  t_leaf = wall_now() - t0;
  t0 = wall_now();
  /* bottom-up merges, one level at a time, nodes of a level in parallel */
  for (int d = nlv - 2; d >= 0; d--) {
    node *L = lv[d], *N = lv[d + 1];
    long m = (long)cnt[d];
#pragma omp parallel for schedule(dynamic, 1) if (m >= 16)  /* few big nodes: merge in parallel inside */
    for (long i = 0; i < m; i++) {
      node *x = &L[i];
      if (x->k <= KT) continue;
      node *h = &N[x->child_h], *l = &N[x->child_l];
      merge(&x->s, &h->s, &l->s, x->kl);
      bigfloat_free(&h->s);
      bigfloat_free(&l->s);
      bigfloat_free(&h->owner);
      bigfloat_free(&l->owner);
    }
    free(N);
  }
  t_merge = wall_now() - t0;
  if (getenv("BC_STATS"))
    printf("    conversion: %d levels, splits and products %.3f s, leaves %.3f s, merges %.3f s\n", nlv, t_split,
           t_leaf, t_merge);
  /* hand the root's digits to the target */
  free(target->coef);
  *target = lv[0][0].s;
  free(lv[0]);
  free(lv);
  free(cnt);
}

/* ---------------------------------------------------------------- tree on the device */

/* The same tree planned here (split_sizes, power-table entries) and run in
 * one call, bc_gpu_radix_tree_pow, with the power table built from its plan
 * and every product, leaf and merge in device memory: the fraction and the
 * table's first entry go over once, the digits come back once. */
static bc_radix_pow_step g_steps[TABLE_SLOTS];

static void convert_tree(uint32_t *out, size_t k0, const _bigfloat_struct *y0, size_t n0, size_t g) {
  double t0 = wall_now();
  size_t cap = 64, nn = 1;
  bc_radix_node *nd = (bc_radix_node *)bc_xmalloc(cap * sizeof(bc_radix_node));
  nd[0].k = k0;
  nd[0].n = n0;
  nd[0].child_h = nd[0].child_l = -1;
  nd[0].kl = 0;
  nd[0].table = -1;
  for (size_t i = 0; i < nn; i++) { /* breadth first: children after their parent */
    if (nd[i].k <= KT) continue;
    size_t kh, kl, nh, nl;
    split_sizes(nd[i].k, g, &kh, &kl, &nh, &nl);
    if (nn + 2 > cap) {
      cap *= 2;
      nd = (bc_radix_node *)bc_xrealloc(nd, cap * sizeof(bc_radix_node));
    }
    nd[i].kl = kl;
    nd[i].table = table_find(&g_tab, nd[i].k - kl);
    nd[i].child_h = (long)nn;
    nd[i].child_l = (long)nn + 1;
    bc_radix_node h = {kh, nh, -1, -1, 0, -1}, l = {kl, nl, -1, -1, 0, -1};
    nd[nn++] = h;
    nd[nn++] = l;
  }
  bc_host_ensure_gpu();
  int rc;
  if (g_tab.n > 0) {
    rc = bc_gpu_radix_tree_pow(y0->coef, y0->len, nd, nn, g_tab.val[0]->coef, g_tab.val[0]->len, g_steps, g_tab.n,
                               ALPHA, out);
  } else {
    rc = bc_gpu_radix_tree(y0->coef, y0->len, nd, nn, NULL, NULL, 0, ALPHA, out);
  }
  if (rc != BC_OK) {
    fprintf(stderr, "bigfloat_radix: GPU conversion tree of %zu nodes failed: %s\n", nn, bc_gpu_strerror(rc));
    abort();
  }
  if (getenv("BC_STATS")) printf("    conversion: %zu nodes on the device, %.3f s\n", nn, wall_now() - t0);
  free(nd);
}

/* bigfloat/radix.c:321-360 */
void bigfloat_radix(bigfloat_t target, const bigfloat_t a) {
  if (-a->exp + 1 != (int64_t)a->len) {
    fprintf(stderr, "Not implemented\n");
    abort();
  }
  size_t n = (size_t)(-a->exp);
  size_t k = (size_t)ceil((double)n * LOGR) - 1;
  double gd = ceil(log((double)k) / log(OLDBASE)) + 1;
  size_t g = (size_t)(gd > KT ? gd : KT);
  const int tree = !getenv("BC_RADIX_PERCALL") && !getenv("BC_RADIX_LEVELS");
  task_start(2, "Precomputing base conversion table");
  if (tree) table_plan(&g_tab, k, g_steps); /* the tree builds the rest on the device */
  else table_build(&g_tab, k);
  task_end(2);
  bigfloat_alloc(target, k);
  task_start(2, "Conversion");
  if (getenv("BC_RADIX_PERCALL")) convert_rec_percall(target, k, a, n, g);
  else if (getenv("BC_RADIX_LEVELS")) convert_levels(target, k, a, n, g);
  else convert_tree(target->coef, k, a, n, g);
  task_end(2);
  table_free(&g_tab);
  if (target->coef[target->len - 1] > NEWBASE) {
    bigfloat_realloc(target, target->len + 1);
    target->coef[target->len - 1] = target->coef[target->len - 2] / NEWBASE;
    target->coef[target->len - 2] = target->coef[target->len - 2] % NEWBASE;
  }
  target->exp = -(int64_t)target->len + 1;
}

/* ---------------------------------------------------------------- strings */

/* bigfloat/string.c:15-37: 8 hex or 9 decimal digits of one limb. */
static size_t limb_hex(uint32_t v, char *s) {
  for (int i = 7; i >= 0; i--) {
    int d = v % 16;
    s[i] = (char)(d < 10 ? '0' + d : 'a' + d - 10);
    v /= 16;
  }
  return 8;
}

static size_t limb_dec(uint32_t v, char *s) {
  for (int i = 8; i >= 0; i--) {
    s[i] = (char)('0' + v % 10);
    v /= 10;
  }
  return 9;
}

/* bigfloat/string.c:62-125's layout, including its choice of how many limbs
 * to print (digits/8 for base 10, digits/9 for base 16) and its final
 * truncation: after `head` characters ("2." for a value in [1, 2^32), "."
 * below), the limbs c-1, c-2, ... down to at most c-n, w characters each,
 * and the length the reference returns, which is how many bytes its caller
 * writes.  The reference's loop stops after the first limb that brings the
 * string to `digits` characters; every limb's place is known in advance, so
 * the limbs can be printed in parallel. */
typedef struct {
  size_t head, c, n, w, len;
} text_plan;

static text_plan plan_text(size_t vlen, int64_t exp, uint32_t top, size_t digits, int base) {
  text_plan t;
  const int mag = (int)((int64_t)vlen + exp);
  t.c = vlen - 1;
  if (mag == 1 && top != 2) {
    fprintf(stderr, "Not implemented\n");
    abort();
  }
  t.head = mag == 1 ? 2 : 1;
  const size_t per = base == 10 ? 8 : 9;
  const size_t min_c = vlen > digits / per ? vlen - digits / per - 1 : 0;
  t.w = base == 10 ? 9 : 8;
  t.n = t.c > min_c ? t.c - min_c : 0;
  if (t.n) {
    const size_t need = digits > t.head ? (digits - t.head + t.w - 1) / t.w : 1;
    if (need < t.n) t.n = need;
  }
  const size_t total = t.head + t.n * t.w; /* characters before the terminator */
  t.len = total + 1 > digits ? digits - 1 : total;
  return t;
}

size_t bigfloat_to_string(char *string, const bigfloat_t value, size_t digits, int base) {
  if (value->len == 0) {
    string[0] = '0';
    string[1] = '\0';
    return 1;
  }
  const text_plan t = plan_text(value->len, value->exp, value->coef[value->len - 1], digits, base);
  if (t.head == 2) string[0] = '2';
  string[t.head - 1] = '.';
  const long nn = (long)t.n;
#pragma omp parallel for schedule(static) if (nn > 100000)
  for (long k = 0; k < nn; k++) {
    const uint32_t v = value->coef[t.c - 1 - (size_t)k];
    if (base == 10) limb_dec(v, string + t.head + (size_t)k * t.w);
    else limb_hex(v, string + t.head + (size_t)k * t.w);
  }
  const size_t total = t.head + t.n * t.w;
  string[total] = '\0';
  if (t.len < total) string[digits + 1] = '\0';
  return t.len;
}

/* ---------------------------------------------------------------- decimal text on the device */

/* bigfloat_radix with the default (device tree) driver, leaving the digits
 * in device memory: the same plan, the same tree, and the same split of a top
 * limb above 10^9 (bigfloat/radix.c:351-357), whose low part is written back
 * into the device array.  Returns 0, or -1 when another driver is selected
 * (BC_RADIX_PERCALL, BC_RADIX_LEVELS), in which case nothing was done. */
int bigfloat_radix_device(bc_dec_device *d, const bigfloat_t a) {
  if (getenv("BC_RADIX_PERCALL") || getenv("BC_RADIX_LEVELS")) return -1;
  if (-a->exp + 1 != (int64_t)a->len) {
    fprintf(stderr, "Not implemented\n");
    abort();
  }
  size_t n = (size_t)(-a->exp);
  size_t k = (size_t)ceil((double)n * LOGR) - 1;
  double gd = ceil(log((double)k) / log(OLDBASE)) + 1;
  size_t g = (size_t)(gd > KT ? gd : KT);
  task_start(2, "Precomputing base conversion table");
  table_plan(&g_tab, k, g_steps);
  task_end(2);
  task_start(2, "Conversion");
  bc_host_ensure_gpu();
  void *dev = NULL;
  int rc = bc_gpu_device_alloc(k * sizeof(uint32_t), &dev);
  if (rc != BC_OK) {
    fprintf(stderr, "bigfloat_radix: %zu limbs of device memory: %s\n", k, bc_gpu_strerror(rc));
    abort();
  }
  convert_tree((uint32_t *)dev, k, a, n, g);
  task_end(2);
  table_free(&g_tab);
  uint32_t top = 0;
  if ((rc = bc_gpu_copy(&top, (uint32_t *)dev + (k - 1), 4)) != BC_OK) {
    fprintf(stderr, "bigfloat_radix: %s\n", bc_gpu_strerror(rc));
    abort();
  }
  d->dev = (uint32_t *)dev;
  d->len = k;
  if (top > NEWBASE) {
    const uint32_t lo = top % NEWBASE;
    if ((rc = bc_gpu_copy((uint32_t *)dev + (k - 1), &lo, 4)) != BC_OK) {
      fprintf(stderr, "bigfloat_radix: %s\n", bc_gpu_strerror(rc));
      abort();
    }
    top /= NEWBASE;
    d->len = k + 1;
  }
  d->top = top;
  d->exp = -(int64_t)d->len + 1;
  return 0;
}

/* The first bigfloat_to_string(s, value, digits, 10) bytes of the converted
 * value, written at the start of the open file fd: the head on the host, the
 * limbs' text rendered on the GPU from the device array
 * (bc_gpu_decimal_write).  Returns 0, or -1 when writing fails. */
int bc_dec_device_write(const bc_dec_device *d, size_t digits, int fd) {
  const text_plan t = plan_text(d->len, d->exp, d->top, digits, 10);
  const char head[2] = {t.head == 2 ? '2' : '.', '.'};
  const size_t hl = t.len < t.head ? t.len : t.head;
  if (hl && pwrite(fd, t.head == 2 ? head : head + 1, hl, 0) != (ssize_t)hl) return -1;
  if (t.len > t.head) {
    /* limbs c-1, c-2, ...: all below index len-1, inside the device array */
    const int rc = bc_gpu_decimal_write(d->dev, t.c - 1, t.n, t.len - t.head, fd, (long long)t.head);
    if (rc != BC_OK) {
      fprintf(stderr, "decimal output: %s\n", bc_gpu_strerror(rc));
      return -1;
    }
  }
  return 0;
}

void bc_dec_device_free(bc_dec_device *d) {
  if (d->dev) bc_gpu_device_free(d->dev);
  d->dev = NULL;
}
