/* e.c — e = sum 1/k! to N decimal digits (the reference's main.c:38-167).
 *
 * Binary splitting P(a,b), Q(a,b): leaves P = 1, Q = b; a node combines its
 * halves (split at m = (a+b)/2) as P = P0*Q1 + P1, Q = Q0*Q1
 * (main.c:63-109).  Then e = 1 + P/Q by Newton division at p limbs
 * (main.c:131-140), hex output, radix conversion and decimal output
 * (main.c:143-166).
 *
 * Two drivers for the splitting tree, same values:
 *   mode 0  the reference's recursion, one product per GPU call;
 *   mode 1  level order: subtrees of at most LEAF_TERMS terms run the same
 *           recursion on host threads (all their products are below 100
 *           limbs, the reference's host range), and every level above them
 *           multiplies all of its 2*nodes products in one bigfloat_mul_batch;
 *   mode 2  the whole tree in device memory (bc_gpu_e_series): P and Q
 *           cross to the host once, at the root.
 * P and Q are the same integers in every mode (they do not depend on where
 * ranges split) and come out exponent 0 with no top zero limbs, as the
 * reference's products and additions leave them.
 *
 * The hex digits are formatted and written on a host thread while the
 * radix conversion runs (it only reads e, as the conversion does); the
 * "Writing hex digits" phase reports what is left of it afterwards.  With
 * the default conversion driver the decimal digits never reach host memory
 * as numbers: the conversion leaves them in device memory, their text is
 * rendered there and written to e.txt straight from the pinned staging
 * buffers (bigfloat_radix_device, bc_dec_device_write), the same bytes as
 * bigfloat_to_string would give.
 */
#include <fcntl.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "bc_gpu.h"
#include "bc_host.h"
#include "bench.h"
#include "bigfloat.h"

/* main.c:38-61: terms so that log(terms!) exceeds p limbs of precision. */
static size_t e_terms(size_t p) {
  long double sizeL = (long double)p * logl(4294967296.0L) + 1;
  size_t a = 0, b = 1;
  while (lgammal((long double)b) < sizeL) b *= 2;
  while (b - a > 1) {
    size_t m = (a + b) / 2;
    if (lgammal((long double)m) < sizeL) a = m;
    else b = m;
  }
  return b + 2;
}

/* main.c:63-109 without the DEBUG timers. */
static void bsr(bigfloat_t P, bigfloat_t Q, uint32_t a, uint32_t b) {
  if (b - a == 1) {
    bigfloat_set(P, 1);
    bigfloat_set(Q, b);
    return;
  }
  uint32_t m = (a + b) / 2;
  bigfloat_t P0, Q0, P1, Q1, t;
  bigfloat_new(P0); bigfloat_new(Q0); bigfloat_new(P1); bigfloat_new(Q1); bigfloat_new(t);
  bsr(P0, Q0, a, m);
  bsr(P1, Q1, m, b);
  bigfloat_mul(t, P0, Q1, 0);
  bigfloat_free(P0);
  bigfloat_add(P, t, P1, 0);
  bigfloat_free(t);
  bigfloat_free(P1);
  bigfloat_mul(Q, Q0, Q1, 0);
  bigfloat_free(Q1);
  bigfloat_free(Q0);
}

/* Subtrees of this many terms or fewer stay on host threads: their P and Q
 * stay below 64 limbs for up to 2^32 terms, so every product is < 100 limbs. */
#define LEAF_TERMS 64

typedef struct {
  uint32_t a, b;
  int c0, c1;           /* children in the next level, -1 if computed on the host */
  _bigfloat_struct P, Q;
} bnode;

static double wall_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* mode 2: the series on the GPU, the root's P and Q back as bigfloats. */
static void bsr_device(bigfloat_t P, bigfloat_t Q, uint32_t a, uint32_t b) {
  double t0 = wall_s();
  bc_host_ensure_gpu();
  if (getenv("BC_STATS")) printf("    GPU engine start: %.3f s\n", wall_s() - t0);
  uint32_t *p = NULL, *q = NULL;
  size_t pl = 0, ql = 0;
  t0 = wall_s();
  int rc = bc_gpu_e_series(a, b, &p, &pl, &q, &ql);
  if (rc != BC_OK) {
    fprintf(stderr, "bluecrunch: binary splitting on the GPU failed: %s\n", bc_gpu_strerror(rc));
    abort();
  }
  if (getenv("BC_STATS")) printf("    binary splitting on the GPU: %.3f s\n", wall_s() - t0);
  free(P->coef);
  P->coef = p; P->len = pl; P->exp = 0; P->sign = 1;
  free(Q->coef);
  Q->coef = q; Q->len = ql; Q->exp = 0; Q->sign = 1;
}

static void bsr_levels(bigfloat_t P, bigfloat_t Q, uint32_t a0, uint32_t b0) {
  const int stats = getenv("BC_STATS") != NULL;
  double t_leaf = 0, t_mul = 0, t_add = 0, t0 = wall_s();
  /* top-down: the tree above the host subtrees, one array per depth */
  bnode **lv = (bnode **)bc_xmalloc(sizeof(bnode *));
  size_t *cnt = (size_t *)bc_xmalloc(sizeof(size_t));
  lv[0] = (bnode *)calloc(1, sizeof(bnode));
  lv[0][0].a = a0;
  lv[0][0].b = b0;
  cnt[0] = 1;
  int nlv = 1;
  for (;;) {
    bnode *L = lv[nlv - 1];
    size_t m = cnt[nlv - 1], nin = 0;
    for (size_t i = 0; i < m; i++) nin += (L[i].b - L[i].a) > LEAF_TERMS;
    if (!nin) break;
    bnode *N = (bnode *)calloc(2 * nin, sizeof(bnode));
    size_t c = 0;
    for (size_t i = 0; i < m; i++) {
      bnode *x = &L[i];
      x->c0 = x->c1 = -1;
      if (x->b - x->a <= LEAF_TERMS) continue;
      uint32_t mid = (x->a + x->b) / 2;
      N[c].a = x->a; N[c].b = mid; x->c0 = (int)c++;
      N[c].a = mid; N[c].b = x->b; x->c1 = (int)c++;
    }
    lv = (bnode **)bc_xrealloc(lv, (size_t)(nlv + 1) * sizeof(bnode *));
    cnt = (size_t *)bc_xrealloc(cnt, (size_t)(nlv + 1) * sizeof(size_t));
    lv[nlv] = N;
    cnt[nlv] = c;
    nlv++;
  }
  /* host subtrees (every level may hold some), in parallel */
  for (int d = 0; d < nlv; d++) {
    bnode *L = lv[d];
    long m = (long)cnt[d];
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < m; i++) {
      bnode *x = &L[i];
      if (x->b - x->a > LEAF_TERMS) continue;
      bigfloat_new(&x->P);
      bigfloat_new(&x->Q);
      bsr(&x->P, &x->Q, x->a, x->b);
    }
  }
  t_leaf = wall_s() - t0;
  /* bottom-up: one batch of 2 products per internal node, then the adds */
  for (int d = nlv - 2; d >= 0; d--) {
    bnode *L = lv[d], *N = lv[d + 1];
    size_t m = cnt[d], q = 0;
    for (size_t i = 0; i < m; i++) q += L[i].c0 >= 0;
    bigfloat_mul_item *it = (bigfloat_mul_item *)bc_xmalloc(2 * q * sizeof(bigfloat_mul_item));
    _bigfloat_struct *tmp = (_bigfloat_struct *)calloc(q ? q : 1, sizeof(_bigfloat_struct));
    size_t j = 0;
    for (size_t i = 0; i < m; i++) {
      bnode *x = &L[i];
      if (x->c0 < 0) continue;
      bnode *l = &N[x->c0], *r = &N[x->c1];
      bigfloat_new(&tmp[j / 2]);
      bigfloat_new(&x->P);
      bigfloat_new(&x->Q);
      it[j].target = &tmp[j / 2]; it[j].a = &l->P; it[j].b = &r->Q; it[j].p = 0; j++;  /* P0*Q1 */
      it[j].target = &x->Q;       it[j].a = &l->Q; it[j].b = &r->Q; it[j].p = 0; j++;  /* Q0*Q1 */
    }
    t0 = wall_s();
    bigfloat_mul_batch(it, j);
    t_mul += wall_s() - t0;
    t0 = wall_s();
    free(it);
    long mm = (long)m;
    j = 0;
    size_t *slot = (size_t *)bc_xmalloc((m ? m : 1) * sizeof(size_t));
    for (size_t i = 0; i < m; i++) { slot[i] = j; j += L[i].c0 >= 0; }
#pragma omp parallel for schedule(dynamic, 16) if (mm >= 64)  /* few big nodes: their adds run in parallel inside */
    for (long i = 0; i < mm; i++) {
      bnode *x = &L[i];
      if (x->c0 < 0) continue;
      bnode *l = &N[x->c0], *r = &N[x->c1];
      bigfloat_add(&x->P, &tmp[slot[i]], &r->P, 0);   /* P = P0*Q1 + P1 */
      bigfloat_free(&tmp[slot[i]]);
      bigfloat_free(&l->P); bigfloat_free(&l->Q); bigfloat_free(&r->P); bigfloat_free(&r->Q);
    }
    free(slot);
    free(tmp);
    free(N);
    t_add += wall_s() - t0;
  }
  if (stats)
    printf("    binary splitting: host subtrees %.3f s, level products %.3f s, adds and frees %.3f s\n", t_leaf,
           t_mul, t_add);
  free(P->coef);
  free(Q->coef);
  *P = lv[0][0].P;
  *Q = lv[0][0].Q;
  free(lv[0]);
  free(lv);
  free(cnt);
}

static int dump(const char *dir, const char *name, const char *s, size_t len);

typedef struct {
  const _bigfloat_struct *x;
  size_t digits;
  const char *outdir;
  int rc;
} hex_job;

static void *hex_writer(void *arg) {
  hex_job *j = (hex_job *)arg;
  char *out = (char *)bc_xmalloc(j->digits + 22);
  size_t len = bigfloat_to_string(out, j->x, j->digits, 16);
  j->rc = dump(j->outdir, "e-hex.txt", out, len);
  free(out);
  return NULL;
}

/* Outputs of 64 MiB and more are written by several threads, each with
 * pwrite at its own offset (the copy into the page cache is most of the
 * time of a gigabyte-sized write). */
static int dump(const char *dir, const char *name, const char *s, size_t len) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir ? dir : ".", name);
  if (len >= ((size_t)64 << 20)) {
    const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) {
      fprintf(stderr, "Cannot create file %s\n", path);
      return -1;
    }
    const long nch = 16;
    const size_t chunk = (len + (size_t)nch - 1) / (size_t)nch;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (long h = 0; h < nch; h++) {
      size_t off = (size_t)h * chunk;
      const size_t end = off + chunk < len ? off + chunk : len;
      while (off < end) {
        const ssize_t w = pwrite(fd, s + off, end - off, (off_t)off);
        if (w <= 0) {
          bad = 1;
          break;
        }
        off += (size_t)w;
      }
    }
    if (close(fd) != 0 || bad) {
      fprintf(stderr, "Cannot write file %s\n", path);
      return -1;
    }
    return 0;
  }
  FILE *f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "Cannot create file %s\n", path);
    return -1;
  }
  fwrite(s, 1, len, f);
  fclose(f);
  return 0;
}

/* The decimal text of a conversion held in device memory, as dump() would
 * write bigfloat_to_string's output for it. */
static int dump_device(const char *dir, const char *name, const bc_dec_device *d, size_t digits) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir ? dir : ".", name);
  const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) {
    fprintf(stderr, "Cannot create file %s\n", path);
    return -1;
  }
  const int bad = bc_dec_device_write(d, digits, fd);
  if (close(fd) != 0 || bad) {
    fprintf(stderr, "Cannot write file %s\n", path);
    return -1;
  }
  return 0;
}

/* main.c:111-167 */
int bluecrunch_e(size_t digits, int mode, const char *outdir) {
  digits++;  /* the leading 2 does not count */
  size_t p = (digits + 8) / 9;
  size_t terms = e_terms(p);
  if ((uint32_t)terms != terms) {
    fprintf(stderr, "Limit Exceeded");
    return -1;
  }
  /* the GPU engine first, in a phase of its own: opening the device (driver
   * and context start) takes from under one to several seconds on a fresh
   * process, and would otherwise land in the first phase that multiplies.
   * Below 100 limbs every product stays on the host (as in the reference),
   * and the engine starts only if one is needed after all. */
  if (p >= 100) {
    task_start(1, "Starting GPU engine");
    bc_host_ensure_gpu();
    task_end(1);
  }
  task_start(1, "Summing");
  bigfloat_t P, Q;
  bigfloat_new(P);
  bigfloat_new(Q);
  if (mode == 2) bsr_device(P, Q, 0, (uint32_t)terms);
  else if (mode == 1) bsr_levels(P, Q, 0, (uint32_t)terms);
  else bsr(P, Q, 0, (uint32_t)terms);
  task_end(1);

  const int stats = getenv("BC_STATS") != NULL;
  if (stats)
    printf("    P: %zu limbs, top %08x; Q: %zu limbs, top %08x\n", P->len, P->len ? P->coef[P->len - 1] : 0,
           Q->len, Q->len ? Q->coef[Q->len - 1] : 0);
  task_start(1, "Dividing");
  bigfloat_t one, tmp;
  bigfloat_new(one);
  bigfloat_set(one, 1);
  bigfloat_new(tmp);
  bigfloat_div(tmp, P, Q, p);
  if (stats)
    printf("    P/Q: %zu limbs, exp %lld, top %08x\n", tmp->len, (long long)tmp->exp,
           tmp->len ? tmp->coef[tmp->len - 1] : 0);
  bigfloat_free(Q);
  bigfloat_add(P, tmp, one, p);
  bigfloat_free(tmp);
  bigfloat_free(one);
  task_end(1);

  size_t out_len = digits + 2;
  hex_job hj = {P, out_len, outdir, 0};
  pthread_t hex_thread;
  const int hex_async = pthread_create(&hex_thread, NULL, hex_writer, &hj) == 0;
  if (!hex_async) hex_writer(&hj);

  /* the default conversion leaves its digits in device memory, and their
   * text is rendered there and written straight from the staging buffers;
   * the other conversion drivers print on the host */
  task_start(1, "Converting to decimal");
  fflush(stdout);
  bigfloat_t dec;
  bigfloat_new(dec);
  bc_dec_device dd = {NULL, 0, 0, 0};
  const int on_device = bigfloat_radix_device(&dd, P) == 0;
  if (!on_device) bigfloat_radix(dec, P);
  task_end(1);

  task_start(1, "Writing hex digits");
  if (hex_async) pthread_join(hex_thread, NULL);
  int rc = hj.rc;
  task_end(1);

  task_start(1, "Writing decimal digits");
  if (on_device) {
    rc |= dump_device(outdir, "e.txt", &dd, out_len);
    bc_dec_device_free(&dd);
  } else {
    char *out = (char *)bc_xmalloc(out_len + 22);
    size_t len = bigfloat_to_string(out, dec, out_len, 10);
    rc |= dump(outdir, "e.txt", out, len);
    free(out);
  }
  bigfloat_free(P);
  bigfloat_free(dec);
  task_end(1);
  return rc;
}
