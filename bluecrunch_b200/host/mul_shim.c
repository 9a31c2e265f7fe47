/* mul_shim.c — the reference's multiply entry points (include/mul.h) on top
 * of libbcgpu.
 *
 * _fft_mul keeps the prototype of bigfloat/mul.c:108 and its contract
 * (exactly CL limbs of A*B mod 2^(32 CL), CT may alias AT or BT, no status
 * return) but runs on the GPU.  The engine is initialised on first use; a
 * failure is reported on stderr and aborts, as the reference aborts on the
 * widths it cannot handle (fft/convert.c:66-68).  There is no CPU fallback.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>

#include "bc_gpu.h"
#include "bc_host.h"
#include "bigfloat.h"
#include "mul.h"

static pthread_once_t g_once = PTHREAD_ONCE_INIT;
static int g_init_rc = 0;
static bigfloat_mul_counters g_cnt;
static unsigned long long g_device_us;
static pthread_mutex_t g_cnt_mu = PTHREAD_MUTEX_INITIALIZER;

/* Blocks of 32 MiB and more (limb arrays of long operands) start on a 2 MiB
 * boundary and are advised for transparent huge pages: their first touch
 * then faults once per 2 MiB instead of once per 4 KiB, which is most of the
 * cost of writing a fresh result of 10^8 limbs.  They stay ordinary malloc
 * blocks (free() releases them). */
#define BC_BIG_BLOCK ((size_t)32 << 20)
#define BC_HUGE_PAGE ((size_t)2 << 20)
void *bc_xmalloc(size_t n) {
  void *p = NULL;
  if (n >= BC_BIG_BLOCK) {
    if (posix_memalign(&p, BC_HUGE_PAGE, n) != 0) p = NULL;
    if (p) madvise(p, n & ~(BC_HUGE_PAGE - 1), MADV_HUGEPAGE);
  } else {
    p = malloc(n ? n : 1);
  }
  if (!p) {
    fprintf(stderr, "bluecrunch: out of host memory (%zu bytes)\n", n);
    abort();
  }
  return p;
}

void *bc_xrealloc(void *p, size_t n) {
  void *q = realloc(p, n ? n : 1);
  if (!q) {
    fprintf(stderr, "bluecrunch: out of host memory (%zu bytes)\n", n);
    abort();
  }
  return q;
}

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * t.tv_nsec;
}

/* Width table: $BC_TUNE_FILE, else tune/widths.txt next to this library. */
static void init_once(void) {
  static char path[4096];
  bc_gpu_config cfg;
  memset(&cfg, 0, sizeof cfg);
  const char *env = getenv("BC_TUNE_FILE");
  if (env) {
    cfg.tune_path = env;
  } else {
    Dl_info info;
    if (dladdr((void *)&init_once, &info) && info.dli_fname) {
      snprintf(path, sizeof path, "%s", info.dli_fname);
      char *slash = strrchr(path, '/');
      if (slash) {
        snprintf(slash + 1, sizeof path - (size_t)(slash + 1 - path), "tune/widths.txt");
        cfg.tune_path = path;
      }
    }
  }
  const char *dev = getenv("BC_DEVICE");
  cfg.device = dev ? atoi(dev) : 0;
  g_init_rc = bc_gpu_init(&cfg);
}

void bc_host_ensure_gpu(void) {
  pthread_once(&g_once, init_once);
  if (g_init_rc != BC_OK) {
    fprintf(stderr, "bluecrunch: GPU engine unavailable: %s\n", bc_gpu_strerror(g_init_rc));
    abort();
  }
}

/* Optional FP64-free check of every GPU product (BC_VERIFY=1): A*B mod p for
 * the reference's CHECKPRIME 0x9f063b05 and a second 32-bit prime, as the
 * reference's DEBUG build checks every FFT product (bigfloat/mul.c:650-658).
 * Only meaningful when CL >= AL+BL, which bigfloat_mul always passes. */
static uint32_t residue(const uint32_t *T, size_t L, uint64_t p) {
  uint64_t r = 0;
  const uint64_t base = ((uint64_t)1 << 32) % p;
  for (size_t i = L; i-- > 0;) r = ((r * base) % p + T[i] % p) % p;
  return (uint32_t)r;
}

static int verify_on(void) {
  static int v = -1;
  if (v < 0) v = getenv("BC_VERIFY") != NULL;
  return v;
}

/* 0 when C = A*B passes the check modulo both primes (or cannot be checked,
 * CL < AL+BL), else the failing prime. */
uint64_t bc_host_product_check(const uint32_t *C, size_t CL, const uint32_t *A, size_t AL, const uint32_t *B,
                               size_t BL) {
  static const uint64_t primes[2] = {0x9f063b05u, 4294967291u};
  if (CL < AL + BL) return 0;
  for (int k = 0; k < 2; k++) {
    uint64_t p = primes[k];
    uint64_t want = ((uint64_t)residue(A, AL, p) * residue(B, BL, p)) % p;
    if (want != residue(C, CL, p)) return p;
  }
  return 0;
}

static void verify(const uint32_t *C, size_t CL, const uint32_t *A, size_t AL, const uint32_t *B, size_t BL) {
  const uint64_t p = bc_host_product_check(C, CL, A, AL, B, BL);
  if (p) {
    fprintf(stderr, "bluecrunch: GPU product fails the modular check (AL=%zu BL=%zu CL=%zu prime %llx)\n", AL, BL,
            CL, (unsigned long long)p);
    abort();
  }
}

/* Fault injection on the host, for tests of the check above:
 * BC_FAULT_FLIP_PRODUCT=k flips one bit of the k-th GPU product's result
 * (counting _fft_mul calls from 1) after the GPU has returned it and before
 * the check runs.  Unset: no effect. */
static void maybe_flip(uint32_t *C, size_t CL) {
  static long target = -1;
  static unsigned long calls = 0;
  if (target < 0) {
    const char *e = getenv("BC_FAULT_FLIP_PRODUCT");
    target = e ? atol(e) : 0;
  }
  if (target <= 0) return;
  if (__atomic_add_fetch(&calls, 1, __ATOMIC_RELAXED) == (unsigned long)target && CL) C[CL / 2] ^= 1u;
}

static void count(size_t products, size_t calls, double secs) {
  pthread_mutex_lock(&g_cnt_mu);
  g_cnt.gpu_products += products;
  g_cnt.gpu_calls += calls;
  g_cnt.gpu_seconds += secs;
  pthread_mutex_unlock(&g_cnt_mu);
}

int _fft_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  bc_host_ensure_gpu();
  bc_mul_stats st;
  double t0 = now_s();
  int rc = bc_gpu_mul(CT, CL, AT, AL, BT, BL, &st);
  count(1, 1, now_s() - t0);
  if (rc != BC_OK) {
    fprintf(stderr, "_fft_mul: GPU multiply failed (CL=%zu): %s\n", CL, bc_gpu_strerror(rc));
    abort();
  }
  maybe_flip(CT, CL);
  if (verify_on() && CT != AT && CT != BT) verify(CT, CL, AT, AL, BT, BL);
  return st.width;
}

void bc_host_gpu_batch(bc_gpu_item *items, size_t n) {
  bc_host_ensure_gpu();
  bc_mul_desc *d = (bc_mul_desc *)bc_xmalloc(n * sizeof(bc_mul_desc));
  for (size_t i = 0; i < n; i++) {
    d[i].C = items[i].C; d[i].CL = items[i].CL;
    d[i].A = items[i].A; d[i].AL = items[i].AL;
    d[i].B = items[i].B; d[i].BL = items[i].BL;
  }
  bc_batch_stats st;
  double t0 = now_s();
  int rc = bc_gpu_mul_batch_flags(d, n, BC_BATCH_HOST_OPERANDS, &st);
  count(n, 1, now_s() - t0);
  __atomic_add_fetch(&g_device_us, (unsigned long long)(st.device_ms * 1000.0), __ATOMIC_RELAXED);
  free(d);
  if (rc != BC_OK) {
    fprintf(stderr, "bigfloat_mul_batch: GPU batch of %zu products failed: %s\n", n, bc_gpu_strerror(rc));
    abort();
  }
  if (verify_on())
    for (size_t i = 0; i < n; i++) verify(items[i].C, items[i].CL, items[i].A, items[i].AL, items[i].B, items[i].BL);
}

/* Small products (fewer than BC_SMALL_PRODUCT_LIMBS output limbs) of a batch
 * on the GPU in one launch (bc_gpu_mul_small_batch); aborts with a message on
 * failure.  C must not alias A or B (bigfloat_mul_batch writes fresh arrays). */
void bc_host_gpu_small_batch(bc_gpu_item *items, size_t n) {
  bc_host_ensure_gpu();
  bc_mul_desc *d = (bc_mul_desc *)bc_xmalloc(n * sizeof(bc_mul_desc));
  for (size_t i = 0; i < n; i++) {
    d[i].C = items[i].C; d[i].CL = items[i].CL;
    d[i].A = items[i].A; d[i].AL = items[i].AL;
    d[i].B = items[i].B; d[i].BL = items[i].BL;
  }
  double t0 = now_s();
  int rc = bc_gpu_mul_small_batch(d, n);
  count(n, 1, now_s() - t0);
  free(d);
  if (rc != BC_OK) {
    fprintf(stderr, "bigfloat_mul_batch: GPU batch of %zu small products failed: %s\n", n, bc_gpu_strerror(rc));
    abort();
  }
  if (verify_on())
    for (size_t i = 0; i < n; i++) verify(items[i].C, items[i].CL, items[i].A, items[i].AL, items[i].B, items[i].BL);
}

/* Exact schoolbook product of the low CL limbs (the value the reference's
 * _basecase_mul, bigfloat/mul.c:176-220, and _karatzuba_mul, :367-553,
 * produce).  Works through a temporary so CT may alias AT or BT. */
void bc_small_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL, const uint32_t *BT, size_t BL) {
  uint32_t stackbuf[256];
  uint32_t *P = CL <= 256 ? stackbuf : (uint32_t *)bc_xmalloc(CL * sizeof(uint32_t));
  memset(P, 0, CL * sizeof(uint32_t));
  for (size_t i = 0; i < AL && i < CL; i++) {
    uint64_t carry = 0;
    const uint64_t ai = AT[i];
    size_t j = 0;
    for (; j < BL && i + j < CL; j++) {
      uint64_t v = (uint64_t)P[i + j] + ai * BT[j] + carry;
      P[i + j] = (uint32_t)v;
      carry = v >> 32;
    }
    for (size_t k = i + j; k < CL && carry; k++) {
      uint64_t v = (uint64_t)P[k] + carry;
      P[k] = (uint32_t)v;
      carry = v >> 32;
    }
  }
  memcpy(CT, P, CL * sizeof(uint32_t));
  if (P != stackbuf) free(P);
  __atomic_add_fetch(&g_cnt.small_products, 1, __ATOMIC_RELAXED);
}

void _basecase_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  bc_small_mul(CT, CL, AT, AL, BT, BL);
}

void _karatzuba_mul(uint32_t *CT, size_t CL, uint32_t *AT, size_t AL, uint32_t *BT, size_t BL) {
  bc_small_mul(CT, CL, AT, AL, BT, BL);
}

void bigfloat_get_counters(bigfloat_mul_counters *out) {
  pthread_mutex_lock(&g_cnt_mu);
  *out = g_cnt;
  out->gpu_kernel_seconds = 1e-6 * (double)__atomic_load_n(&g_device_us, __ATOMIC_RELAXED);
  pthread_mutex_unlock(&g_cnt_mu);
}

void bigfloat_reset_counters(void) {
  pthread_mutex_lock(&g_cnt_mu);
  memset(&g_cnt, 0, sizeof g_cnt);
  __atomic_store_n(&g_device_us, 0, __ATOMIC_RELAXED);
  pthread_mutex_unlock(&g_cnt_mu);
}
