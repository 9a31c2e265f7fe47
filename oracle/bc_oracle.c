/* bc_oracle.c — CPU restatement of the reference's FFT multiply path.
 *
 * TEST INFRASTRUCTURE ONLY (see bc_oracle.h): the checker, never the product.
 * Every function cites the reference file:line it restates.  The restatement
 * is plain C (no SIMD): the arithmetic is the same as the reference's SSE/AVX
 * code, written with C99 complex doubles.
 */
#define _GNU_SOURCE
#include "bc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------ sizes */

/* bigfloat/mul.c:109-124.  The reference subtracts 7 from a table that starts
 * at 20; it only has packers for 7..22 bits, so it aborts for CL > 4e6.  Here
 * the table continues (6..2 bits) as the documented extended oracle. */
int bco_width(size_t CL) {
  int b = 20;
  if (CL > 2000) b = 19;
  if (CL > 9000) b = 18;
  if (CL > 25000) b = 17;
  if (CL > 80000) b = 16;
  if (CL > 280000) b = 15;
  if (CL > 1000000) b = 14;
  if (CL > 4000000) b = 13;
  if (CL > 13000000) b = 12;
  if (CL > 50000000) b = 11;
  if (CL > 200000000) b = 10;
  if (CL > 800000000) b = 9;
  return b - 7;
}

/* fft/fft.c:22-41: smallest 2*2^k or 3*2^k that is >= n (5*2^k disabled). */
size_t bco_fft_length(size_t n) {
  size_t len = 1;
  for (;;) {
    if (2 * len >= n) return 2 * len;
    if (3 * len >= n) return 3 * len;
    len *= 2;
  }
}

/* ------------------------------------------------------------ packers */

/* Bits [pos, pos+b) of the little-endian word stream A[0..AL), zero beyond. */
static inline uint32_t bits_at(const uint32_t *A, size_t AL, uint64_t pos, int b) {
  size_t w = (size_t)(pos >> 5);
  unsigned s = (unsigned)(pos & 31);
  uint64_t v = 0;
  if (w < AL) v = A[w];
  if (w + 1 < AL) v |= (uint64_t)A[w + 1] << 32;
  return (uint32_t)((v >> s) & ((1ull << b) - 1));
}

/* fft/convert.c:45-80 + gen.rb:111-160: point i = bits [b*i, b*i+b) in the
 * real part; ceil(32*AL/b) points, then zeros up to length. */
size_t bco_int_to_fft(double complex *V, size_t length, const uint32_t *A, size_t AL, int b) {
  size_t npts = (size_t)((32 * (uint64_t)AL + (uint64_t)b - 1) / (uint64_t)b);
  for (size_t i = 0; i < npts; i++) V[i] = (double)bits_at(A, AL, (uint64_t)i * (uint64_t)b, b);
  for (size_t i = npts; i < length; i++) V[i] = 0.0;
  return npts;
}

/* fft/convert.c:83-111 + gen.rb:162-208.  `length` only sets the scale
 * 1/length (fft/convert.c:85); points are consumed until AL words are full.
 * The carry update keeps the generated code's `c += i` with i a double. */
void bco_fft_to_int(const double complex *T, size_t length, uint32_t *A, size_t AL, int b) {
  const double scale = 1.0 / (double)length;
  const uint64_t total_bits = 32 * (uint64_t)AL;
  uint64_t c = 0, pos = 0;
  uint64_t buf = 0;      /* pending output bits, LSB first */
  unsigned nbuf = 0;
  size_t w = 0;
  const uint64_t mask = (1ull << b) - 1;
  while (pos < total_bits) {
    double f = creal(*T++) * scale;
    double i = (double)(uint64_t)(f + 0.5);
    c = (uint64_t)((double)c + i);
    buf |= (c & mask) << nbuf;
    nbuf += (unsigned)b;
    c >>= b;
    pos += (uint64_t)b;
    while (nbuf >= 32 && w < AL) {
      A[w++] = (uint32_t)buf;
      buf >>= 32;
      nbuf -= 32;
    }
  }
  if (w < AL) A[w] = (uint32_t)buf; /* last partial word (not reached: 32*AL bits exact) */
}

/* ------------------------------------------------------------ transforms */

/* Twiddles e^{+2 pi i c / L} for c < L/2, computed like fft/table.c:189-209
 * (angle = (2*pi/L)*c in double, then cos/sin). */
static double complex *make_table(size_t L) {
  size_t h = L / 2;
  double complex *t = (double complex *)malloc((h ? h : 1) * sizeof(double complex));
  double omega = 2 * M_PI / (double)L;
  for (size_t c = 0; c < h; c++) {
    double a = omega * (double)c;
    t[c] = cos(a) + I * sin(a);
  }
  return t;
}

/* One table per recursion length, built lazily for the top call. */
typedef struct { double complex *tab[128]; size_t len[128]; int n; } tables_t;

static double complex *table_for(tables_t *ts, size_t L) {
  for (int i = 0; i < ts->n; i++) if (ts->len[i] == L) return ts->tab[i];
  ts->tab[ts->n] = make_table(L);
  ts->len[ts->n] = L;
  return ts->tab[ts->n++];
}

static void free_tables(tables_t *ts) {
  for (int i = 0; i < ts->n; i++) free(ts->tab[i]);
  ts->n = 0;
}

/* include/intrinsic.h:198-329 dft_3p: V1 = a + w b + w^2 c, w = e^{+2 pi i/3}. */
static void dft3(double complex *V, double sgn) {
  const double complex w1 = -0.5 + sgn * I * 0.8660254037844386467637231707529361834714026269051903140;
  const double complex w2 = conj(w1);
  double complex a = V[0], b = V[1], c = V[2];
  V[0] = a + b + c;
  V[1] = a + w1 * b + w2 * c;
  V[2] = a + w2 * b + w1 * c;
}

/* fft/fft.c:43-96: DIF, butterflies a+b, (a-b)*w, recurse on both halves. */
static void fwd_rec(tables_t *ts, double complex *T, size_t L) {
  if (L == 2) { double complex a = T[0], b = T[1]; T[0] = a + b; T[1] = a - b; return; }
  if (L == 3) { dft3(T, +1.0); return; }
  size_t h = L / 2;
  const double complex *w = table_for(ts, L);
  for (size_t c = 0; c < h; c++) {
    double complex a = T[c], b = T[c + h];
    T[c] = a + b;
    T[c + h] = (a - b) * w[c];
  }
  fwd_rec(ts, T, h);
  fwd_rec(ts, T + h, h);
}

/* fft/fft.c:289-329: DIT mirror with conjugate twiddles, no 1/N. */
static void inv_rec(tables_t *ts, double complex *T, size_t L) {
  if (L == 2) { double complex a = T[0], b = T[1]; T[0] = a + b; T[1] = a - b; return; }
  if (L == 3) { dft3(T, -1.0); return; }
  size_t h = L / 2;
  inv_rec(ts, T, h);
  inv_rec(ts, T + h, h);
  const double complex *w = table_for(ts, L);
  for (size_t c = 0; c < h; c++) {
    double complex a = T[c], b = T[c + h] * conj(w[c]);
    T[c] = a + b;
    T[c + h] = a - b;
  }
}

void bco_fft_forward(double complex *T, size_t n) {
  tables_t ts = {0};
  if (n == 1) return;
  fwd_rec(&ts, T, n);
  free_tables(&ts);
}

void bco_fft_inverse(double complex *T, size_t n) {
  tables_t ts = {0};
  if (n == 1) return;
  inv_rec(&ts, T, n);
  free_tables(&ts);
}

/* fft/pointwise.c:9-20. */
void bco_pointwise(double complex *a, const double complex *b, size_t n) {
  for (size_t i = 0; i < n; i++) a[i] *= b[i];
}

/* ------------------------------------------------------------ multiply */

/* Max |x - round(x)| over the first npts real parts after scaling. */
static double round_error(const double complex *T, size_t n, size_t npts) {
  double e = 0, s = 1.0 / (double)n;
  for (size_t i = 0; i < npts && i < n; i++) {
    double f = creal(T[i]) * s;
    double d = fabs(f - nearbyint(f));
    if (d > e) e = d;
  }
  return e;
}

/* bigfloat/mul.c:108-174: width from CL, length fft_length(32/b*CL), pack
 * both operands, forward transforms (one when AT==BT && AL==BL), pointwise
 * product or square, inverse, round and carry into CL words. */
double bco_fft_mul_width(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                         const uint32_t *BT, size_t BL, int b) {
  size_t length = bco_fft_length((size_t)(32.0 / b * (double)CL));
  int needB = (AT != BT || AL != BL);
  size_t na = (size_t)((32 * (uint64_t)AL + b - 1) / b);
  size_t nb = (size_t)((32 * (uint64_t)BL + b - 1) / b);
  size_t need = na > nb ? na : nb;
  size_t alloc = length > need ? length : need;
  size_t nout = (size_t)((32 * (uint64_t)CL + b - 1) / b);
  if (nout > alloc) alloc = nout;
  double complex *Ta = (double complex *)calloc(alloc, sizeof(double complex));
  double complex *Tb = needB ? (double complex *)calloc(alloc, sizeof(double complex)) : NULL;
  bco_int_to_fft(Ta, length, AT, AL, b);
  if (needB) bco_int_to_fft(Tb, length, BT, BL, b);
  tables_t ts = {0};
  fwd_rec(&ts, Ta, length);
  if (needB) fwd_rec(&ts, Tb, length);
  bco_pointwise(Ta, needB ? Tb : Ta, length);
  inv_rec(&ts, Ta, length);
  free_tables(&ts);
  double err = round_error(Ta, length, nout);
  bco_fft_to_int(Ta, length, CT, CL, b);
  free(Tb);
  free(Ta);
  return err;
}

int bco_fft_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                const uint32_t *BT, size_t BL) {
  int b = bco_width(CL);
  bco_fft_mul_width(CT, CL, AT, AL, BT, BL, b);
  return b;
}

/* bigfloat/mul.c:176-220: schoolbook with a 64-bit carry per row, low CL
 * words kept.  Writes through a temporary so CT may alias AT or BT. */
void bco_basecase_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                      const uint32_t *BT, size_t BL) {
  uint32_t *P = (uint32_t *)calloc(CL ? CL : 1, sizeof(uint32_t));
  for (size_t i = 0; i < AL && i < CL; i++) {
    uint64_t carry = 0;
    size_t j = 0;
    for (; j < BL && i + j < CL; j++) {
      uint64_t v = (uint64_t)P[i + j] + (uint64_t)AT[i] * BT[j] + carry;
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
  free(P);
}

/* ------------------------------------------------------------ exact NTT */
/* Own FP64-free exact multiply (not in the reference): 16-bit digits,
 * negacyclic-free cyclic NTT over p = 2^64 - 2^32 + 1 whose 2^32-th roots of
 * unity come from the generator 7.  Coefficients stay below
 * min(nA,nB) * 2^32 < p, so the convolution is exact. */

#define GL_P 0xFFFFFFFF00000001ull

static inline uint64_t gl_add(uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  if (s < a) s += 0xFFFFFFFFull;      /* 2^64 = 2^32 - 1 (mod p) */
  if (s >= GL_P) s -= GL_P;
  return s;
}
static inline uint64_t gl_sub(uint64_t a, uint64_t b) {
  return a >= b ? a - b : a + (GL_P - b);
}
static inline uint64_t gl_mul(uint64_t a, uint64_t b) {
  unsigned __int128 x = (unsigned __int128)a * b;
  uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  uint64_t hh = hi >> 32, hl = hi & 0xFFFFFFFFull;
  uint64_t t0 = lo - hh;               /* 2^96 = -1 (mod p) */
  if (lo < hh) t0 -= 0xFFFFFFFFull;
  uint64_t t1 = hl * 0xFFFFFFFFull;    /* 2^64 = 2^32 - 1 (mod p) */
  uint64_t r = t0 + t1;
  if (r < t1) r += 0xFFFFFFFFull;
  if (r >= GL_P) r -= GL_P;
  return r;
}
static uint64_t gl_pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) { if (e & 1) r = gl_mul(r, a); a = gl_mul(a, a); e >>= 1; }
  return r;
}

static void ntt_dif(uint64_t *a, size_t N, const uint64_t *tw) {
  for (size_t len = N; len >= 2; len >>= 1) {
    size_t h = len / 2, step = N / len;
    #pragma omp parallel for schedule(static) if (N >= (1u << 16))
    for (size_t bidx = 0; bidx < N / 2; bidx++) {
      size_t s = (bidx / h) * len, j = bidx % h;
      uint64_t u = a[s + j], v = a[s + j + h];
      a[s + j] = gl_add(u, v);
      a[s + j + h] = gl_mul(gl_sub(u, v), tw[j * step]);
    }
  }
}

static void ntt_dit(uint64_t *a, size_t N, const uint64_t *tw) {
  for (size_t len = 2; len <= N; len <<= 1) {
    size_t h = len / 2, step = N / len;
    #pragma omp parallel for schedule(static) if (N >= (1u << 16))
    for (size_t bidx = 0; bidx < N / 2; bidx++) {
      size_t s = (bidx / h) * len, j = bidx % h;
      uint64_t u = a[s + j], v = gl_mul(a[s + j + h], tw[j * step]);
      a[s + j] = gl_add(u, v);
      a[s + j + h] = gl_sub(u, v);
    }
  }
}

int bco_ntt_mul(uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                const uint32_t *BT, size_t BL) {
  if (CL == 0) return 0;
  if (AL > CL) AL = CL;
  if (BL > CL) BL = CL;
  size_t nA = 2 * AL, nB = 2 * BL;
  size_t ncoef = nA + nB - 1;
  size_t N = 1;
  while (N < ncoef) N <<= 1;
  if (N > (1ull << 31)) return -1;
  uint64_t *a = (uint64_t *)calloc(N, 8), *b = (uint64_t *)calloc(N, 8);
  uint64_t *tw = (uint64_t *)malloc((N / 2 + 1) * 8), *itw = (uint64_t *)malloc((N / 2 + 1) * 8);
  if (!a || !b || !tw || !itw) { free(a); free(b); free(tw); free(itw); return -1; }
  for (size_t i = 0; i < AL; i++) { a[2 * i] = AT[i] & 0xFFFF; a[2 * i + 1] = AT[i] >> 16; }
  for (size_t i = 0; i < BL; i++) { b[2 * i] = BT[i] & 0xFFFF; b[2 * i + 1] = BT[i] >> 16; }
  uint64_t w = gl_pow(7, (GL_P - 1) / N), iw = gl_pow(w, GL_P - 2);
  tw[0] = itw[0] = 1;
  for (size_t j = 1; j < N / 2 + 1; j++) { tw[j] = gl_mul(tw[j - 1], w); itw[j] = gl_mul(itw[j - 1], iw); }
  ntt_dif(a, N, tw);
  ntt_dif(b, N, tw);
  #pragma omp parallel for schedule(static) if (N >= (1u << 16))
  for (size_t i = 0; i < N; i++) a[i] = gl_mul(a[i], b[i]);
  ntt_dit(a, N, itw);
  uint64_t ninv = gl_pow(N % GL_P, GL_P - 2);
  unsigned __int128 acc = 0;
  size_t need = 2 * CL;
  uint32_t half[2];
  for (size_t i = 0; i < need; i++) {
    if (i < ncoef) acc += gl_mul(a[i], ninv);
    half[i & 1] = (uint32_t)(acc & 0xFFFF);
    acc >>= 16;
    if (i & 1) CT[i / 2] = half[0] | (half[1] << 16);
  }
  free(a); free(b); free(tw); free(itw);
  return 0;
}

/* ------------------------------------------------------------ checksums */

/* bigfloat/mul.c:21-34 (checksum) with the prime as a parameter. */
uint32_t bco_checksum(const uint32_t *AT, size_t AL, uint32_t p) {
  uint64_t base = 1, sum = 0, prime = p;
  for (size_t i = 0; i < AL; i++) {
    sum = (sum + ((uint64_t)AT[i] * base) % prime) % prime;
    base = (base << 32) % prime;
  }
  return (uint32_t)sum;
}

static const uint32_t kPrimes[8] = {
  0x9f063b05u,            /* CHECKPRIME, bigfloat/mul.c:19 */
  4294967291u, 4294967279u, 4294967231u, 4294967197u, 4294967189u,
  4294967161u, 4294967143u,
};

/* bigfloat/mul.c:650-658 (DEBUG check cs(C) == cs(A)*cs(B)), several primes. */
int bco_modcheck(const uint32_t *CT, size_t CL, const uint32_t *AT, size_t AL,
                 const uint32_t *BT, size_t BL, int nprimes) {
  if (nprimes > 8) nprimes = 8;
  for (int k = 0; k < nprimes; k++) {
    uint32_t p = kPrimes[k];
    uint64_t ca = bco_checksum(AT, AL, p), cb = bco_checksum(BT, BL, p);
    uint64_t cc = bco_checksum(CT, CL, p);
    if ((ca * cb) % p != cc) return 0;
  }
  return 1;
}
