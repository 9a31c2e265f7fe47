/* bc_gpu.h — C ABI of libbcgpu, the B200 (sm_100a) exact multiply engine.
 *
 * The library computes exact products of little-endian base-2^32 integers
 * (the limb format of bigfloat_t, include/bigfloat.h:6-13 in the reference)
 * with an FP64 FFT convolution on one GPU.  It is what the reference's
 * _fft_mul (include/mul.h:3, bigfloat/mul.c:108-174) becomes when it crosses
 * to the device: include/mul.h in this repository keeps that prototype and
 * forwards to bc_gpu_mul; batched tree levels use bc_gpu_mul_batch.
 *
 * All functions return BC_OK (0) or a negative BC_ERR_* code; nothing aborts.
 * Pointers may be host memory or device memory of the selected GPU; the
 * library detects which.  Calls are serialised internally (re-entrant).
 */
#ifndef BC_GPU_H
#define BC_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  BC_OK = 0,
  BC_ERR_INVALID = -1,     /* bad argument (null pointer with nonzero length, ...) */
  BC_ERR_NOMEM = -2,       /* device memory could not be reserved */
  BC_ERR_CUDA = -3,        /* a CUDA runtime call failed (see bc_gpu_last_cuda_error) */
  BC_ERR_TIMEOUT = -4,     /* carry lookback gave up waiting (bounded spin ran out) */
  BC_ERR_PRECISION = -5,   /* rounding error stayed >= the limit down to the minimum width */
  BC_ERR_NOT_INIT = -6,    /* bc_gpu_init has not succeeded */
  BC_ERR_TOO_LARGE = -7,   /* product needs a transform longer than supported (2^30 points) */
  BC_ERR_NO_DEVICE = -8,   /* no usable sm_100 device */
  BC_ERR_CARRY = -9,       /* carry out of the top word of an exact product (internal check) */
  BC_ERR_IO = -10          /* writing an output file failed (bc_gpu_decimal_write) */
};

/* Configuration for bc_gpu_init; a NULL pointer means all defaults. */
typedef struct {
  int device;             /* CUDA device ordinal (default 0) */
  size_t arena_bytes;     /* device work arena cap; 0 = 90% of free memory at init */
  const char *tune_path;  /* width table file (bc_tune format); NULL = built-in/env BC_TUNE_FILE */
  double max_round_err;   /* retry threshold on max |x - round(x)| (default 0.25) */
  int verbose;            /* 1: print plans and retries to stderr */
} bc_gpu_config;

/* Per-product statistics (optional out-parameter). */
typedef struct {
  int width;              /* bits per balanced digit actually used */
  int retries;            /* times the product was redone at a narrower width */
  size_t fft_points;      /* complex transform length M (2M real coefficients) */
  double max_round_err;   /* max |x - round(x)| over all 2M coefficients */
  double device_ms;       /* GPU time of the kernels (CUDA events) */
  double total_ms;        /* wall time of the call including copies */
} bc_mul_stats;

/* One independent product of a batch.  C receives exactly CL words of
 * A*B mod 2^(32*CL).  C may alias its own A or B (all inputs are read before
 * any output is written); items must not alias each other's outputs. */
typedef struct {
  uint32_t *C;
  size_t CL;
  const uint32_t *A;
  size_t AL;
  const uint32_t *B;
  size_t BL;
} bc_mul_desc;

typedef struct {
  size_t items;
  size_t classes;         /* distinct transform shapes launched */
  size_t launches;        /* kernel launches issued (per attempt) */
  int retries;            /* items redone at a narrower width */
  double max_round_err;
  double device_ms;       /* GPU time of the kernels */
  double total_ms;        /* wall time including copies */
  size_t h2d_bytes, d2h_bytes;
  size_t graph_launches;  /* CUDA graph launches (BC_BATCH_GRAPH; per attempt) */
  size_t graph_nodes;     /* kernel and event nodes in those graphs */
  size_t graph_updates;   /* of them, the kept executable graph updated in place */
} bc_batch_stats;

/* Plan of one product (no GPU needed; for inspection and tests). */
typedef struct {
  size_t fft_points;      /* M */
  int width;              /* b */
  int levels;             /* 1 = single-CTA kernel, 2 or 3 = passes over HBM */
  int L1, L2, Lr;         /* decomposition M = L1 * L2 * Lr (L2 = 1 for two levels) */
  size_t digits_a, digits_b;
  size_t out_words;       /* words produced by the transform (the rest are 0) */
  size_t work_bytes;      /* device scratch for this product */
} bc_plan_info;

int bc_gpu_init(const bc_gpu_config *cfg);
int bc_gpu_shutdown(void);

/* C[0..CL) = A*B mod 2^(32*CL).  AL, BL >= 0 (a zero length means zero).
 * Same semantics as _fft_mul (bigfloat/mul.c:108-174) minus its aborts. */
int bc_gpu_mul(uint32_t *C, size_t CL, const uint32_t *A, size_t AL,
               const uint32_t *B, size_t BL, bc_mul_stats *stats);

/* Independent products in as few launches as their shapes allow: items are
 * bucketed by transform length and every pass covers a whole bucket. */
int bc_gpu_mul_batch(const bc_mul_desc *items, size_t n, bc_batch_stats *stats);

/* Small products, exact, in one launch: every operand at most 256 limbs and
 * every C at most 512 limbs (BC_ERR_TOO_LARGE beyond), all arrays in host
 * memory (BC_ERR_INVALID for device memory).  C = A*B mod 2^(32 CL), zero
 * above AL + BL limbs.  The reference computes products of this size on the
 * CPU with its basecase / Karatsuba code (bigfloat/mul.c:176-553, below 100
 * output limbs, mul.c:640-648); here a batch of them is one schoolbook
 * kernel (one warp per product, integer column sums, no rounding). */
int bc_gpu_mul_small_batch(const bc_mul_desc *items, size_t n);

/* Same, with hints: BC_BATCH_HOST_OPERANDS declares every A, B and C to be
 * host memory, BC_BATCH_DEVICE_OPERANDS every one to be device memory (each
 * skips the per-pointer memory query, which dominates batches of millions of
 * small products). */
enum { BC_BATCH_HOST_OPERANDS = 1, BC_BATCH_DEVICE_OPERANDS = 2, BC_BATCH_GRAPH = 4 };
/* BC_BATCH_GRAPH (or $BC_GRAPH=1 for every batch): the batch's passes, every
 * length bucket on its class stream, are captured into one CUDA graph and
 * started with a single cudaGraphLaunch.  The library keeps the executable
 * graph and updates it in place (cudaGraphExecUpdate) when the next batch has
 * the same launch structure, so a batch of the same lengths repeated (one
 * tree level after another of the same shape, a benchmark loop) pays neither
 * per-kernel launch calls nor a new instantiation.  Products, rounding checks
 * and retries are the same as without the flag; per-kernel timing
 * (bc_gpu_time_kernels) and the opt-in fused middle pass ($BC_FUSED=1) turn
 * it off.  The reference has no counterpart (its task tree, main.c:82-90,
 * runs products one call each). */
int bc_gpu_mul_batch_flags(const bc_mul_desc *items, size_t n, unsigned flags, bc_batch_stats *stats);

/* The binary-splitting sum of e's series on the GPU: P and Q with
 * P/Q = sum_{j=a+1}^{b} 1/((a+1)(a+2)...j) and Q = (a+1)(a+2)...b, the
 * integers the reference's e_BSR (main.c:63-109) builds on the host.  Every
 * intermediate value stays in device memory (leaves of up to 1024 terms, one
 * warp each, then one batched product level and one addition kernel per tree
 * level).  On
 * success *P and *Q are malloc'd host arrays of *PL and *QL little-endian
 * limbs without top zeros (the caller frees them).  Needs b < 2^32 - 16. */
int bc_gpu_e_series(uint32_t a, uint32_t b, uint32_t **P, size_t *PL, uint32_t **Q, size_t *QL);

/* Leaves of the binary-to-decimal conversion (the reference's
 * convert_trunc, bigfloat/radix.c:41-91), all in one GPU launch: for each
 * leaf, k base-10^9 digits of the fraction y (len host limbs below the
 * point, n the limb count the digit positions refer to) into s[0..k), most
 * significant last.  alpha is the caller's log(10^9)/log(2^32), so that
 * every truncation point matches the caller's own arithmetic.  len + 1 and
 * n + 1 must not exceed 1024 limbs (leaves of up to 1000 digits). */
typedef struct {
  const uint32_t *y;
  size_t len;
  size_t n;
  size_t k;
  uint32_t *s;
} bc_radix_leaf;
int bc_gpu_radix_leaves(const bc_radix_leaf *leaves, size_t count, double alpha);

/* The whole binary-to-decimal conversion tree of the reference's convert_rec
 * (bigfloat/radix.c:228-318) on the GPU, as planned by the caller: node 0 is
 * the root (k digits of the fraction y, n limbs below the point); an internal
 * node names its high and low children (later in the array), the low
 * child's digit count kl and the index of 10^(9(k-kl)) in `table`; a leaf
 * has child_h = child_l = -1.  Every product, leaf and merge runs in device
 * memory; y and the table entries cross once, the root's k digits come back
 * into out (most significant last; when out is device memory, e.g. from
 * bc_gpu_device_alloc, they stay on the device).  alpha as for
 * bc_gpu_radix_leaves. */
typedef struct {
  size_t k, n;
  long child_h, child_l;
  size_t kl;
  int table;
} bc_radix_node;
int bc_gpu_radix_tree(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nnodes,
                      const uint32_t *const *table, const size_t *table_len, int ntable, double alpha,
                      uint32_t *out);

/* Same tree with the power table built in device memory: entry 0 is t0
 * (t0len limbs, host); entry i >= 1 comes from entry steps[i].src (< i) by
 * op 1 = times 10^9 (src length + 1 limbs), op 2 = squaring (product
 * trimmed as bigfloat_mul trims it), op 3 = squaring then times 10^9 (trimmed
 * square plus one limb) — the steps of the reference's table construction
 * (bigfloat/radix.c:156-205).  Only y, t0 and the digits cross the bus. */
typedef struct {
  int src;
  int op;
} bc_radix_pow_step;
/* A bigfloat as the host library holds it (include/bigfloat.h): value =
 * +-sum coef[i] 2^(32(i+exp)), sign 1 positive, 0 negative, len 0 for zero. */
typedef struct {
  const uint32_t *coef;
  size_t len;
  int64_t exp;
  int sign;
} bc_bignum;
typedef struct {
  uint32_t *coef; /* malloc'd (the caller frees it); NULL when len == 0 */
  size_t len;
  int64_t exp;
  int sign;
} bc_bignum_out;

/* The upper levels of the reciprocal's Newton iteration (bigfloat/rcp.c:15-101)
 * in device memory: from r0 (the reciprocal of den at the lowest of these
 * levels' predecessor precision), for each precision levels[0] <
 * levels[1] < ...:  r <- r - (r*den - 1)*r, every product and difference
 * with the host library's semantics at that precision; then, when num is not
 * NULL, the quotient num*r at precision pdiv (bigfloat/div.c:14-27).  Only
 * den, num, r0 and the result cross the bus. */
int bc_gpu_newton(const bc_bignum *den, const bc_bignum *r0, const size_t *levels, int nlevels, const bc_bignum *num,
                  size_t pdiv, bc_bignum_out *out);

/* Diagnostic (no counterpart in the reference): runs one carry lookback
 * whose predecessor never publishes, so its bounded wait runs out; returns
 * BC_ERR_TIMEOUT (the wait gave up and flagged the sum) and the kernel's
 * time in *seconds.  The context stays usable.  Shows that a wait that
 * cannot end ends the kernel with an error status instead of a hang. */
int bc_gpu_selftest_wait(double *seconds);

int bc_gpu_radix_tree_pow(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nnodes,
                          const uint32_t *t0, size_t t0len, const bc_radix_pow_step *steps, int ntable, double alpha,
                          uint32_t *out);

/* Decimal text of base-10^9 limbs, written to an open file: nine
 * zero-padded characters per limb for limbs[top], limbs[top-1], ...,
 * limbs[top-n+1] (most significant first, the order of the reference's
 * printing loop, bigfloat/string.c:93-111), the whole text cut at maxbytes
 * bytes and placed at byte `offset` of fd (pwrite; the file position is not
 * used).  limbs may be host or device memory (with bc_gpu_radix_tree_pow
 * writing its root into a device array, the digits never cross to the host:
 * the text is rendered on the GPU and leaves through the pinned staging ring,
 * each chunk written by several threads while the next one crosses).  Each
 * limb must be below 10^9.  BC_ERR_IO when a write fails. */
int bc_gpu_decimal_write(const uint32_t *limbs, size_t top, size_t n, size_t maxbytes, int fd, long long offset);

/* Device memory for callers that keep results on the GPU (e.g. the `out` of
 * bc_gpu_radix_tree_pow, which then stays on the device), and a synchronous
 * copy between any two host or device ranges. */
int bc_gpu_device_alloc(size_t bytes, void **p);
int bc_gpu_device_free(void *p);
int bc_gpu_copy(void *dst, const void *src, size_t bytes);

/* Launch on this CUDA stream (cudaStream_t as void*; NULL = library stream).
 * Calls still return only when their results are complete. */
int bc_gpu_set_stream(void *stream);

int bc_gpu_plan(size_t AL, size_t BL, size_t CL, int square, bc_plan_info *out);

/* Load a width table (lines "M width"); no GPU needed.  bc_gpu_init loads
 * bc_gpu_config.tune_path or $BC_TUNE_FILE itself. */
int bc_gpu_load_width_table(const char *path);
/* Largest width allowed at transform length M by the loaded width table. */
int bc_gpu_width_limit(size_t fft_points);
/* Override the width limit for one transform length (autotuner); 0 = reset. */
int bc_gpu_set_width_limit(size_t fft_points, int width);

/* Force the width of subsequent products (0 = automatic); for error sweeps. */
int bc_gpu_force_width(int width);
/* Host-only check that every supported transform shape's launches are
 * consistent (staged bytes equal awaited bytes, tiles cover rows); returns
 * BC_OK or the first failing transform length.  No GPU needed. */
int bc_gpu_check_shapes(void);
/* Supported transform lengths in increasing order; returns the count. */
int bc_gpu_lengths(size_t *out, int cap);
/* Force transform length and width (0, 0 = automatic); for the autotuner. */
int bc_gpu_force_plan(size_t fft_points, int width);

/* Decompositions of one transform length (no counterpart in the reference,
 * whose CPU transform has a single recursive form, fft/fft.c:43-96).  A
 * length of two or more levels can run as several L1 x Lr or L1 x L2 x Lr
 * splits over the compiled pass lengths; the shape autotuner
 * (bluecrunch_b200/tune/autotune.py --shapes) times them on the GPU and
 * writes the fastest per length to tune/shapes.txt, which bc_gpu_init loads
 * from beside the width table (or $BC_SHAPE_FILE).  No GPU needed for these
 * calls.
 *   bc_gpu_shape_candidates: the valid splits of fft_points as
 *     (levels, L1, L2, Lr) quadruples in out[4*i..4*i+3] (up to cap of them);
 *     returns how many there are;
 *   bc_gpu_set_shape: run fft_points with that split (0, 0, 0 = built-in);
 *     BC_ERR_INVALID if it is not one of the candidates;
 *   bc_gpu_load_shape_table: lines "M L1 L2 Lr" (L2 = 1 for two levels). */
int bc_gpu_shape_candidates(size_t fft_points, int *out, int cap);
int bc_gpu_set_shape(size_t fft_points, int L1, int L2, int Lr);
int bc_gpu_load_shape_table(const char *path);

/* Allocation-free product, for callers that cannot allocate device memory
 * or have a library do it (under a pool or allocator that owns the device,
 * in hosts that forbid cudaMalloc after start-up).  No counterpart in the
 * reference.
 *
 * C, A, B are device pointers of the current device; C must not overlap A or
 * B.  Computes C[0..CL) = A*B mod 2^(32 CL) like bc_gpu_mul, on `stream`
 * (cudaStream_t as void*, NULL = legacy default stream), and returns when the
 * product is complete.  Limits: min(AL,CL) + min(BL,CL) <= 131072 limbs
 * (transforms up to 2^17 points); larger products return BC_ERR_TOO_LARGE.
 *
 * Scratch is one 8 MiB file-scope __device__ array that every GPU loading
 * this library holds until the process exits; nothing is allocated per call
 * (no cudaMalloc/cudaFree or allocating library routine).  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current.  Every call on a device shares the array and clears
 * what must start at zero; calls whose GPU work overlaps would race on it.
 * The function serialises host callers, synchronises `stream` and reads the
 * outcome back before it returns, so it must not be called on a stream that
 * is being captured into a CUDA graph. */
int bc_gpu_mul_noalloc(uint32_t *C, size_t CL, const uint32_t *A, size_t AL,
                       const uint32_t *B, size_t BL, void *stream);

int bc_gpu_sync(void);
int bc_gpu_last_error(void);
int bc_gpu_last_cuda_error(void);
const char *bc_gpu_strerror(int code);

/* Per-kernel GPU time of the last bc_gpu_mul / bc_gpu_mul_batch when kernel
 * timing is on (bc_gpu_time_kernels(1)).  names[i] / ms[i], returns count. */
int bc_gpu_time_kernels(int on);
int bc_gpu_kernel_times(const char **names, double *ms, int cap);

#ifdef __cplusplus
}
#endif
#endif
