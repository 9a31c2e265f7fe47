// bc_gpu.cu — host side of libbcgpu: planning, tables, device arena, class
// batching, launches, rounding-error checks with narrower-width retry, and
// the C ABI declared in include/bc_gpu.h.
//
// The reference multiply (_fft_mul, bigfloat/mul.c:108-174) picks a width
// from CL alone (mul.c:109-124), allocates two arrays per call (mul.c:133-138)
// and aborts on widths it has no packer for (fft/convert.c:66-68).  Here the
// width is the narrowest one that fits the smallest transform allowed by the
// width table, scratch comes from one device arena, and every failure is a
// status code.
#include <algorithm>
#include <thread>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <unistd.h>

#include <cudaTypedefs.h>

#include "bc_gpu.h"
#include "bc_pipe.cuh"
#include "bc_bsr.cuh"
#include "bc_radix.cuh"
#include "bc_rows_warp.cuh"
#include "bc_rows_w512.cuh"
#include "bc_arith.cuh"
#include "bc_pass16.cuh"
#include "bc_block.cuh"
#include "bc_text.cuh"
#include "bc_school.cuh"

using namespace bc;

namespace {

// ------------------------------------------------------------------ shapes
struct Shape {
  int M = 0, L1 = 0, L2 = 1, Lr = 1, levels = 0;
};

// Transform lengths are 2^k, 3*2^k and 5*2^k: the odd factor lives in the
// row length (or the one-CTA length), the outer and middle lengths are
// powers of two.
constexpr int kRowLens[] = {128, 192, 256, 320, 384, 512, 640, 768, 1024, 1280, 1536, 2048, 2560, 3072, 4096};
constexpr int kSmallLens[] = {256, 512, 768, 1024, 1280, 1536, 2048, 2560, 3072, 4096, 5120};
constexpr int kOuterLens[] = {64, 128, 256, 512};
constexpr size_t kMaxM = size_t(1) << 30;

bool is_row_len(size_t L) {
  for (int x : kRowLens) if ((size_t)x == L) return true;
  return false;
}
size_t pow2part(size_t x) { return x & (~x + 1); }

// The built-in decomposition of transform length M (shape_for below may
// replace it by a tuned one with the same number of levels).
bool shape_default(size_t M, Shape &s) {
  if (M < 256 || M > kMaxM) return false;
  const size_t p2 = (M % 3 == 0) ? M / 3 : ((M % 5 == 0) ? M / 5 : M);
  if (p2 & (p2 - 1)) return false;
  if (M <= 5120) {
    for (int x : kSmallLens)
      if ((size_t)x == M) { s.M = (int)M; s.L1 = (int)M; s.L2 = 1; s.Lr = 1; s.levels = 1; return true; }
    return false;
  }
  for (int L1 : kOuterLens) {
    if (M % L1) continue;
    const size_t Lr = M / L1;
    if (is_row_len(Lr) && pow2part(Lr) >= (size_t)pass_tile_w(L1)) {
      s.M = (int)M; s.L1 = L1; s.L2 = 1; s.Lr = (int)Lr; s.levels = 2; return true;
    }
  }
  // three levels: rows of about 1024 points keep the fused row pass free of
  // spills with two rows per CTA; longer rows only when the outer passes run out
  static const int kRowPref[] = {1024, 768, 1536, 512, 2048, 3072, 4096, 1280, 640, 2560};
  for (int Lri : kRowPref) {
    const size_t Lr = (size_t)Lri;
    if (M % Lr) continue;
    const size_t R = M / Lr;
    for (int L1 : kOuterLens) {
      if (R % L1) continue;
      const size_t L2 = R / L1;
      if (L2 < 64 || L2 > 512 || (L2 & (L2 - 1)) || L2 > (size_t)L1) continue;
      if (pow2part(Lr) < (size_t)pass_tile_w((int)L2) || pow2part(L2 * Lr) < (size_t)pass_tile_w(L1)) continue;
      s.M = (int)M; s.L1 = L1; s.L2 = (int)L2; s.Lr = (int)Lr; s.levels = 3; return true;
    }
  }
  return false;
}

// Transform lengths in increasing order: 2^k and 3*2^k with a valid shape.
const std::vector<size_t> &lengths() {
  static std::vector<size_t> v = [] {
    std::vector<size_t> r;
    for (size_t p = 256; p <= kMaxM; p *= 2) {
      Shape s;
      if (shape_default(p, s)) r.push_back(p);
      if (3 * p / 2 <= kMaxM && shape_default(3 * p / 2, s)) r.push_back(3 * p / 2);
      if (5 * p / 4 <= kMaxM && shape_default(5 * p / 4, s)) r.push_back(5 * p / 4);
    }
    std::sort(r.begin(), r.end());
    return r;
  }();
  return v;
}

// ------------------------------------------------------------------ state
struct Tables {
  double2 *dev = nullptr;
  const double2 *twL1 = nullptr, *twL2 = nullptr, *twLr = nullptr, *pw_fwd = nullptr, *pw_inv = nullptr;
  Tw2 tw4M{};
};

struct Ctx {
  bool init = false;
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  char *arena = nullptr;
  size_t arena_cap = 0, arena_limit = 0;
  std::map<std::tuple<size_t, int, int, int>, Tables> tables;  // per (M, L1, L2, Lr)
  std::map<size_t, int> width_override;
  std::map<size_t, int> width_file;
  std::map<size_t, Shape> shape_table;  // tuned decompositions (shapes file, bc_gpu_set_shape)
  int forced_width = 0;
  size_t forced_M = 0;
  double max_err = 0.25;
  int verbose = 0;
  int last_error = 0;
  int last_cuda = 0;
  bool time_kernels = false;
  bool rows_warp = true;  // 512- and 1024-point rows one warp per row ($BC_ROWS_WARP=0: the block kernel)
  bool pass16 = true;     // outer passes of L1 <= 256 with 16 points per thread ($BC_PASS16=0: 8 points)
  bool fused = false;     // three-level middle in one kernel where it applies ($BC_FUSED=1; default: separate passes)
  bool share_b = true;    // one B transform for items with the same device B ($BC_SHARE_B=0: one per item)
  // second operand's copy of a single product from pinned host memory: on
  // copy_stream, so the outer pass packs the first operand meanwhile
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ev[2] = {nullptr, nullptr};
  // the classes of a batch run on these streams side by side (they share no
  // data): a small class's kernels fill the SMs a large one leaves idle
  cudaStream_t class_stream[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t class_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // [4]: fork
  // BC_BATCH_GRAPH: the launches are captured on cap_stream (which never runs
  // work itself) and the kept executable graph is updated or re-instantiated
  bool graph_all = false;  // $BC_GRAPH=1: every batch as a graph
  // passes after a class's first one start while the previous pass drains
  // (programmatic dependent launch; $BC_PDL=0: plain stream order)
  bool pdl = true;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<std::pair<const char *, double>> ktimes;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> kev;
  std::vector<cudaEvent_t> kev_pool;  // recycled timing events
  // pinned host blocks for the per-call descriptor upload and outcome
  // readback (copies from pinned memory need no staging by the driver)
  void *pin_small = nullptr;
  size_t pin_small_cap = 0;
  int sm_count = 148;
};

Ctx g;
std::recursive_mutex g_mu;

// The decomposition a product of length M runs with: the tuned one when the
// shapes table has M, else the built-in one.
bool shape_for(size_t M, Shape &s) {
  auto it = g.shape_table.find(M);
  if (it != g.shape_table.end()) {
    s = it->second;
    return true;
  }
  return shape_default(M, s);
}

// Structural candidates for length M with as many levels as the built-in
// shape: two levels L1 x Lr, three levels L1 x L2 x Lr, over the compiled
// outer, middle and row lengths (launch consistency is checked separately,
// shape_launch_ok).
std::vector<Shape> shape_candidates(size_t M) {
  std::vector<Shape> out;
  Shape d;
  if (!shape_default(M, d) || d.levels < 2) return out;
  for (int L1 : kOuterLens) {
    if (M % L1) continue;
    const size_t R = M / L1;
    if (d.levels == 2) {
      if (is_row_len(R) && pow2part(R) >= (size_t)pass_tile_w(L1)) {
        Shape s;
        s.M = (int)M; s.L1 = L1; s.L2 = 1; s.Lr = (int)R; s.levels = 2;
        out.push_back(s);
      }
      continue;
    }
    for (int Lr : kRowLens) {
      if (R % Lr) continue;
      const size_t L2 = R / Lr;
      if (L2 < 64 || L2 > 512 || (L2 & (L2 - 1))) continue;
      if (pow2part(Lr) < (size_t)pass_tile_w((int)L2) || pow2part(L2 * Lr) < (size_t)pass_tile_w(L1)) continue;
      Shape s;
      s.M = (int)M; s.L1 = L1; s.L2 = (int)L2; s.Lr = Lr; s.levels = 3;
      out.push_back(s);
    }
  }
  return out;
}

int fail(int code) {
  g.last_error = code;
  return code;
}

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      g.last_cuda = (int)e_;                                                     \
      if (g.verbose) fprintf(stderr, "bc_gpu: %s failed: %s (%s:%d)\n", #call,   \
                             cudaGetErrorString(e_), __FILE__, __LINE__);        \
      return fail(e_ == cudaErrorMemoryAllocation ? BC_ERR_NOMEM : BC_ERR_CUDA); \
    }                                                                            \
  } while (0)

// ------------------------------------------------------------------ widths
// Default width limit at transform length M: about 2b + log2(M)/2 stays near
// the FP64 budget for a max rounding error below 0.25 on random digits.
// Replaced per length by the tuned table (bc_tune file) when present.
int default_width_limit(size_t M) {
  const double lg = std::log2((double)M);
  int b = (int)std::floor(23.0 - 0.3 * lg);
  return std::max(8, std::min(24, b));
}

int width_limit(size_t M) {
  auto it = g.width_override.find(M);
  if (it != g.width_override.end()) return it->second;
  it = g.width_file.find(M);
  if (it != g.width_file.end()) return it->second;
  // a length the table does not hold takes the width of the next longer one
  // it does (the limit only falls with the length)
  it = g.width_file.upper_bound(M);
  if (it != g.width_file.end()) return std::min(it->second, default_width_limit(M) + 4);
  return default_width_limit(M);
}

void load_width_file(const char *path) {
  if (!path) path = getenv("BC_TUNE_FILE");
  std::string p;
  if (path) p = path;
  if (p.empty()) return;
  FILE *f = fopen(p.c_str(), "r");
  if (!f) return;
  char line[256];
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    unsigned long long M = 0;
    int b = 0;
    if (sscanf(line, "%llu %d", &M, &b) == 2 && b >= 8 && b <= 24) g.width_file[(size_t)M] = b;
  }
  fclose(f);
}

// ------------------------------------------------------------------ plans
struct Plan {
  Shape shape;
  int b = 0;
  size_t AL = 0, BL = 0;     // clamped to CL
  size_t ndA = 0, ndB = 0;
  size_t nwords = 0, nruns = 0, ntiles = 0;
  bool square = false;
  size_t CL = 0;
};

size_t ndigits(size_t XL, int b) { return (32 * (uint64_t)XL + b - 1) / b; }

// HBM passes over the complex data per product, relative to two levels: the
// 3-level shape adds a read+write of every operand and of the product.
double shape_cost(const Shape &s) { return (double)s.M * (s.levels == 3 ? 2.0 : 1.0); }

void plan_finish(Plan &pl);

bool make_plan(size_t AL, size_t BL, size_t CL, bool square, int bcap, Plan &pl, size_t maxM = 0) {
  pl = Plan();
  pl.AL = std::min(AL, CL);
  pl.BL = std::min(BL, CL);
  pl.CL = CL;
  pl.square = square;
  bool found = false;
  double best = 0;
  size_t first_fit = 0;
  for (size_t M : lengths()) {
    if (maxM && M > maxM) break;
    if (g.forced_M && M != g.forced_M) continue;
    if (first_fit && M > 4 * first_fit) break;
    int bmax = std::min(width_limit(M), bcap);
    if (g.forced_width) bmax = g.forced_width;
    if (bmax < 8) continue;
    auto fits = [&](int b) {
      const size_t na = ndigits(pl.AL, b), nb = ndigits(pl.BL, b);
      return na + nb <= 2 * M + 1;
    };
    if (!fits(bmax)) continue;
    if (!first_fit) first_fit = M;
    Shape s;
    shape_for(M, s);
    const double cost = shape_cost(s);
    if (found && cost >= best) continue;
    int b = bmax;
    if (!g.forced_width)
      while (b > 8 && fits(b - 1)) b--;
    found = true;
    best = cost;
    pl.shape = s;
    pl.b = b;
  }
  if (!found) return false;
  plan_finish(pl);
  return true;
}

// The quantities of a plan that follow from its shape and width.
void plan_finish(Plan &pl) {
  const size_t M = pl.shape.M;
  const int b = pl.b;
  pl.ndA = ndigits(pl.AL, b);
  pl.ndB = ndigits(pl.BL, b);
  const size_t prod_words = (2 * M * (uint64_t)b) / 32;
  pl.nwords = std::min(pl.CL, prod_words);
  pl.nruns = std::min((size_t)(2 * M / 8), (pl.nwords * 32 + 8 * b - 1) / (8 * b));
  pl.ntiles = std::max<size_t>(1, (pl.nruns + CARRY_TILE_RUNS - 1) / CARRY_TILE_RUNS);
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The packing pass stages limb words with 16-byte copies when the operand is
// 16-byte aligned and every row segment of a tile shares one alignment
// (S1*b/32 and M*b/32 multiples of 4 words); otherwise with 4-byte copies.
int stage16_ok(const uint32_t *X, const Plan &pl) {
  if (pl.shape.levels < 2 || ((uintptr_t)X & 15)) return 0;
  const uint64_t S1 = (uint64_t)pl.shape.M / pl.shape.L1, b = (uint64_t)pl.b;
  return ((S1 * b / 32) % 4 == 0 && ((uint64_t)pl.shape.M * b / 32) % 4 == 0) ? 1 : 0;
}

size_t work_bytes(const Plan &pl) {
  const size_t M = pl.shape.M;
  size_t w = align256(M * 16);                           // bufA
  if (!pl.square) w += align256(M * 16);                 // bufB
  if (pl.shape.levels > 1) w += align256(M / 4 * sizeof(RunRec)) + align256(pl.ntiles * 4);  // run records + status
  return w;
}

// ------------------------------------------------------------------ tables
double2 cis_neg(long double num, long double den, long double scale) {
  // e^{-2 pi i num/den} * scale, evaluated in long double
  long double a = 2.0L * 3.141592653589793238462643383279502884L * (num / den);
  return make_double2((double)(cosl(a) * scale), (double)(-sinl(a) * scale));
}

// Offsets (in double2 entries) of each table inside one contiguous block.
struct TableLayout {
  size_t oL1 = 0, oL2 = 0, oLr = 0, opf = 0, opi = 0, olo = 0, ohi = 0, total = 0, nlo = 0;
  int h = 0;
  bool has_L2 = false, has_Lr = false, has_tw = false;
};

TableLayout table_layout(const Shape &s) {
  TableLayout t;
  const size_t four = 4 * (size_t)s.M;
  while ((size_t(1) << (2 * t.h)) < four) t.h++;
  t.nlo = size_t(1) << t.h;
  const size_t nhi = (four + t.nlo - 1) / t.nlo;
  t.has_L2 = s.levels == 3;
  t.has_Lr = s.levels >= 2;
  t.has_tw = s.levels >= 2;
  size_t o = 0;
  t.oL1 = o; o += s.L1;
  if (t.has_L2) { t.oL2 = o; o += s.L2; }
  if (t.has_Lr) { t.oLr = o; o += s.Lr; }
  t.opf = o; o += s.L1;
  t.opi = o; o += s.L1;
  if (t.has_tw) { t.olo = o; o += t.nlo; t.ohi = o; o += nhi; }
  t.total = o;
  return t;
}

// All tables of a shape, computed in long double on the host into `host`
// (t.total entries).
void fill_tables(const Shape &s, const TableLayout &t, double2 *host) {
  const size_t M = s.M, four = 4 * M;
  auto block = [&](size_t at, size_t L) {
    for (size_t m = 0; m < L; m++) host[at + m] = cis_neg((long double)m, (long double)L, 1.0L);
  };
  block(t.oL1, s.L1);
  if (t.has_L2) block(t.oL2, s.L2);
  if (t.has_Lr) block(t.oLr, s.Lr);
  for (size_t n = 0; n < (size_t)s.L1; n++) {
    // e^{+i pi n/(2 L1)} = conj(e^{-2 pi i n/(4 L1)}), and its conjugate / M
    double2 w = cis_neg((long double)n, 4.0L * s.L1, 1.0L);
    host[t.opf + n] = make_double2(w.x, -w.y);
    host[t.opi + n] = cis_neg((long double)n, 4.0L * s.L1, 1.0L / (long double)M);
  }
  if (t.has_tw) {
    const size_t nhi = t.ohi ? (four + t.nlo - 1) / t.nlo : 0;
    for (size_t m = 0; m < t.nlo; m++) host[t.olo + m] = cis_neg((long double)m, (long double)four, 1.0L);
    for (size_t m = 0; m < nhi; m++) host[t.ohi + m] = cis_neg((long double)(m * t.nlo), (long double)four, 1.0L);
  }
}

Tables tables_at(const TableLayout &t, double2 *dev) {
  Tables r;
  r.dev = dev;
  r.twL1 = dev + t.oL1;
  r.twL2 = t.has_L2 ? dev + t.oL2 : nullptr;
  r.twLr = t.has_Lr ? dev + t.oLr : nullptr;
  r.pw_fwd = dev + t.opf;
  r.pw_inv = dev + t.opi;
  if (t.has_tw) {
    r.tw4M.lo = dev + t.olo;
    r.tw4M.hi = dev + t.ohi;
    r.tw4M.mask = t.nlo - 1;
    r.tw4M.h = t.h;
  }
  return r;
}

// Tables are cached per decomposition (their layout and entries depend on
// L1, L2 and Lr, not on M alone).
int ensure_tables(const Shape &s, Tables **out) {
  const auto key = std::make_tuple((size_t)s.M, s.L1, s.L2, s.Lr);
  auto it = g.tables.find(key);
  if (it != g.tables.end()) { *out = &it->second; return BC_OK; }
  const TableLayout lay = table_layout(s);
  std::vector<double2> host(lay.total);
  fill_tables(s, lay, host.data());
  double2 *dev = nullptr;
  CK(cudaMalloc(&dev, lay.total * sizeof(double2)));
  // On the library stream, then waited for: a plain cudaMemcpy from pageable
  // memory returns once the data is staged, before the copy lands, and the
  // legacy stream it uses does not order with the library's non-blocking
  // stream, so the first kernels of a new length could read stale tables.
  CK(cudaMemcpyAsync(dev, host.data(), lay.total * sizeof(double2), cudaMemcpyHostToDevice, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  auto res = g.tables.emplace(key, tables_at(lay, dev));
  *out = &res.first->second;
  return BC_OK;
}

// ------------------------------------------------------------------ kernels
// Kernel parameter lists: (ClassParams), (ClassParams, map), (ClassParams, map, map).
enum KSig { SIG_P = 0, SIG_P_MAP = 1, SIG_P_MAP2 = 2 };

struct KInfo {
  const void *fn = nullptr;
  int threads = 0;
  size_t smem = 0;
  const char *name = "";
  int sig = SIG_P;
  int box = 0;            // TMA box lines (rows) the kernel expects per box
  unsigned unit_bytes = 0; // bytes the kernel waits for per staged unit (per operand)
  int parts = 1;          // boxes per column group (or per row)
  bool warp_rows = false; // a row kernel with one warp per row and no tensor maps
  int pts = PTS;          // points per thread of a column pass (tile width = threads / (L / pts))
  bool coop = false;      // cooperative launch: every CTA resident (its warps wait on one another)
};

template <int L>
KInfo outer_fwd_info() {
  using T = PassTile<L>;
  using K = PackTile<L>;
  return {(const void *)k2_outer_fwd<L>, T::NT, K::SMEM, "outer_fwd", SIG_P};
}
template <int L>
KInfo outer_inv_info() {
  using T = PassTile<L>;
  return {(const void *)k2_outer_inv<L>, T::NT, T::SMEM_OUTER_INV, "outer_inv", SIG_P_MAP,
          T::BOX_ROWS, T::BYTES, T::HALVES};
}
template <int L, bool INV>
KInfo mid_info() {
  using T = PassTile<L>;
  return {(const void *)k2_mid<L, INV>, T::NT, T::SMEM_MID, INV ? "mid_inv" : "mid_fwd",
          SIG_P_MAP2, T::BOX_ROWS, T::BYTES, T::HALVES};
}
template <int L, bool SQ>
KInfo rows_info() {
  using R = RowTile<L>;
  return {(const void *)k2_rows<L, SQ>, R::NT, R::SMEM, "rows", SIG_P_MAP2,
          R::BOX_LINES, (unsigned)(R::NR * L * 16), R::PARTS};
}
template <int M, bool SQ>
KInfo small_info() {
  return {(const void *)k_small<M, SQ>, M / PTS, TileSmem<M, 1>::elems * sizeof(double2), "small", SIG_P};
}

template <int L>
KInfo outer_fwd16_info() {
  using T = Pass16<L>;
  KInfo k{(const void *)k3_outer_fwd<L>, T::NT, T::SMEM_FWD, "outer_fwd", SIG_P};
  k.pts = P16;
  return k;
}
template <int L>
KInfo outer_inv16_info() {
  using T = Pass16<L>;
  KInfo k{(const void *)k3_outer_inv<L>, T::NT, T::SMEM_INV, "outer_inv", SIG_P_MAP, PassTile<L>::BOX_ROWS,
          PassTile<L>::BYTES, PassTile<L>::HALVES};
  k.pts = P16;
  return k;
}

KInfo get_outer(int L, bool inv) {
  if (g.pass16) {
    switch (L) {
      case 64: return inv ? outer_inv16_info<64>() : outer_fwd16_info<64>();
      case 128: return inv ? outer_inv16_info<128>() : outer_fwd16_info<128>();
      case 256: return inv ? outer_inv16_info<256>() : outer_fwd16_info<256>();
    }
  }
  switch (L) {
    case 64: return inv ? outer_inv_info<64>() : outer_fwd_info<64>();
    case 128: return inv ? outer_inv_info<128>() : outer_fwd_info<128>();
    case 256: return inv ? outer_inv_info<256>() : outer_fwd_info<256>();
    case 512: return inv ? outer_inv_info<512>() : outer_fwd_info<512>();
  }
  return {};
}
KInfo get_mid(int L, bool inv) {
  switch (L) {
    case 64: return inv ? mid_info<64, true>() : mid_info<64, false>();
    case 128: return inv ? mid_info<128, true>() : mid_info<128, false>();
    case 256: return inv ? mid_info<256, true>() : mid_info<256, false>();
    case 512: return inv ? mid_info<512, true>() : mid_info<512, false>();
  }
  return {};
}
#define ROWCASE(L) \
  case L: return sq ? rows_info<L, true>() : rows_info<L, false>();
KInfo get_rows(int L, bool sq) {
  if (L == R5_L && g.rows_warp) {
    KInfo k{sq ? (const void *)k2_rows_w512<true> : (const void *)k2_rows_w512<false>, 32 * R5_WARPS, R5_SMEM,
            "rows", SIG_P_MAP2};
    k.warp_rows = true;
    return k;
  }
  if (L == RW_L && g.rows_warp) {
    KInfo k{sq ? (const void *)k2_rows_w1024<true> : (const void *)k2_rows_w1024<false>, 32 * RW_WARPS, RW_SMEM,
            "rows", SIG_P_MAP2};
    k.warp_rows = true;
    return k;
  }
  switch (L) {
    ROWCASE(128) ROWCASE(192) ROWCASE(256) ROWCASE(320) ROWCASE(384) ROWCASE(512) ROWCASE(640) ROWCASE(768)
    ROWCASE(1024) ROWCASE(1280) ROWCASE(1536) ROWCASE(2048) ROWCASE(2560) ROWCASE(3072) ROWCASE(4096)
  }
  return {};
}
#define SMALLCASE(L) \
  case L: return sq ? small_info<L, true>() : small_info<L, false>();
KInfo get_small(int M, bool sq) {
  switch (M) {
    SMALLCASE(256) SMALLCASE(512) SMALLCASE(768) SMALLCASE(1024) SMALLCASE(1280) SMALLCASE(1536) SMALLCASE(2048)
    SMALLCASE(2560) SMALLCASE(3072) SMALLCASE(4096) SMALLCASE(5120)
  }
  return {};
}

// Grid cap (resident CTAs per SM x SMs) per (device, kernel): the dynamic
// shared-memory attribute is a per-device setting of the function, so a call
// on another device (bc_gpu_mul_noalloc takes the caller's current device)
// sets it there too.
std::map<std::pair<int, const void *>, int> g_occ;

int prepare(const KInfo &k, int *grid_cap) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto it = g_occ.find({dev, k.fn});
  if (it == g_occ.end()) {
    if (k.smem > 48 * 1024) CK(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
    int n = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k.fn, k.threads, k.smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (n < 1) n = 1;
    it = g_occ.emplace(std::make_pair(dev, k.fn), n * std::max(sms, 1)).first;
  }
  *grid_cap = it->second;
  return BC_OK;
}

// pdl: launch with programmatic stream serialisation (the kernel may start
// while the previous kernel of the stream finishes; it waits in pdl_wait
// before touching data that kernel reads or writes)
int launch(const KInfo &k, long long units, const ClassParams &p, size_t *nlaunch, cudaStream_t stream, bool timed,
           const CUtensorMap *mA = nullptr, const CUtensorMap *mB = nullptr, bool pdl = false) {
  int cap = 0;
  int r = prepare(k, &cap);
  if (r) return r;
  const int grid = (int)std::max<long long>(1, std::min<long long>(units, cap));
  ClassParams pc = p;
  CUtensorMap a{}, b{};
  if (mA) a = *mA;
  if (mB) b = *mB;
  else b = a;
  void *args[3] = {&pc, &a, &b};
  if (k.coop) {
    CK(cudaLaunchCooperativeKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, stream));
  } else if (pdl) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(k.threads);
    cfg.dynamicSmemBytes = k.smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelExC(&cfg, k.fn, args));
  } else {
    CK(cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, stream));
  }
  (*nlaunch)++;
  if (timed && g.time_kernels) {
    cudaEvent_t e;
    if (!g.kev_pool.empty()) {
      e = g.kev_pool.back();
      g.kev_pool.pop_back();
    } else {
      CK(cudaEventCreate(&e));
    }
    CK(cudaEventRecord(e, stream));
    g.kev.push_back(e);
    g.ktimes.push_back({k.name, 0.0});
  }
  return BC_OK;
}

// ------------------------------------------------------------------ tensor maps
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder() {
  if (g_encode) return BC_OK;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  CK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || !fn) return fail(BC_ERR_CUDA);
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return BC_OK;
}

// FLOAT64 elements, 128-byte swizzle, innermost box dimension 16 doubles.
int encode_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
               const cuuint32_t *box, CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B) {
  int r = get_encoder();
  if (r) return r;
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult cr = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void *>(base), dims, strides,
                         box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) {
    if (g.verbose) fprintf(stderr, "bc_gpu: cuTensorMapEncodeTiled failed (%d)\n", (int)cr);
    return fail(BC_ERR_CUDA);
  }
  return BC_OK;
}

// Host-side consistency of a shape's pipelined launches: every staged unit's
// TMA boxes must deliver exactly the bytes its kernel waits for, boxes must
// tile the rows, and column tiles must tile the rows of each pass.  Checked
// before every launch and, for all lengths, by bc_gpu_check_shapes.
// Dynamic shared memory a CTA may use on sm_100 (227 KB).
constexpr size_t kMaxSmemPerCta = 227 * 1024;

bool shape_launch_ok(const Shape &s, bool sq) {
  if (s.levels == 1) {
    const KInfo k = get_small(s.M, sq);
    return k.fn != nullptr && k.smem <= kMaxSmemPerCta;
  }
  const size_t S1 = s.M / s.L1, Lr = s.levels == 3 ? (size_t)s.Lr : S1;
  KInfo ko = get_outer(s.L1, false), ki = get_outer(s.L1, true), kr = get_rows((int)Lr, sq);
  if (!ko.fn || !ki.fn || !kr.fn) return false;
  if (ko.smem > kMaxSmemPerCta || ki.smem > kMaxSmemPerCta || kr.smem > kMaxSmemPerCta) return false;
  if (s.levels == 3) {
    const KInfo kmf = get_mid(s.L2, false), kmi = get_mid(s.L2, true);
    if (!kmf.fn || !kmi.fn || kmf.smem > kMaxSmemPerCta || kmi.smem > kMaxSmemPerCta) return false;
  }
  const int W1 = ko.threads / (s.L1 / ko.pts);
  if (S1 % W1 || W1 % 8 || ki.threads / (s.L1 / ki.pts) != W1) return false;
  if ((size_t)(W1 / 8) * ki.parts * 128 * ki.box != ki.unit_bytes || (size_t)ki.box * ki.parts != (size_t)s.L1)
    return false;
  const int NR = kr.warp_rows ? 1 : kr.threads / ((int)Lr / PTS);
  if (!kr.warp_rows && ((size_t)kr.parts * 128 * kr.box * NR != kr.unit_bytes || (size_t)kr.box * kr.parts != Lr / 8 ||
                        (s.M / Lr) % NR != 0 || kr.box > 256 || kr.box % 8))
    return false;
  if (s.levels == 3) {
    KInfo km = get_mid(s.L2, false);
    if (!km.fn) return false;
    const int W2 = km.threads / (s.L2 / km.pts);
    if (Lr % W2 || W2 % 8) return false;
    if ((size_t)(W2 / 8) * km.parts * 128 * km.box != km.unit_bytes || (size_t)km.box * km.parts != (size_t)s.L2)
      return false;
  }
  return true;
}

// The fused middle pass covers three-level shapes with 1024-point rows and
// L2 = 64 or 128 (on with $BC_FUSED=1).
bool fused_ok(const Shape &s) {
  return g.fused && s.levels == 3 && s.Lr == RW_L && (s.L2 == 64 || s.L2 == 128);
}
KInfo get_fused(int L2, bool sq) {
  const void *fn = L2 == 64 ? (sq ? (const void *)k4_mid_fused<64, true> : (const void *)k4_mid_fused<64, false>)
                            : (sq ? (const void *)k4_mid_fused<128, true> : (const void *)k4_mid_fused<128, false>);
  KInfo k{fn, 32 * RW_WARPS, BLK_SMEM, "mid_fused", SIG_P_MAP2};
  k.coop = true;
  return k;
}

// The pass sequence of one class (all items share shape and squaring).  The
// items' A and B buffers are the contiguous slabs slabA / slabB (item i at
// i*M).  Scratch (records, lookback status, counter) must be set up and the
// counter and status words zeroed by the caller.
int launch_class(const Shape &s, bool sq, const ClassParams &p, long long n, unsigned long long carry_tiles,
                 double2 *slabA, double2 *slabB, cudaStream_t stream, bool timed, size_t *nl,
                 cudaEvent_t b_ready = nullptr, bool w16 = false, bool pdl_ok = false) {
  int r;
  // the first pass follows copies or event waits: a normal launch; every
  // later pass of the class follows the previous pass directly
  bool pdl = false;
  if (!shape_launch_ok(s, sq)) return fail(BC_ERR_INVALID);
  if (s.levels == 1) return launch(get_small(s.M, sq), n, p, nl, stream, timed);
  const cuuint64_t M16 = (cuuint64_t)s.M * 16, S1 = (cuuint64_t)p.S1, Lr = (cuuint64_t)p.Lr;
  KInfo ko = get_outer(s.L1, false), ki = get_outer(s.L1, true);
  const int W1 = ko.threads / (s.L1 / ko.pts);
  // forward operands: every item's A, then the B slab's slots (items sharing
  // a B share a slot)
  const long long nb = sq ? 0 : (long long)p.nb;
  if (b_ready && !sq) {
    // operand A is on the device, B still crossing: pack A, then wait for B
    ClassParams pa = p, pb = p;
    pa.fwd_ops = 1;
    pb.fwd_ops = 2;
    if ((r = launch(ko, n * (long long)(S1 / W1), pa, nl, stream, timed))) return r;
    CK(cudaStreamWaitEvent(stream, b_ready, 0));
    if ((r = launch(ko, nb * (long long)(S1 / W1), pb, nl, stream, timed))) return r;
  } else if ((r = launch(ko, (n + nb) * (long long)(S1 / W1), p, nl, stream, timed))) {
    return r;
  }
  pdl = pdl_ok;
  if (fused_ok(s) && p.blkdone && (sq || p.nb == n)) {
    // the middle (column pass, row products, inverse column pass) in one
    // persistent cooperative kernel; per-block counters in p.blkdone
    const KInfo kf = get_fused(s.L2, sq);
    const long long items = (n * s.L1 + BLK_LAG_I) * (long long)s.L2 * (sq ? 3 : 4);
    // column tiles by TMA: 4-d view (2*Lr doubles, L2 rows, L1 blocks, items),
    // boxes of 8 complex columns x L2 rows, unswizzled
    const cuuint64_t dims[4] = {2 * Lr, (cuuint64_t)s.L2, (cuuint64_t)s.L1, (cuuint64_t)n};
    const cuuint64_t str[3] = {Lr * 16, S1 * 16, M16};
    const cuuint32_t box[4] = {16, (cuuint32_t)s.L2, 1, 1};
    CUtensorMap fA, fB;
    if ((r = encode_map(&fA, slabA, 4, dims, str, box, CU_TENSOR_MAP_SWIZZLE_NONE))) return r;
    if (!sq && (r = encode_map(&fB, slabB, 4, dims, str, box, CU_TENSOR_MAP_SWIZZLE_NONE))) return r;
    if ((r = launch(kf, (items + RW_WARPS - 1) / RW_WARPS, p, nl, stream, timed, &fA, sq ? &fA : &fB))) return r;
  } else {
    CUtensorMap midA, midB;
    if (s.levels == 3) {
      const cuuint64_t dims[4] = {2 * Lr, (cuuint64_t)s.L2, (cuuint64_t)s.L1, (cuuint64_t)n};
      const cuuint64_t str[3] = {Lr * 16, S1 * 16, M16};
      KInfo km = get_mid(s.L2, false);
      const int W2 = km.threads / (s.L2 / km.pts);
      const cuuint32_t box[4] = {16, (cuuint32_t)km.box, 1, 1};
      // the boxes of one tile must deliver exactly what the kernel waits for
      if ((size_t)(W2 / 8) * km.parts * 128 * km.box != km.unit_bytes || (size_t)km.box * km.parts != (size_t)s.L2)
        return fail(BC_ERR_INVALID);
      if ((r = encode_map(&midA, slabA, 4, dims, str, box))) return r;
      const cuuint64_t dimsB[4] = {dims[0], dims[1], dims[2], (cuuint64_t)std::max<long long>(nb, 1)};
      if (!sq && (r = encode_map(&midB, slabB, 4, dimsB, str, box))) return r;
      if ((r = launch(km, (n + nb) * s.L1 * (long long)(Lr / W2), p, nl, stream, timed, &midA, sq ? &midA : &midB,
                      pdl)))
        return r;
    }
    if (get_rows(s.Lr, sq).warp_rows) {
      // one warp per row, plain loads and stores: no tensor maps
      KInfo kr = get_rows(s.Lr, sq);
      const long long rows = n * (long long)(s.M / s.Lr);
      const long long wpc = kr.threads / 32;  // rows (warps) per CTA
      if ((r = launch(kr, (rows + wpc - 1) / wpc, p, nl, stream, timed, nullptr, nullptr, pdl))) return r;
    } else {
      KInfo kr = get_rows(s.Lr, sq);
      const int NR = kr.threads / (s.Lr / PTS);
      const cuuint64_t rows = (cuuint64_t)n * (cuuint64_t)(s.M / s.Lr);
      const cuuint64_t dims[3] = {16, Lr / 8, rows};
      const cuuint64_t str[2] = {128, Lr * 16};
      const cuuint32_t box[3] = {16, (cuuint32_t)kr.box, (cuuint32_t)NR};
      if ((size_t)kr.parts * 128 * kr.box * NR != kr.unit_bytes || (size_t)kr.box * kr.parts != (size_t)(Lr / 8) ||
          (s.M / s.Lr) % NR != 0)
        return fail(BC_ERR_INVALID);
      CUtensorMap rA, rB;
      if ((r = encode_map(&rA, slabA, 3, dims, str, box))) return r;
      // B's rows by slot: nb slots of M/Lr rows
      const cuuint64_t dimsB[3] = {16, Lr / 8, (cuuint64_t)std::max<long long>(nb, 1) * (cuuint64_t)(s.M / s.Lr)};
      if (!sq && (r = encode_map(&rB, slabB, 3, dimsB, str, box))) return r;
      if ((r = launch(kr, (long long)(rows / NR), p, nl, stream, timed, &rA, sq ? &rA : &rB, pdl))) return r;
    }
    if (s.levels == 3) {
      KInfo km = get_mid(s.L2, true);
      const int W2 = km.threads / (s.L2 / km.pts);
      if ((r = launch(km, n * s.L1 * (long long)(Lr / W2), p, nl, stream, timed, &midA, &midA, pdl))) return r;
    }
  }
  {
    const cuuint64_t dims[3] = {2 * S1, (cuuint64_t)s.L1, (cuuint64_t)n};
    const cuuint64_t str[2] = {S1 * 16, M16};
    const cuuint32_t box[3] = {16, (cuuint32_t)ki.box, 1};
    if ((size_t)(W1 / 8) * ki.parts * 128 * ki.box != ki.unit_bytes || (size_t)ki.box * ki.parts != (size_t)s.L1)
      return fail(BC_ERR_INVALID);
    CUtensorMap oA;
    if ((r = encode_map(&oA, slabA, 3, dims, str, box))) return r;
    if ((r = launch(ki, n * (long long)(S1 / W1), p, nl, stream, timed, &oA, nullptr, pdl))) return r;
  }
  KInfo kc{w16 ? (const void *)k_carry<128> : (const void *)k_carry<0>, CARRY_NT, 0, "carry", SIG_P};
  return launch(kc, (long long)carry_tiles, p, nl, stream, timed, nullptr, nullptr, pdl);
}

ClassParams class_params(const Shape &s, const Tables &tb) {
  ClassParams p{};
  p.M = s.M; p.L1 = s.L1; p.S1 = s.M / s.L1; p.L2 = s.L2; p.Lr = s.levels == 3 ? s.Lr : p.S1;
  p.tw4M = tb.tw4M; p.pw_fwd = tb.pw_fwd; p.pw_inv = tb.pw_inv;
  p.twL1 = tb.twL1; p.twL2 = tb.twL2; p.twLr = tb.twLr;
  return p;
}

// ------------------------------------------------------------------ arena
// $BC_POISON: fill fresh device scratch with 0xA5 bytes, so that a kernel
// that reads scratch it has not written gives different results (a check
// for the tests; off by default).
bool poison_on() {
  static const bool on = getenv("BC_POISON") != nullptr;
  return on;
}

int arena_reserve(size_t bytes) {
  if (bytes <= g.arena_cap) return BC_OK;
  if (bytes > g.arena_limit) return fail(BC_ERR_NOMEM);
  if (g.arena) {
    CK(cudaStreamSynchronize(g.stream));
    CK(cudaFree(g.arena));
    g.arena = nullptr;
    g.arena_cap = 0;
  }
  size_t want = std::min(g.arena_limit, std::max(bytes + bytes / 4, (size_t)64 << 20));
  cudaError_t e = cudaMalloc(&g.arena, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // give back what the scratch pool keeps (DevBuf), then try the exact size
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    want = bytes;
    e = cudaMalloc(&g.arena, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      g.arena = nullptr;
      return fail(BC_ERR_NOMEM);
    }
  }
  g.arena_cap = want;
  if (poison_on()) CK(cudaMemsetAsync(g.arena, 0xA5, want, g.stream));  // ordered with the library stream
  return BC_OK;
}

enum MemKind { MEM_PAGEABLE = 0, MEM_PINNED = 1, MEM_DEVICE = 2 };
MemKind mem_kind(const void *p) {
  if (!p) return MEM_PAGEABLE;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return MEM_PAGEABLE;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return MEM_DEVICE;
  return a.type == cudaMemoryTypeHost ? MEM_PINNED : MEM_PAGEABLE;
}
bool is_device_ptr(const void *p) { return mem_kind(p) == MEM_DEVICE; }

// Host memcpy of many arrays on up to $BC_COPY_THREADS (default: all
// hardware threads, at most 32) threads, in pieces of at least 1 MiB.
struct CopyJob {
  char *dst;
  const char *src;
  size_t n;
};
unsigned copy_threads() {
  static unsigned n = [] {
    unsigned t = std::thread::hardware_concurrency();
    if (const char *e = getenv("BC_COPY_THREADS")) t = (unsigned)atoi(e);
    return std::max(1u, std::min(t ? t : 1u, 32u));
  }();
  return n;
}
void par_copy(const std::vector<CopyJob> &jobs) {
  size_t total = 0;
  for (const CopyJob &j : jobs) total += j.n;
  const unsigned nt = (unsigned)std::min<size_t>(copy_threads(), total / (size_t(4) << 20) + 1);
  if (nt <= 1) {
    for (const CopyJob &j : jobs) memcpy(j.dst, j.src, j.n);
    return;
  }
  const size_t piece = std::max<size_t>(size_t(1) << 20, total / (4 * nt));
  std::vector<CopyJob> pieces;
  for (const CopyJob &j : jobs) {
    if (j.n <= piece) { pieces.push_back(j); continue; }
    for (size_t o = 0; o < j.n; o += piece) pieces.push_back({j.dst + o, j.src + o, std::min(piece, j.n - o)});
  }
  std::atomic<size_t> next{0};
  auto worker = [&] {
    for (size_t i; (i = next.fetch_add(1, std::memory_order_relaxed)) < pieces.size();)
      memcpy(pieces[i].dst, pieces[i].src, pieces[i].n);
  };
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (unsigned k = 1; k < nt; k++) th.emplace_back(worker);
  worker();
  for (std::thread &t : th) t.join();
}

// ------------------------------------------------------------------ batch core
struct Work {
  size_t idx;      // index into the caller's items
  Plan pl;
  int bcap;
  int retries = 0;
  double err = 0;
  unsigned flags = 0;
  bool done = false;
};

struct Run {
  // per item device pointers (inside the arena)
  const uint32_t *dA = nullptr, *dB = nullptr;
  uint32_t *dC = nullptr;
  bool hostC = false;    // destination is host memory (copied out after the check)
  bool stagedC = false;  // device destination overlaps an input: computed in scratch
};

bool overlaps(const void *a, size_t abytes, const void *b, size_t bbytes) {
  const char *x = (const char *)a, *y = (const char *)b;
  return abytes && bbytes && x < y + bbytes && y < x + abytes;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Pageable host operands and results cross through a ring of two pinned
// chunks of kRingChunk bytes: the operands of a batch form one contiguous
// span on the device, filled chunk by chunk (par_copy into one chunk while
// the other's copy to the device runs), and the results leave the same way.
// No per-item copies and no pinned allocation that grows with the batch.
// Pinned host arrays copy directly.
constexpr size_t kRingChunk = size_t(64) << 20;
struct PinnedRing {
  char *half[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool pending[2] = {false, false};
};
PinnedRing g_ring;

// One array's place in a staged span: span offset, host address, bytes.
struct SpanJob {
  size_t off;
  char *host;
  size_t n;
};

// Host-side phase times of the batch path, printed at exit when $BC_PROFILE
// is set (seconds).
struct HostProfile {
  double plan = 0, layout = 0, pin_alloc = 0, copy_in = 0, launch = 0, wait = 0, copy_out = 0;
  size_t calls = 0, items = 0, bytes_in = 0, bytes_out = 0;
};
HostProfile g_prof;
double g_prof_rest = 0;  // time outside the phases above
bool g_prof_on = false;
void print_profile() {
  const HostProfile &h = g_prof;
  fprintf(stderr,
          "bc_gpu profile: %zu batch calls, %zu items, in %.2f GB, out %.2f GB, %u copy threads\n"
          "  plan %.3f s, layout %.3f s, pinned alloc %.3f s, copy in %.3f s, launch %.3f s, "
          "wait %.3f s, copy out %.3f s\n",
          h.calls, h.items, h.bytes_in / 1e9, h.bytes_out / 1e9, copy_threads(), h.plan, h.layout, h.pin_alloc,
          h.copy_in, h.launch, h.wait, h.copy_out);
}
// Adds the time since construction (or the last next()) to *acc.
struct PhaseTimer {
  double *acc;
  std::chrono::steady_clock::time_point t0;
  explicit PhaseTimer(double *a) : acc(a), t0(std::chrono::steady_clock::now()) {}
  void next(double *a) {
    auto t = std::chrono::steady_clock::now();
    *acc += std::chrono::duration<double>(t - t0).count();
    t0 = t;
    acc = a;
  }
  ~PhaseTimer() { next(acc); }
};

int ring_ready() {
  if (g_ring.half[0]) return BC_OK;
  PhaseTimer pt(&g_prof.pin_alloc);
  for (int h = 0; h < 2; h++) {
    CK(cudaHostAlloc((void **)&g_ring.half[h], kRingChunk, cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&g_ring.ev[h], cudaEventDisableTiming));
  }
  return BC_OK;
}

// Pieces of the jobs (sorted by offset) inside span window [w0, w0 + len),
// as copies between `chunk` (the window's pinned image) and the host arrays.
// `j` walks the jobs across successive windows.
void window_pieces(const std::vector<SpanJob> &jobs, size_t &j, size_t w0, size_t len, char *chunk, bool to_chunk,
                   std::vector<CopyJob> &out) {
  out.clear();
  while (j < jobs.size() && jobs[j].off < w0 + len) {
    const SpanJob &sj = jobs[j];
    const size_t s0 = std::max(sj.off, w0), s1 = std::min(sj.off + sj.n, w0 + len);
    if (s1 > s0) {
      char *c = chunk + (s0 - w0), *h = sj.host + (s0 - sj.off);
      out.push_back(to_chunk ? CopyJob{c, h, s1 - s0} : CopyJob{h, c, s1 - s0});
    }
    if (sj.off + sj.n <= w0 + len) j++;
    else break;
  }
}

// Host arrays -> device span [dev, dev + total) through the ring.
int stage_h2d(char *dev, const std::vector<SpanJob> &jobs, size_t total) {
  int r = ring_ready();
  if (r) return r;
  std::vector<CopyJob> pieces;
  size_t j = 0;
  for (size_t w0 = 0, c = 0; w0 < total; w0 += kRingChunk, c++) {
    const int h = (int)(c & 1);
    const size_t len = std::min(kRingChunk, total - w0);
    if (g_ring.pending[h]) CK(cudaEventSynchronize(g_ring.ev[h]));
    window_pieces(jobs, j, w0, len, g_ring.half[h], true, pieces);
    par_copy(pieces);
    CK(cudaMemcpyAsync(dev + w0, g_ring.half[h], len, cudaMemcpyHostToDevice, g.stream));
    CK(cudaEventRecord(g_ring.ev[h], g.stream));
    g_ring.pending[h] = true;
  }
  return BC_OK;
}

// Device span [dev, dev + total) -> host arrays through the ring (the copy
// of chunk c+1 runs while chunk c is drained).
int stage_d2h(const char *dev, const std::vector<SpanJob> &jobs, size_t total) {
  int r = ring_ready();
  if (r) return r;
  for (int h = 0; h < 2; h++)
    if (g_ring.pending[h]) { CK(cudaEventSynchronize(g_ring.ev[h])); g_ring.pending[h] = false; }
  const size_t nch = (total + kRingChunk - 1) / kRingChunk;
  auto issue = [&](size_t c) -> int {
    const int h = (int)(c & 1);
    const size_t w0 = c * kRingChunk, len = std::min(kRingChunk, total - w0);
    CK(cudaMemcpyAsync(g_ring.half[h], dev + w0, len, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaEventRecord(g_ring.ev[h], g.stream));
    return BC_OK;
  };
  if (nch && (r = issue(0))) return r;
  std::vector<CopyJob> pieces;
  size_t j = 0;
  for (size_t c = 0; c < nch; c++) {
    if (c + 1 < nch && (r = issue(c + 1))) return r;
    const int h = (int)(c & 1);
    CK(cudaEventSynchronize(g_ring.ev[h]));
    const size_t w0 = c * kRingChunk, len = std::min(kRingChunk, total - w0);
    window_pieces(jobs, j, w0, len, g_ring.half[h], false, pieces);
    par_copy(pieces);
  }
  return BC_OK;
}

// Run one attempt over `works` (none done yet).  Fills err/flags and copies
// out the products that pass the rounding check.
// A pinned host block of at least `bytes` (grown on demand; its previous
// contents are not kept).
int pin_small_reserve(size_t bytes) {
  if (bytes <= g.pin_small_cap) return BC_OK;
  if (g.pin_small) {
    CK(cudaStreamSynchronize(g.stream));
    CK(cudaFreeHost(g.pin_small));
    g.pin_small = nullptr;
    g.pin_small_cap = 0;
  }
  const size_t want = std::max<size_t>(align256(bytes), 64 << 10);
  CK(cudaHostAlloc(&g.pin_small, want, cudaHostAllocDefault));
  g.pin_small_cap = want;
  return BC_OK;
}

// Longest transform whose passes use programmatic dependent launch.  On B200
// it shortened every product up to 2^25 points (2^14-limb products by 14 %,
// 2^20 by 5 %, 2^24 by 1 %) and left 2^27 unchanged, while the 2^28-point
// products ran 2-3 % slower; above this length passes launch in plain order.
constexpr size_t kPdlMaxPoints = size_t(1) << 27;

// Ends a stream capture that an error path leaves open, so that the capture
// stream is usable by the next call.
struct CaptureGuard {
  cudaStream_t s = nullptr;
  ~CaptureGuard() {
    if (!s) return;
    cudaGraph_t gr = nullptr;
    cudaStreamEndCapture(s, &gr);
    if (gr) cudaGraphDestroy(gr);
    cudaGetLastError();
  }
};

// The captured graph replaces the kept executable graph's contents when its
// launch structure is the same (cudaGraphExecUpdate), else it is instantiated
// anew; then one cudaGraphLaunch on the library stream runs every class.
int launch_graph(cudaGraph_t gr, bc_batch_stats *st) {
  size_t nodes = 0;
  cudaGraphGetNodes(gr, nullptr, &nodes);
  bool updated = false;
  if (g.gexec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(g.gexec, gr, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();  // a structural mismatch is not an error: instantiate
      cudaGraphExecDestroy(g.gexec);
      g.gexec = nullptr;
    }
  }
  cudaError_t e = updated ? cudaSuccess : cudaGraphInstantiate(&g.gexec, gr, 0);
  if (e != cudaSuccess) g.gexec = nullptr;
  cudaGraphDestroy(gr);
  CK(e);
  CK(cudaEventRecord(g.ev0, g.stream));
  CK(cudaGraphLaunch(g.gexec, g.stream));
  st->graph_launches++;
  st->graph_nodes += nodes;
  st->graph_updates += updated ? 1 : 0;
  return BC_OK;
}

int run_attempt(const bc_mul_desc *items, std::vector<Work *> &works, bc_batch_stats *st, unsigned flags_in) {
  const bool all_host = flags_in & BC_BATCH_HOST_OPERANDS;
  const bool all_dev = flags_in & BC_BATCH_DEVICE_OPERANDS;
  const bool graph = ((flags_in & BC_BATCH_GRAPH) || g.graph_all) && !g.time_kernels && !g.fused;
  const size_t nw = works.size();
  PhaseTimer pt(&g_prof.layout);
  g_prof.items += nw;
  // ---- classes (M, square); items of a class get contiguous slabs
  std::map<std::pair<size_t, bool>, std::vector<size_t>> classes;
  for (size_t i = 0; i < nw; i++) classes[{(size_t)works[i]->pl.shape.M, works[i]->pl.square}].push_back(i);

  // ---- memory layout
  struct Slot { size_t off_dA = 0, off_dB = 0, off_dC = 0, off_rec = 0, off_status = 0; };
  std::vector<Slot> slots(nw);
  std::vector<Run> runs(nw);
  std::vector<char> hostA(nw), hostB(nw);
  size_t off = 0, stage_in = 0, stage_out = 0;
  std::vector<size_t> pin_in_off(nw, SIZE_MAX), pin_inB_off(nw, SIZE_MAX), pin_out_off(nw, SIZE_MAX);
  for (size_t i = 0; i < nw; i++) {
    const bc_mul_desc &d = items[works[i]->idx];
    const Plan &pl = works[i]->pl;
    const MemKind ka = all_dev ? MEM_DEVICE : all_host ? MEM_PAGEABLE : mem_kind(d.A);
    const MemKind kb = pl.square ? ka : (all_dev ? MEM_DEVICE : all_host ? MEM_PAGEABLE : mem_kind(d.B));
    const MemKind kc = all_dev ? MEM_DEVICE : all_host ? MEM_PAGEABLE : mem_kind(d.C);
    hostA[i] = pl.AL && ka != MEM_DEVICE;
    hostB[i] = !pl.square && pl.BL && kb != MEM_DEVICE;
    runs[i].hostC = kc != MEM_DEVICE;
    runs[i].stagedC = !runs[i].hostC && (overlaps(d.C, d.CL * 4, d.A, d.AL * 4) || overlaps(d.C, d.CL * 4, d.B, d.BL * 4));
    if (hostA[i] && ka == MEM_PAGEABLE) { pin_in_off[i] = stage_in; stage_in += align256(pl.AL * 4); }
    if (hostB[i] && kb == MEM_PAGEABLE) { pin_inB_off[i] = stage_in; stage_in += align256(pl.BL * 4); }
    if (runs[i].hostC && kc == MEM_PAGEABLE) { pin_out_off[i] = stage_out; stage_out += align256(d.CL * 4); }
    slots[i].off_dA = off; if (hostA[i] && pin_in_off[i] == SIZE_MAX) off += align256(pl.AL * 4);
    slots[i].off_dB = off; if (hostB[i] && pin_inB_off[i] == SIZE_MAX) off += align256(pl.BL * 4);
    slots[i].off_dC = off;
    if ((runs[i].hostC && pin_out_off[i] == SIZE_MAX) || runs[i].stagedC) off += align256(d.CL * 4);
  }
  // staged inputs and staged outputs each sit contiguously in the arena, in
  // the order of their pinned host copies, so one copy moves each way
  const size_t off_stage_in = off;
  off += align256(stage_in);
  const size_t off_stage_out = off;
  off += align256(stage_out);
  // ---- shared B transforms: in a class of two or more levels, items whose B
  // is the same device array (same pointer and length) get one B slot, packed
  // and transformed once (the splitting tree's P_l*Q_r and Q_l*Q_r share Q_r,
  // the nodes of a conversion depth share their power); they take the widest
  // of their widths, which fits each of them at the class's length
  std::vector<int> bslot(nw, -1);
  std::map<std::pair<size_t, bool>, std::vector<int>> owners;  // per class: item (class order) of each slot
  for (auto &c : classes) {
    std::vector<int> &own = owners[c.first];
    if (c.first.second) continue;
    std::map<std::pair<const uint32_t *, size_t>, std::vector<size_t>> groups;
    for (size_t k = 0; k < c.second.size(); k++) {
      const size_t i = c.second[k];
      const Plan &pl = works[i]->pl;
      const bc_mul_desc &d = items[works[i]->idx];
      if (pl.shape.levels >= 2 && !hostB[i] && !g.forced_width && g.share_b) groups[{d.B, pl.BL}].push_back(k);
      else { bslot[i] = (int)own.size(); own.push_back((int)k); }
    }
    for (auto &gr : groups) {
      int bmax = 0;
      for (size_t k : gr.second) bmax = std::max(bmax, works[c.second[k]]->pl.b);
      int slot = -1;
      for (size_t k : gr.second) {
        Work *w = works[c.second[k]];
        if (w->bcap < bmax) {  // redone at a narrower width: keeps its own B
          bslot[c.second[k]] = (int)own.size();
          own.push_back((int)k);
          continue;
        }
        if (slot < 0) {
          slot = (int)own.size();
          own.push_back((int)k);
        }
        if (w->pl.b != bmax) {
          w->pl.b = bmax;
          plan_finish(w->pl);
        }
        bslot[c.second[k]] = slot;
      }
    }
  }
  struct ClassSlab { size_t offA = 0, offB = 0; };
  std::map<std::pair<size_t, bool>, ClassSlab> slab;
  for (auto &c : classes) {
    const size_t M = c.first.first, n = c.second.size();
    ClassSlab cs;
    cs.offA = off; off += n * align256(M * 16);
    if (!c.first.second) { cs.offB = off; off += owners[c.first].size() * align256(M * 16); }
    slab[c.first] = cs;
  }
  size_t status_words = 0;
  for (size_t i = 0; i < nw; i++) {
    const Plan &pl = works[i]->pl;
    if (pl.shape.levels > 1) {
      slots[i].off_rec = off;
      off += align256((size_t)pl.shape.M / 4 * sizeof(RunRec));
      slots[i].off_status = status_words;
      status_words += pl.ntiles;
    }
  }
  // err, flags, counters and status words: one region, cleared by one memset
  const size_t off_err = off; off += align256(nw * 8);
  const size_t off_flags = off; off += align256(nw * 4);
  const size_t off_ctr = off; off += 256 * (classes.size() + 1);
  // per-block counters of the fused middle pass, per class that uses it
  std::map<std::pair<size_t, bool>, size_t> blk_off;
  const size_t off_blk = off;
  for (auto &c : classes) {
    const Shape &cs = works[c.second[0]]->pl.shape;
    if (!fused_ok(cs)) continue;
    blk_off[c.first] = off - off_blk;
    off += align256((size_t)8 * c.second.size() * cs.L1);
  }
  const size_t off_status = off; off += align256(status_words * 4);
  const size_t zero_end = off;
  const size_t off_desc = off; off += align256(nw * sizeof(ItemDesc));
  // B-slot owners of every class, after the descriptors (copied with them)
  std::map<std::pair<size_t, bool>, size_t> own_off;
  size_t own_words = 0;
  for (auto &c : classes) {
    own_off[c.first] = own_words;
    own_words += owners[c.first].size();
  }
  off += align256(own_words * 4);
  int r = arena_reserve(off);
  if (r) return r;
  char *base = g.arena;

  // ---- inputs
  pt.next(&g_prof.copy_in);
  if (stage_in) {
    std::vector<SpanJob> jobs;  // in increasing span offset
    jobs.reserve(2 * nw);
    for (size_t i = 0; i < nw; i++) {
      const bc_mul_desc &d = items[works[i]->idx];
      if (pin_in_off[i] != SIZE_MAX) jobs.push_back({pin_in_off[i], (char *)d.A, works[i]->pl.AL * 4});
      if (pin_inB_off[i] != SIZE_MAX) jobs.push_back({pin_inB_off[i], (char *)d.B, works[i]->pl.BL * 4});
    }
    if ((r = stage_h2d(base + off_stage_in, jobs, stage_in))) return r;
    st->h2d_bytes += stage_in;
    g_prof.bytes_in += stage_in;
  }
  bool b_late = false;  // B of the single product arrives on the copy stream
  for (size_t i = 0; i < nw; i++) {
    const bc_mul_desc &d = items[works[i]->idx];
    const Plan &pl = works[i]->pl;
    if (!hostA[i]) runs[i].dA = d.A;
    else if (pin_in_off[i] != SIZE_MAX) runs[i].dA = (const uint32_t *)(base + off_stage_in + pin_in_off[i]);
    else {
      runs[i].dA = (const uint32_t *)(base + slots[i].off_dA);
      CK(cudaMemcpyAsync((void *)runs[i].dA, d.A, pl.AL * 4, cudaMemcpyHostToDevice, g.stream));
      st->h2d_bytes += pl.AL * 4;
    }
    if (pl.square) runs[i].dB = runs[i].dA;
    else if (!hostB[i]) runs[i].dB = d.B;
    else if (pin_inB_off[i] != SIZE_MAX) runs[i].dB = (const uint32_t *)(base + off_stage_in + pin_inB_off[i]);
    else {
      runs[i].dB = (const uint32_t *)(base + slots[i].off_dB);
      if (nw == 1 && pl.shape.levels >= 2 && pl.BL >= ((size_t)1 << 20) && !graph) {
        // a single large product: B crosses on the copy stream (after the
        // library stream's earlier work, which may still read this slot)
        // while the outer pass packs A
        if (!g.copy_stream) CK(cudaStreamCreateWithFlags(&g.copy_stream, cudaStreamNonBlocking));
        for (auto &e : g.copy_ev)
          if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaEventRecord(g.copy_ev[0], g.stream));
        CK(cudaStreamWaitEvent(g.copy_stream, g.copy_ev[0], 0));
        CK(cudaMemcpyAsync((void *)runs[i].dB, d.B, pl.BL * 4, cudaMemcpyHostToDevice, g.copy_stream));
        CK(cudaEventRecord(g.copy_ev[1], g.copy_stream));
        b_late = true;
      } else {
        CK(cudaMemcpyAsync((void *)runs[i].dB, d.B, pl.BL * 4, cudaMemcpyHostToDevice, g.stream));
      }
      st->h2d_bytes += pl.BL * 4;
    }
    if (pin_out_off[i] != SIZE_MAX) runs[i].dC = (uint32_t *)(base + off_stage_out + pin_out_off[i]);
    else runs[i].dC = (runs[i].hostC || runs[i].stagedC) ? (uint32_t *)(base + slots[i].off_dC) : d.C;
  }
  CK(cudaMemsetAsync(base + off_err, 0, zero_end - off_err, g.stream));

  // ---- descriptors
  std::vector<ItemDesc> desc(nw);
  std::vector<size_t> order;
  order.reserve(nw);
  for (auto &c : classes) {
    unsigned long long tile0 = 0;
    const ClassSlab &cs = slab[c.first];
    size_t k = 0;
    for (size_t i : c.second) {
      const bc_mul_desc &d = items[works[i]->idx];
      const Plan &pl = works[i]->pl;
      ItemDesc &it = desc[order.size()];
      order.push_back(i);
      const size_t M = pl.shape.M;
      it.A = runs[i].dA;
      it.B = runs[i].dB;
      it.C = runs[i].dC;
      it.AL = pl.AL; it.BL = pl.BL; it.CL = d.CL;
      it.ndA = pl.ndA; it.ndB = pl.square ? pl.ndA : pl.ndB;
      it.bufA = (double2 *)(base + cs.offA + k * align256(M * 16));
      it.bslot = pl.square ? 0 : bslot[i];
      it.bufB = pl.square ? nullptr : (double2 *)(base + cs.offB + (size_t)it.bslot * align256(M * 16));
      it.rec = nullptr; it.status = nullptr;
      if (pl.shape.levels > 1) {
        it.rec = (RunRec *)(base + slots[i].off_rec);
        it.status = (uint32_t *)(base + off_status) + slots[i].off_status;
      }
      it.nwords = pl.nwords;
      it.nruns = pl.nruns;
      it.tile0 = tile0;
      tile0 += pl.ntiles;
      it.err = (unsigned long long *)(base + off_err) + i;
      it.flags = (unsigned int *)(base + off_flags) + i;
      it.b = pl.b;
      it.square = pl.square ? 1 : 0;
      it.a16 = stage16_ok(it.A, pl);
      it.b16 = stage16_ok(it.B, pl);
      k++;
    }
  }
  ItemDesc *ddesc = (ItemDesc *)(base + off_desc);
  // descriptors and, later, the outcomes go through one pinned block: the
  // descriptors at its start, the outcomes (err, flags) after them
  // (the B-slot owners right after the descriptors, as in the arena)
  const size_t desc_bytes = align256(nw * sizeof(ItemDesc)) + own_words * 4;
  const size_t pin_desc = align256(desc_bytes), pin_outc = off_flags + nw * 4 - off_err;
  if ((r = pin_small_reserve(pin_desc + pin_outc))) return r;
  memcpy(g.pin_small, desc.data(), nw * sizeof(ItemDesc));
  {
    int *po = (int *)((char *)g.pin_small + align256(nw * sizeof(ItemDesc)));
    for (auto &c : classes) {
      const std::vector<int> &own = owners[c.first];
      std::copy(own.begin(), own.end(), po + own_off[c.first]);
    }
  }
  CK(cudaMemcpyAsync(ddesc, g.pin_small, desc_bytes, cudaMemcpyHostToDevice, g.stream));
  const int *down = (const int *)((const char *)ddesc + align256(nw * sizeof(ItemDesc)));
  unsigned int *ctr = (unsigned int *)(base + off_ctr);

  // ---- launches: one class after another on the library stream, or, for
  // several classes, round robin over the class streams (forked from and
  // joined back into the library stream).  Per-kernel timing and the
  // cooperative fused kernel keep the single stream.
  pt.next(&g_prof.launch);
  // graph mode: every table exists before the capture (a new table's upload
  // synchronises the library stream), launches go to the capture stream
  cudaStream_t lstream = g.stream;
  CaptureGuard cap;
  if (graph) {
    for (auto &c : classes) {
      Tables *tb = nullptr;
      if ((r = ensure_tables(works[c.second[0]]->pl.shape, &tb))) return r;
    }
    if (!g.cap_stream) CK(cudaStreamCreateWithFlags(&g.cap_stream, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(g.cap_stream, cudaStreamCaptureModeRelaxed));
    cap.s = lstream = g.cap_stream;
  } else {
    CK(cudaEventRecord(g.ev0, g.stream));
  }
  const int nstreams = (classes.size() > 1 && !g.time_kernels && !g.fused && !b_late)
                           ? (int)std::min<size_t>(classes.size(), 4) : 0;
  if (nstreams) {
    for (int k = 0; k < 5; k++)
      if (!g.class_ev[k]) CK(cudaEventCreateWithFlags(&g.class_ev[k], cudaEventDisableTiming));
    CK(cudaEventRecord(g.class_ev[4], lstream));
    for (int k = 0; k < nstreams; k++) {
      if (!g.class_stream[k]) CK(cudaStreamCreateWithFlags(&g.class_stream[k], cudaStreamNonBlocking));
      CK(cudaStreamWaitEvent(g.class_stream[k], g.class_ev[4], 0));
    }
  }
  size_t first = 0, cls = 0;
  for (auto &c : classes) {
    const size_t n = c.second.size();
    const Plan &pl = works[c.second[0]]->pl;
    const Shape &s = pl.shape;
    const bool sq = c.first.second;
    Tables *tb = nullptr;
    r = ensure_tables(s, &tb);
    if (r) return r;
    ClassParams p = class_params(s, *tb);
    p.items = ddesc + first;
    p.nitems = (int)n;
    p.sq = sq ? 1 : 0;
    p.counter = ctr + 64 * cls;
    p.blkdone = nullptr;
    if (blk_off.count(c.first)) p.blkdone = (unsigned int *)(base + off_blk + blk_off[c.first]);
    p.slabA = (double2 *)(base + slab[c.first].offA);
    p.slabB = sq ? nullptr : (double2 *)(base + slab[c.first].offB);
    p.nb = sq ? 0 : (int)owners[c.first].size();
    p.bowner = sq ? nullptr : down + own_off[c.first];
    p.fwd_ops = 0;
    p.slab_elems = align256(s.M * 16) / 16;
    unsigned long long tiles = 0;
    bool w16 = true;  // every item of the class has width 16: the carry pass specialised for it
    for (size_t k = first; k < first + n; k++) {
      tiles += works[order[k]]->pl.ntiles;
      w16 = w16 && works[order[k]]->pl.b == 16;
    }
    p.carry_tiles = tiles;
    const ClassSlab &cs = slab[c.first];
    cudaStream_t cstream = nstreams ? g.class_stream[cls % nstreams] : lstream;
    if ((r = launch_class(s, sq, p, (long long)n, tiles, (double2 *)(base + cs.offA),
                          sq ? nullptr : (double2 *)(base + cs.offB), cstream, true, &st->launches,
                          b_late ? g.copy_ev[1] : nullptr, w16,
                          g.pdl && !graph && !g.time_kernels && !g.fused && (size_t)s.M <= kPdlMaxPoints)))
      return r;
    first += n;
    cls++;
  }
  for (int k = 0; k < nstreams; k++) {
    CK(cudaEventRecord(g.class_ev[k], g.class_stream[k]));
    CK(cudaStreamWaitEvent(lstream, g.class_ev[k], 0));
  }
  if (graph) {
    cudaGraph_t gr = nullptr;
    cap.s = nullptr;
    CK(cudaStreamEndCapture(g.cap_stream, &gr));
    if ((r = launch_graph(gr, st))) return r;
  }
  CK(cudaEventRecord(g.ev1, g.stream));
  st->classes += classes.size();

  // ---- outcomes, then outputs of the products that passed
  char *outc = (char *)g.pin_small + pin_desc;
  CK(cudaMemcpyAsync(outc, base + off_err, pin_outc, cudaMemcpyDeviceToHost, g.stream));
  pt.next(&g_prof.wait);
  CK(cudaStreamSynchronize(g.stream));
  std::vector<unsigned long long> errs(nw);
  std::vector<unsigned> flags(nw);
  memcpy(errs.data(), outc, nw * 8);
  memcpy(flags.data(), outc + (off_flags - off_err), nw * 4);
  pt.next(&g_prof.copy_out);
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, g.ev0, g.ev1));
  st->device_ms += ms;
  if (g.time_kernels && !g.kev.empty()) {
    cudaEvent_t prev = g.ev0;
    for (size_t k = 0; k < g.kev.size(); k++) {
      float km = 0;
      cudaEventElapsedTime(&km, prev, g.kev[k]);
      g.ktimes[g.ktimes.size() - g.kev.size() + k].second = km;
      prev = g.kev[k];
    }
    for (auto e : g.kev) g.kev_pool.push_back(e);
    g.kev.clear();
  }
  bool copies = false, staged_out = false;
  std::vector<char> ok(nw);
  for (size_t i = 0; i < nw; i++) {
    double e;
    memcpy(&e, &errs[i], 8);
    works[i]->err = e;
    works[i]->flags = flags[i];
    ok[i] = (((e < g.max_err) && !(flags[i] & FLAG_TOPCARRY)) || g.forced_width) && !(flags[i] & FLAG_TIMEOUT);
    const bc_mul_desc &d = items[works[i]->idx];
    if (!ok[i]) continue;
    if (runs[i].hostC) {
      if (pin_out_off[i] != SIZE_MAX) {
        staged_out = true;  // one copy of the whole staged span below
      } else {
        CK(cudaMemcpyAsync(d.C, runs[i].dC, d.CL * 4, cudaMemcpyDeviceToHost, g.stream));
        st->d2h_bytes += d.CL * 4;
      }
      copies = true;
    } else if (runs[i].stagedC) {
      CK(cudaMemcpyAsync(d.C, runs[i].dC, d.CL * 4, cudaMemcpyDeviceToDevice, g.stream));
      copies = true;
    }
  }
  if (staged_out) {
    std::vector<SpanJob> jobs;  // in increasing span offset
    jobs.reserve(nw);
    for (size_t i = 0; i < nw; i++)
      if (ok[i] && pin_out_off[i] != SIZE_MAX)
        jobs.push_back({pin_out_off[i], (char *)items[works[i]->idx].C, items[works[i]->idx].CL * 4});
    if ((r = stage_d2h(base + off_stage_out, jobs, stage_out))) return r;
    st->d2h_bytes += stage_out;
    g_prof.bytes_out += stage_out;
  }
  if (copies) CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

int mul_batch_locked(const bc_mul_desc *items, size_t n, bc_batch_stats *st, Plan *first_plan = nullptr,
                     unsigned flags = 0) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (n && !items) return fail(BC_ERR_INVALID);
  auto t0 = std::chrono::steady_clock::now();
  g_prof.calls++;
  std::vector<Work> works;
  works.reserve(n);
  PhaseTimer ppt(&g_prof.plan);
  for (size_t i = 0; i < n; i++) {
    const bc_mul_desc &d = items[i];
    if (d.CL && !d.C) return fail(BC_ERR_INVALID);
    if ((d.AL && !d.A) || (d.BL && !d.B)) return fail(BC_ERR_INVALID);
    if (d.CL == 0) continue;
    const bool zero = d.AL == 0 || d.BL == 0;
    if (zero) {
      if ((flags & BC_BATCH_DEVICE_OPERANDS) || (!(flags & BC_BATCH_HOST_OPERANDS) && is_device_ptr(d.C)))
        CK(cudaMemsetAsync(d.C, 0, d.CL * 4, g.stream));
      else memset(d.C, 0, d.CL * 4);
      continue;
    }
    Work w;
    w.idx = i;
    w.bcap = 24;
    const bool square = d.A == d.B && d.AL == d.BL;
    if (!make_plan(d.AL, d.BL, d.CL, square, w.bcap, w.pl)) return fail(BC_ERR_TOO_LARGE);
    works.push_back(w);
  }
  st->items = n;
  ppt.next(&g_prof_rest);  // the attempts are timed inside run_attempt
  if (g.time_kernels) g.ktimes.clear();
  // attempts: redo items whose rounding error reached the limit at a narrower width
  for (int attempt = 0; attempt < 12; attempt++) {
    std::vector<Work *> todo;
    for (auto &w : works) if (!w.done) todo.push_back(&w);
    if (todo.empty()) break;
    // split into chunks that fit the arena limit
    size_t i0 = 0;
    while (i0 < todo.size()) {
      size_t bytes = 0, i1 = i0;
      while (i1 < todo.size()) {
        const bc_mul_desc &d = items[todo[i1]->idx];
        size_t need = work_bytes(todo[i1]->pl) + align256(d.AL * 4) + align256(d.BL * 4) + align256(d.CL * 4) + 1024;
        if (i1 > i0 && bytes + need > g.arena_limit / 2) break;
        bytes += need;
        i1++;
      }
      std::vector<Work *> chunk(todo.begin() + i0, todo.begin() + i1);
      int r = run_attempt(items, chunk, st, flags);
      if (r) return r;
      i0 = i1;
    }
    for (Work *w : todo) {
      if (w->flags & FLAG_TIMEOUT) return fail(BC_ERR_TIMEOUT);
      const bool bad = !(w->err < g.max_err) || (w->flags & FLAG_TOPCARRY);
      if (!bad || g.forced_width) {
        st->max_round_err = std::max(st->max_round_err, w->err);  // of the accepted attempt
        if (w->flags & FLAG_TOPCARRY) return fail(BC_ERR_CARRY);
        w->done = true;
        continue;
      }
      // narrower digits (and a longer transform if needed)
      const bc_mul_desc &d = items[w->idx];
      w->bcap = w->pl.b - 1;
      w->retries++;
      st->retries++;
      if (g.verbose)
        fprintf(stderr, "bc_gpu: item %zu M=%d b=%d err=%.3g flags=%u -> retry at b<=%d\n", w->idx,
                w->pl.shape.M, w->pl.b, w->err, w->flags, w->bcap);
      if (w->bcap < 8 || !make_plan(d.AL, d.BL, d.CL, w->pl.square, w->bcap, w->pl)) return fail(BC_ERR_PRECISION);
    }
  }
  for (auto &w : works)
    if (!w.done) return fail(BC_ERR_PRECISION);
  if (first_plan && !works.empty()) *first_plan = works[0].pl;
  st->total_ms += ms_since(t0);
  return BC_OK;
}

// ------------------------------------------------------------------ e's series on the device
// Binary splitting of sum 1/k! with every value kept in device memory: the
// leaves (LEAF_TERMS terms each) by k_bsr_leaves, then one level at a time
// the products P_l*Q_r and Q_l*Q_r of neighbouring nodes in one batch
// (device operands), their lengths by k_trim and P = P_l*Q_r + P_r by k_add.
// Only the lengths cross to the host between steps; P and Q of the root at
// the end.
struct DevNum {
  uint32_t *p = nullptr;
  size_t len = 0;
};

// Scratch of the tree and Newton drivers, freed on scope exit.  Stream-ordered
// (cudaMallocAsync / cudaFreeAsync on the library stream, from the device's
// default pool, which bc_gpu_init tells to keep freed memory): no device-wide
// synchronisation per free and no driver allocation per level or operand.
// Every user of a DevBuf works on the library stream.
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { if (p) cudaFreeAsync(p, g.stream); }
  int alloc(size_t bytes) {
    CK(cudaMallocAsync(&p, std::max<size_t>(bytes, 256), g.stream));
    if (poison_on()) CK(cudaMemsetAsync(p, 0xA5, std::max<size_t>(bytes, 256), g.stream));
    return BC_OK;
  }
};

// ------------------------------------------------------------------ radix conversion leaves
// Leaves whose fractions and digits are already in device memory, in one launch.
int radix_leaves_device(const std::vector<RadixLeaf> &d, double alpha) {
  if (d.empty()) return BC_OK;
  const size_t o_flag = align256(d.size() * sizeof(RadixLeaf)), total = o_flag + 256;
  int r = arena_reserve(total);
  if (r) return r;
  char *base = g.arena;
  CK(cudaMemcpyAsync(base, d.data(), d.size() * sizeof(RadixLeaf), cudaMemcpyHostToDevice, g.stream));
  CK(cudaMemsetAsync(base + o_flag, 0, 256, g.stream));
  const unsigned grid =
      (unsigned)std::min<size_t>((d.size() + RADIX_WARPS - 1) / RADIX_WARPS, (size_t)g.sm_count * 16);
  k_radix_leaves<<<grid, 32 * RADIX_WARPS, 0, g.stream>>>((const RadixLeaf *)base, (int)d.size(), alpha,
                                                          (unsigned *)(base + o_flag));
  CK(cudaGetLastError());
  unsigned flag = 0;
  CK(cudaMemcpyAsync(&flag, base + o_flag, 4, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return flag ? fail(BC_ERR_TOO_LARGE) : BC_OK;
}

// All leaves of one conversion in one launch: the fractions cross to the
// device in one staged span, the digits come back in another.
int radix_leaves_locked(const bc_radix_leaf *lv, size_t count, double alpha) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (count == 0) return BC_OK;
  if (!lv) return fail(BC_ERR_INVALID);
  std::vector<size_t> in_off(count), out_off(count);
  size_t in_bytes = 0, out_bytes = 0;
  for (size_t i = 0; i < count; i++) {
    const bc_radix_leaf &l = lv[i];
    if ((l.len && !l.y) || (l.k && !l.s)) return fail(BC_ERR_INVALID);
    if (l.len + 1 > (size_t)RADIX_WINDOW || l.n + 1 > (size_t)RADIX_WINDOW || l.n > l.len + 1 ||
        l.k > 0xffffffffu)
      return fail(BC_ERR_TOO_LARGE);
    in_off[i] = in_bytes;
    in_bytes += align256(l.len * 4);
    out_off[i] = out_bytes;
    out_bytes += align256(l.k * 4);
  }
  const size_t o_desc = 0, o_in = align256(count * sizeof(RadixLeaf)), o_out = o_in + in_bytes,
               o_flag = o_out + out_bytes, total = o_flag + 256;
  int r = arena_reserve(total);
  if (r) return r;
  char *base = g.arena;
  std::vector<SpanJob> jobs;
  jobs.reserve(count);
  std::vector<RadixLeaf> d(count);
  for (size_t i = 0; i < count; i++) {
    const bc_radix_leaf &l = lv[i];
    if (l.len) jobs.push_back({in_off[i], (char *)l.y, l.len * 4});
    d[i] = {(const uint32_t *)(base + o_in + in_off[i]), (uint32_t *)(base + o_out + out_off[i]), (uint32_t)l.len,
            (uint32_t)l.n, (uint32_t)l.k, 0u};
  }
  if ((r = stage_h2d(base + o_in, jobs, in_bytes))) return r;
  CK(cudaMemcpyAsync(base + o_desc, d.data(), count * sizeof(RadixLeaf), cudaMemcpyHostToDevice, g.stream));
  CK(cudaMemsetAsync(base + o_flag, 0, 256, g.stream));
  const unsigned grid =
      (unsigned)std::min<size_t>((count + RADIX_WARPS - 1) / RADIX_WARPS, (size_t)g.sm_count * 16);
  k_radix_leaves<<<grid, 32 * RADIX_WARPS, 0, g.stream>>>((const RadixLeaf *)(base + o_desc), (int)count, alpha,
                                                          (unsigned *)(base + o_flag));
  CK(cudaGetLastError());
  unsigned flag = 0;
  CK(cudaMemcpyAsync(&flag, base + o_flag, 4, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  if (flag) return fail(BC_ERR_TOO_LARGE);
  jobs.clear();
  for (size_t i = 0; i < count; i++)
    if (lv[i].k) jobs.push_back({out_off[i], (char *)lv[i].s, lv[i].k * 4});
  if ((r = stage_d2h(base + o_out, jobs, out_bytes))) return r;
  CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

// ------------------------------------------------------------------ radix conversion tree on the device
// The conversion tree the caller planned (split sizes and power-table entry
// per internal node, bigfloat/radix.c:228-318), run with every value in
// device memory: top-down, one batch of products y * 10^(9(k-kl)) per depth;
// the high child's fraction is a view of the top limbs of y, the low child's
// a view of limbs [n - nl, n) of the product (zero-padded to n limbs, as the
// reference's realloc pads it); all leaves in one launch; bottom-up, one
// fix-up and one copy launch per depth for the merges.
// The tree on device operands: dy (ylen limbs) and the table entries
// dtab[t] (table_len[t] limbs) are in device memory.
int radix_tree_core(const uint32_t *dy, size_t ylen, const bc_radix_node *nodes, size_t nn,
                    const uint32_t *const *dtab, const size_t *table_len, int ntable, double alpha, uint32_t *out) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!dy || !ylen || !nodes || !nn || !out || (ntable && (!dtab || !table_len))) return fail(BC_ERR_INVALID);
  // depths (children come after their parent) and buffer sizes
  std::vector<int> depth(nn, 0);
  int maxd = 0;
  std::vector<size_t> ylenv(nn, 0), prod_off(nn, SIZE_MAX), prod_len(nn, 0), s_off(nn);
  ylenv[0] = ylen;
  size_t prod_total = 0, s_total = 0;
  for (size_t i = 0; i < nn; i++) {
    const bc_radix_node &x = nodes[i];
    s_off[i] = s_total;
    s_total += (x.k + 63) & ~size_t(63);
    if (x.child_h < 0) continue;
    const size_t h = (size_t)x.child_h, l = (size_t)x.child_l;
    if (h <= i || l <= i || h >= nn || l >= nn || x.table < 0 || x.table >= ntable) return fail(BC_ERR_INVALID);
    depth[h] = depth[l] = depth[i] + 1;
    maxd = std::max(maxd, depth[h]);
    const size_t nh = nodes[h].n, nl = nodes[l].n;
    if (nh > x.n || nl > x.n || ylenv[i] < x.n - nh) return fail(BC_ERR_INVALID);
    ylenv[h] = ylenv[i] - (x.n - nh);
    ylenv[l] = nl;
    prod_len[i] = ylenv[i] + table_len[x.table];
    prod_off[i] = prod_total;
    prod_total += (std::max(prod_len[i], x.n) + 63) & ~size_t(63);
  }
  // $BC_STATS: time of each step (products per depth, leaves, merges) on stderr
  const bool stats = getenv("BC_STATS") != nullptr;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto secs = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  auto sync_secs = [&](std::chrono::steady_clock::time_point t0) -> double {
    if (stats) cudaStreamSynchronize(g.stream);
    return secs(t0);
  };
  double t_mul_total = 0;
  // device buffers: products, digits
  DevBuf dprod, ds, dmeta;
  int r;
  if ((r = dprod.alloc(prod_total * 4)) || (r = ds.alloc(s_total * 4))) return r;
  uint32_t *dp = (uint32_t *)dprod.p, *dsd = (uint32_t *)ds.p;
  std::vector<const uint32_t *> yptr(nn, nullptr);
  yptr[0] = dy;
  // top-down products, one batch per depth
  for (int d = 0; d < maxd; d++) {
    std::vector<bc_mul_desc> md;
    for (size_t i = 0; i < nn; i++) {
      const bc_radix_node &x = nodes[i];
      if (depth[i] != d || x.child_h < 0) continue;
      uint32_t *C = dp + prod_off[i];
      if (x.n > prod_len[i]) CK(cudaMemsetAsync(C + prod_len[i], 0, (x.n - prod_len[i]) * 4, g.stream));
      md.push_back({C, prod_len[i], yptr[i], ylenv[i], dtab[x.table], table_len[x.table]});
      yptr[x.child_h] = yptr[i] + (x.n - nodes[x.child_h].n);
      yptr[x.child_l] = C + (x.n - nodes[x.child_l].n);
    }
    bc_batch_stats st{};
    const auto t0 = now();
    if (!md.empty() && (r = mul_batch_locked(md.data(), md.size(), &st, nullptr, BC_BATCH_DEVICE_OPERANDS)))
      return r;
    if (stats) {
      const double t = secs(t0);
      t_mul_total += t;
      fprintf(stderr, "      conversion depth %d: %zu products, %.4f s (device %.4f s)\n", d, md.size(), t,
              st.device_ms / 1e3);
    }
  }
  auto t_step = now();
  // leaves
  std::vector<RadixLeaf> lv;
  for (size_t i = 0; i < nn; i++) {
    const bc_radix_node &x = nodes[i];
    if (x.child_h >= 0) continue;
    if (ylenv[i] + 1 > (size_t)RADIX_WINDOW || x.n + 1 > (size_t)RADIX_WINDOW || x.n > ylenv[i] + 1 ||
        x.k > 0xffffffffu)
      return fail(BC_ERR_TOO_LARGE);
    lv.push_back({yptr[i], dsd + s_off[i], (uint32_t)ylenv[i], (uint32_t)x.n, (uint32_t)x.k, 0u});
  }
  if ((r = radix_leaves_device(lv, alpha))) return r;
  const double t_leaves = sync_secs(t_step);
  t_step = now();
  // bottom-up merges, one depth at a time
  const size_t o_flag = align256(nn * sizeof(MergeDesc));
  if ((r = dmeta.alloc(o_flag + nn * 4))) return r;
  MergeDesc *dm = (MergeDesc *)dmeta.p;
  unsigned *dflag = (unsigned *)((char *)dmeta.p + o_flag);
  for (int d = maxd - 1; d >= 0; d--) {
    std::vector<MergeDesc> mg;
    unsigned long long units = 0;
    for (size_t i = 0; i < nn; i++) {
      const bc_radix_node &x = nodes[i];
      if (depth[i] != d || x.child_h < 0) continue;
      const size_t h = (size_t)x.child_h, l = (size_t)x.child_l;
      const unsigned long long kh = nodes[h].k, kl = nodes[l].k;
      if (kl != x.kl || kh + kl - 1 != x.k || kh == 0 || kl == 0) return fail(BC_ERR_INVALID);
      mg.push_back({dsd + s_off[h], dsd + s_off[l], dsd + s_off[i], kh, kl, units});
      units += (kh - 1 + kl + MERGE_UNIT - 1) / MERGE_UNIT;
    }
    if (mg.empty()) continue;
    CK(cudaMemcpyAsync(dm, mg.data(), mg.size() * sizeof(MergeDesc), cudaMemcpyHostToDevice, g.stream));
    k_merge_fix<<<(unsigned)((mg.size() + 127) / 128), 128, 0, g.stream>>>(dm, (int)mg.size(), dflag);
    CK(cudaGetLastError());
    const unsigned grid = (unsigned)std::min<unsigned long long>(units, (unsigned long long)g.sm_count * 8);
    k_merge_copy<<<grid, 256, 0, g.stream>>>(dm, (int)mg.size(), units, dflag);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(g.stream));  // mg is rewritten for the next depth
  }
  if (stats)
    fprintf(stderr, "      conversion tree: products %.3f s, %zu leaves %.3f s, merges %.3f s\n", t_mul_total, lv.size(),
            t_leaves, sync_secs(t_step));
  // the root's digits: to the caller's device array, or through the ring
  if (is_device_ptr(out)) {
    CK(cudaMemcpyAsync(out, dsd + s_off[0], nodes[0].k * 4, cudaMemcpyDeviceToDevice, g.stream));
  } else {
    std::vector<SpanJob> jobs{{0, (char *)out, nodes[0].k * 4}};
    if ((r = stage_d2h((const char *)(dsd + s_off[0]), jobs, nodes[0].k * 4))) return r;
  }
  CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

// Host fraction and host table entries: both cross once, then the core.
int radix_tree_locked(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nn,
                      const uint32_t *const *table, const size_t *table_len, int ntable, double alpha,
                      uint32_t *out) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!y || !ylen || !nodes || !nn || !out || (ntable && (!table || !table_len))) return fail(BC_ERR_INVALID);
  size_t tab_total = 0;
  std::vector<size_t> tab_off(ntable);
  for (int t = 0; t < ntable; t++) {
    tab_off[t] = tab_total;
    tab_total += (table_len[t] + 63) & ~size_t(63);
  }
  const size_t ypad = (ylen + 63) & ~size_t(63);
  DevBuf din;
  int r;
  if ((r = din.alloc((ypad + tab_total) * 4))) return r;
  uint32_t *dy = (uint32_t *)din.p;
  std::vector<SpanJob> jobs;
  jobs.push_back({0, (char *)y, ylen * 4});
  for (int t = 0; t < ntable; t++)
    if (table_len[t]) jobs.push_back({(ypad + tab_off[t]) * 4, (char *)table[t], table_len[t] * 4});
  if ((r = stage_h2d((char *)din.p, jobs, (ypad + tab_total) * 4))) return r;
  std::vector<const uint32_t *> dtab(ntable);
  for (int t = 0; t < ntable; t++) dtab[t] = dy + ypad + tab_off[t];
  return radix_tree_core(dy, ylen, nodes, nn, dtab.data(), table_len, ntable, alpha, out);
}

// Significant length of a product of CL limbs under the reference's trimming
// (bigfloat/mul.c:664-675): one top zero limb dropped, then, above 1000
// limbs, every top zero limb.
int trimmed_len(const uint32_t *dC, size_t CL, size_t *len) {
  size_t n = CL;
  uint32_t top[8];
  size_t have = 0, base = 0;  // top[] holds limbs [base, base + have)
  auto limb = [&](size_t i, uint32_t *v) -> int {
    if (i < base || i >= base + have) {
      have = std::min<size_t>(8, i + 1);
      base = i + 1 - have;
      CK(cudaMemcpyAsync(top, dC + base, have * 4, cudaMemcpyDeviceToHost, g.stream));
      CK(cudaStreamSynchronize(g.stream));
    }
    *v = top[i - base];
    return BC_OK;
  };
  uint32_t v = 0;
  int r;
  if (n && ((r = limb(n - 1, &v)))) return r;
  if (n && v == 0) n--;
  if (n > 1000)
    while (n > 0) {
      if ((r = limb(n - 1, &v))) return r;
      if (v) break;
      n--;
    }
  *len = n;
  return BC_OK;
}

// The power table of the conversion built in device memory: entry 0 comes
// from the host; entry i from entry steps[i].src < i by the step the
// reference's table construction takes (bigfloat/radix.c:156-205): times
// 10^9 (len + 1 limbs, untrimmed), a squaring (trimmed product), or a
// squaring then times 10^9 (trimmed square plus one limb).  The products
// are the library's own exact products on device operands.
int radix_tree_pow_locked(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nn, const uint32_t *t0,
                          size_t t0len, const bc_radix_pow_step *steps, int ntable, double alpha, uint32_t *out) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!y || !ylen || !nodes || !nn || !out || ntable < 1 || !t0 || !t0len || !steps) return fail(BC_ERR_INVALID);
  for (int i = 1; i < ntable; i++)
    if (steps[i].src < 0 || steps[i].src >= i || steps[i].op < 1 || steps[i].op > 3) return fail(BC_ERR_INVALID);
  std::vector<DevBuf> tab(ntable + 1);  // the last one holds y and 10^9
  std::vector<size_t> tlen(ntable);
  std::vector<const uint32_t *> dtab(ntable);
  int r;
  const size_t ypad = (ylen + 63) & ~size_t(63);
  if ((r = tab[ntable].alloc((ypad + 64) * 4))) return r;
  uint32_t *dy = (uint32_t *)tab[ntable].p, *dbase = dy + ypad;
  {
    std::vector<SpanJob> jobs{{0, (char *)y, ylen * 4}};
    if ((r = stage_h2d((char *)dy, jobs, ylen * 4))) return r;
    const uint32_t nine = DEC_BASE;
    CK(cudaMemcpyAsync(dbase, &nine, 4, cudaMemcpyHostToDevice, g.stream));
  }
  if ((r = tab[0].alloc(t0len * 4))) return r;
  CK(cudaMemcpyAsync(tab[0].p, t0, t0len * 4, cudaMemcpyHostToDevice, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  tlen[0] = t0len;
  dtab[0] = (const uint32_t *)tab[0].p;
  bc_batch_stats st{};
  const auto t_tab = std::chrono::steady_clock::now();
  for (int i = 1; i < ntable; i++) {
    const int j = steps[i].src, op = steps[i].op;
    const uint32_t *X = dtab[j];
    const size_t XL = tlen[j];
    if (op == 1) {  // times 10^9
      const size_t CL = XL + 1;
      if ((r = tab[i].alloc(CL * 4))) return r;
      bc_mul_desc d{(uint32_t *)tab[i].p, CL, X, XL, dbase, 1};
      if ((r = mul_batch_locked(&d, 1, &st, nullptr, BC_BATCH_DEVICE_OPERANDS))) return r;
      tlen[i] = CL;
    } else {
      const size_t CL = 2 * XL;
      DevBuf sq;
      if ((r = sq.alloc(CL * 4))) return r;
      bc_mul_desc d{(uint32_t *)sq.p, CL, X, XL, X, XL};
      if ((r = mul_batch_locked(&d, 1, &st, nullptr, BC_BATCH_DEVICE_OPERANDS))) return r;
      size_t L = 0;
      if ((r = trimmed_len((const uint32_t *)sq.p, CL, &L))) return r;
      if (op == 2) {
        tab[i].p = sq.p;
        sq.p = nullptr;
        tlen[i] = L;
      } else {  // then times 10^9 into L + 1 limbs
        if ((r = tab[i].alloc((L + 1) * 4))) return r;
        bc_mul_desc d2{(uint32_t *)tab[i].p, L + 1, (const uint32_t *)sq.p, L, dbase, 1};
        if ((r = mul_batch_locked(&d2, 1, &st, nullptr, BC_BATCH_DEVICE_OPERANDS))) return r;
        tlen[i] = L + 1;
      }
    }
    dtab[i] = (const uint32_t *)tab[i].p;
  }
  if (getenv("BC_STATS")) {
    cudaStreamSynchronize(g.stream);
    fprintf(stderr, "      conversion power table: %d entries, %.3f s\n", ntable,
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_tab).count());
  }
  return radix_tree_core(dy, ylen, nodes, nn, dtab.data(), tlen.data(), ntable, alpha, out);
}

// ------------------------------------------------------------------ Newton iteration in device memory
// Bigfloats held in device memory (value = sign * sum p[i] 2^(32(i+exp)),
// sign 1 positive, 0 negative, len 0 for zero), and the operations the
// reciprocal's Newton step uses, each with the semantics of the host library
// (bigfloat/mul.c:555-676, bigfloat/addsub.c:33-237) so the values are the
// same limb for limb.
struct DNum {
  std::shared_ptr<DevBuf> own;
  const uint32_t *p = nullptr;
  size_t len = 0;
  long long exp = 0;
  int sign = 1;
};

int dnum_alloc(DNum &x, size_t limbs) {
  x.own = std::make_shared<DevBuf>();
  int r = x.own->alloc(std::max<size_t>(limbs, 1) * 4);
  if (r) return r;
  x.p = (const uint32_t *)x.own->p;
  return BC_OK;
}

int dnum_upload(DNum &x, const bc_bignum &h) {
  x = DNum();
  x.len = h.len;
  x.exp = h.exp;
  x.sign = h.sign;
  if (!h.len) return BC_OK;
  int r = dnum_alloc(x, h.len);
  if (r) return r;
  std::vector<SpanJob> jobs{{0, (char *)h.coef, h.len * 4}};
  return stage_h2d((char *)x.own->p, jobs, h.len * 4);
}

// bigfloat_mul: operands chopped to their top p+2 limbs (all limbs when
// p = 0), the exact product, its top zero limb dropped (above 1000 limbs
// every top zero limb).
int dnum_mul(DNum &t, const DNum &a, const DNum &b, size_t p) {
  if (!a.len || !b.len) {
    t = DNum();
    return BC_OK;
  }
  const size_t pp = p == 0 ? a.len + b.len : p + 2;
  const uint32_t *A = a.p, *B = b.p;
  size_t AL = a.len, BL = b.len;
  long long ea = a.exp, eb = b.exp;
  if (AL > pp) { A += AL - pp; ea += (long long)(AL - pp); AL = pp; }
  if (BL > pp) { B += BL - pp; eb += (long long)(BL - pp); BL = pp; }
  DNum c;
  const size_t CL = AL + BL;
  int r;
  if ((r = dnum_alloc(c, CL))) return r;
  bc_mul_desc d{(uint32_t *)c.p, CL, A, AL, B, BL};
  bc_batch_stats st{};
  if ((r = mul_batch_locked(&d, 1, &st, nullptr, BC_BATCH_DEVICE_OPERANDS))) return r;
  if ((r = trimmed_len(c.p, CL, &c.len))) return r;
  c.exp = ea + eb;
  c.sign = a.sign == b.sign;
  t = c;
  return BC_OK;
}

// The window [bot, top) of a sum or difference at precision p and the
// exponent the reference gives its result (top - p, p the window length when
// untruncated).
void dnum_window(const DNum &a, const DNum &b, size_t p, long long *bot, long long *top, long long *e) {
  const long long ta = a.exp + (long long)a.len, tb = b.exp + (long long)b.len;
  *top = std::max(ta, tb);
  *bot = std::min(a.exp, b.exp);
  const long long tl = *top - *bot;
  const long long pp = p == 0 ? tl : (long long)p + 2;
  if (tl > pp) *bot = *top - pp;
  *e = *top - pp;
}

WinOp win_of(const DNum &x, long long bot, long long n) {
  WinOp w;
  w.x = x.p;
  w.lo = x.exp - bot;
  w.hi = x.len ? std::min(x.exp + (long long)x.len - bot, n) : w.lo;
  return w;
}

// _bigfloat_uadd / _bigfloat_usub: the window's limbs of a + b or a - b
// (|a| >= |b| assumed by the caller), sign of a; a sum keeps a carry limb, a
// difference drops its top zero limbs (zero when none is left).
int dnum_uaddsub(DNum &t, const DNum &a, const DNum &b, size_t p, bool sub) {
  long long bot, top, e;
  dnum_window(a, b, p, &bot, &top, &e);
  const long long n = top - bot;
  DNum c;
  int r;
  if ((r = dnum_alloc(c, (size_t)n + 1))) return r;
  const unsigned long long tiles = ((unsigned long long)n + ADD_TILE - 1) / ADD_TILE;
  DevBuf scratch;
  const size_t o_st = 256, o_top = o_st + align256(tiles * 4);
  if ((r = scratch.alloc(o_top + 256))) return r;
  char *sp = (char *)scratch.p;
  CK(cudaMemsetAsync(sp, 0, o_top + 256, g.stream));
  AddSubParams ap;
  ap.a = win_of(a, bot, n);
  ap.b = win_of(b, bot, n);
  ap.r = (uint32_t *)c.p;
  ap.n = (unsigned long long)n;
  ap.sub = sub ? 1 : 0;
  ap.tiles = tiles;
  ap.counter = (unsigned int *)sp;
  ap.cout = (unsigned int *)(sp + 4);
  ap.flags = (unsigned int *)(sp + 8);
  ap.status = (uint32_t *)(sp + o_st);
  if (n > 0) {
    const unsigned grid = (unsigned)std::min<unsigned long long>(tiles, (unsigned long long)g.sm_count * 8);
    k_addsub_win<<<grid, ADD_NT, 0, g.stream>>>(ap);
    CK(cudaGetLastError());
  }
  unsigned long long len = (unsigned long long)n;
  if (sub && n > 0) {
    unsigned long long *dtop = (unsigned long long *)(sp + o_top);
    const unsigned grid = (unsigned)std::min<unsigned long long>(((unsigned long long)n + 255) / 256,
                                                                 (unsigned long long)g.sm_count * 8);
    k_top_nonzero<<<grid, 256, 0, g.stream>>>(c.p, (unsigned long long)n, dtop);
    CK(cudaGetLastError());
  }
  unsigned int head[4];
  unsigned long long toplen = 0;
  CK(cudaMemcpyAsync(head, sp, 16, cudaMemcpyDeviceToHost, g.stream));
  if (sub && n > 0) CK(cudaMemcpyAsync(&toplen, sp + o_top, 8, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  if (head[2]) return fail(BC_ERR_TIMEOUT);
  if (sub) {
    len = toplen;
  } else if (head[1]) {
    const uint32_t one = 1;
    CK(cudaMemcpyAsync((uint32_t *)c.p + n, &one, 4, cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    len = (unsigned long long)n + 1;
  }
  if (len == 0) {
    t = DNum();
    return BC_OK;
  }
  c.len = (size_t)len;
  c.exp = e;
  c.sign = a.sign;
  t = c;
  return BC_OK;
}

// Compare |a| and |b| (bigfloat/addsub.c:33-63): 1, -1 or 0.
int dnum_ucmp(const DNum &a, const DNum &b, int *res) {
  const long long ta = a.exp + (long long)a.len, tb = b.exp + (long long)b.len;
  if (ta != tb) {
    *res = ta > tb ? 1 : -1;
    return BC_OK;
  }
  const long long lo = std::min(a.exp, b.exp), n = ta - lo + 1;
  const WinOp wa = win_of(a, lo, n), wb = win_of(b, lo, n);
  DevBuf scratch;
  int r;
  if ((r = scratch.alloc(256))) return r;
  unsigned long long *dhi = (unsigned long long *)scratch.p;
  CK(cudaMemsetAsync(dhi, 0, 8, g.stream));
  if (n > 0) {
    const unsigned grid =
        (unsigned)std::min<unsigned long long>(((unsigned long long)n + 255) / 256, (unsigned long long)g.sm_count * 8);
    k_first_diff<<<grid, 256, 0, g.stream>>>(wa, wb, (unsigned long long)n, dhi);
    CK(cudaGetLastError());
  }
  unsigned long long hi = 0;
  CK(cudaMemcpyAsync(&hi, dhi, 8, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  if (!hi) {
    *res = 0;
    return BC_OK;
  }
  const long long i = (long long)hi - 1;
  uint32_t x = 0, y = 0;
  if (i >= wa.lo && i < wa.hi) CK(cudaMemcpy(&x, wa.x + (i - wa.lo), 4, cudaMemcpyDeviceToHost));
  if (i >= wb.lo && i < wb.hi) CK(cudaMemcpy(&y, wb.x + (i - wb.lo), 4, cudaMemcpyDeviceToHost));
  *res = x > y ? 1 : -1;
  return BC_OK;
}

void dnum_neg(DNum &t) {
  if (t.len) t.sign = !t.sign;
}

// bigfloat_sub (bigfloat/addsub.c:212-237).
int dnum_sub(DNum &t, const DNum &a, const DNum &b, size_t p) {
  if (a.sign != b.sign) return dnum_uaddsub(t, a, b, p, false);
  int c = 0, r;
  if ((r = dnum_ucmp(a, b, &c))) return r;
  if (c > 0) return dnum_uaddsub(t, a, b, p, true);
  if ((r = dnum_uaddsub(t, b, a, p, true))) return r;
  dnum_neg(t);
  return BC_OK;
}

// The reciprocal's Newton levels (bigfloat/rcp.c:15-101) from r0 upward,
// levels[k] the precision of level k in increasing order:
//   r <- r - (r*x - 1)*r, each product and difference at that precision;
// then the quotient num * r at precision pdiv when num is given.
int newton_locked(const bc_bignum *den, const bc_bignum *r0, const size_t *levels, int nlev, const bc_bignum *num,
                  size_t pdiv, bc_bignum_out *out) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!den || !r0 || !out || nlev < 0 || (nlev && !levels)) return fail(BC_ERR_INVALID);
  const bool stats = getenv("BC_STATS") != nullptr;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto secs = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  int r;
  DNum D, R, N, one;
  auto t0 = now();
  if ((r = dnum_upload(D, *den)) || (r = dnum_upload(R, *r0))) return r;
  if (num && (r = dnum_upload(N, *num))) return r;
  {
    const uint32_t v = 1;
    bc_bignum h{&v, 1, 0, 1};
    if ((r = dnum_upload(one, h))) return r;
  }
  if (stats) fprintf(stderr, "      newton on the device: operands up %.3f s\n", secs(t0));
  for (int k = 0; k < nlev; k++) {
    const size_t p = levels[k];
    t0 = now();
    DNum ax, err, corr, next;
    if ((r = dnum_mul(ax, D, R, p)) || (r = dnum_sub(err, ax, one, p)) || (r = dnum_mul(corr, err, R, p)) ||
        (r = dnum_sub(next, R, corr, p)))
      return r;
    R = next;
    if (stats) fprintf(stderr, "      newton level p=%zu on the device: %.3f s\n", p, secs(t0));
  }
  DNum T = R;
  if (num) {
    t0 = now();
    if ((r = dnum_mul(T, N, R, pdiv))) return r;
    if (stats) fprintf(stderr, "      quotient on the device: %.3f s\n", secs(t0));
  }
  out->coef = nullptr;
  out->len = T.len;
  out->exp = T.exp;
  out->sign = T.sign;
  if (T.len) {
    out->coef = (uint32_t *)malloc(T.len * 4);
    if (!out->coef) return fail(BC_ERR_NOMEM);
    std::vector<SpanJob> jobs{{0, (char *)out->coef, T.len * 4}};
    if ((r = stage_d2h((const char *)T.p, jobs, T.len * 4))) {
      free(out->coef);
      out->coef = nullptr;
      return r;
    }
    CK(cudaStreamSynchronize(g.stream));
  }
  return BC_OK;
}

// A wait that runs out, on purpose and without a fault: one windowed sum of
// two tiles whose tile counter starts at 1, so tile 0 is never taken and
// tile 1's lookback has nothing to wait for.  Its bounded spin gives up,
// flags the sum and the kernel finishes; the host sees the flag.
int selftest_wait_locked(double *secs) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  const unsigned long long n = 2ull * ADD_TILE;
  DevBuf buf;
  const size_t o_r = align256(n * 4), o_sc = o_r + align256(n * 4), o_st = o_sc + 256;
  int r;
  if ((r = buf.alloc(o_st + 256))) return r;
  char *bp = (char *)buf.p;
  CK(cudaMemsetAsync(bp, 0, o_st + 256, g.stream));
  const unsigned one = 1;
  CK(cudaMemcpyAsync(bp + o_sc, &one, 4, cudaMemcpyHostToDevice, g.stream));  // the counter
  AddSubParams ap;
  ap.a = WinOp{(const uint32_t *)bp, 0, (long long)n};
  ap.b = WinOp{(const uint32_t *)bp, 0, 0};
  ap.r = (uint32_t *)(bp + o_r);
  ap.n = n;
  ap.sub = 0;
  ap.tiles = 2;
  ap.counter = (unsigned int *)(bp + o_sc);
  ap.cout = (unsigned int *)(bp + o_sc + 4);
  ap.flags = (unsigned int *)(bp + o_sc + 8);
  ap.status = (uint32_t *)(bp + o_st);
  CK(cudaEventRecord(g.ev0, g.stream));
  k_addsub_win<<<1, ADD_NT, 0, g.stream>>>(ap);
  CK(cudaGetLastError());
  CK(cudaEventRecord(g.ev1, g.stream));
  unsigned flags = 0;
  CK(cudaMemcpyAsync(&flags, ap.flags, 4, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, g.ev0, g.ev1));
  if (secs) *secs = ms * 1e-3;
  return (flags & 1u) ? BC_ERR_TIMEOUT : BC_OK;
}

int e_series_locked(uint32_t a, uint32_t b, uint32_t **hP, size_t *PL, uint32_t **hQ, size_t *QL,
                    bc_batch_stats *st) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (b <= a || b > 0xfffffff0u) return fail(BC_ERR_INVALID);
  const auto t_start = std::chrono::steady_clock::now();
  // leaves as wide as a warp holds: T terms give at most T*bits(b)/32 + 1
  // limbs per value, which must stay within WLEAF_CAP
  int bits = 0;
  while (bits < 32 && (b >> bits)) bits++;
  const uint32_t T = (uint32_t)std::min<long long>(1024, (long long)(WLEAF_CAP - 2) * 32 / bits);
  const uint32_t nleaf = (b - a + T - 1) / T;
  DevBuf level, lens;
  int r;
  if ((r = level.alloc((size_t)nleaf * 2 * WLEAF_STRIDE * 4)) || (r = lens.alloc((size_t)nleaf * 2 * 4 + 256)))
    return r;
  unsigned *lflags = (unsigned *)((char *)lens.p + (size_t)nleaf * 2 * 4);
  CK(cudaMemsetAsync(lflags, 0, 4, g.stream));
  k_bsr_leaves_wide<<<(nleaf + WLEAF_WARPS - 1) / WLEAF_WARPS, 32 * WLEAF_WARPS, 0, g.stream>>>(
      a, b, T, nleaf, (uint32_t *)level.p, (uint32_t *)lens.p, lflags);
  CK(cudaGetLastError());
  std::vector<uint32_t> l0(2 * (size_t)nleaf);
  unsigned leaf_overflow = 0;
  CK(cudaMemcpyAsync(l0.data(), lens.p, l0.size() * 4, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaMemcpyAsync(&leaf_overflow, lflags, 4, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  if (leaf_overflow) return fail(BC_ERR_TOO_LARGE);
  const bool stats = getenv("BC_STATS") != nullptr;
  double t_mul = 0, t_add = 0;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto secs = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  const double t_leaves = secs(t_start);
  std::vector<DevNum> P(nleaf), Q(nleaf);
  for (uint32_t j = 0; j < nleaf; j++) {
    P[j] = {(uint32_t *)level.p + (size_t)(2 * j) * WLEAF_STRIDE, l0[2 * j]};
    Q[j] = {(uint32_t *)level.p + (size_t)(2 * j + 1) * WLEAF_STRIDE, l0[2 * j + 1]};
  }
  while (P.size() > 1) {
    const size_t c = P.size(), np = c / 2;
    const bool odd = c & 1;
    // layout of the next level: per pair t = P_l*Q_r, Q' = Q_l*Q_r, P' = t + P_r
    std::vector<size_t> offT(np), offQ(np), offP(np), nT(np), nQ(np), nP(np);
    size_t total = 0;
    for (size_t i = 0; i < np; i++) {
      nT[i] = P[2 * i].len + Q[2 * i + 1].len;
      nQ[i] = Q[2 * i].len + Q[2 * i + 1].len;
      nP[i] = std::max(nT[i], P[2 * i + 1].len) + 1;
      offT[i] = total; total += (nT[i] + 63) & ~size_t(63);
      offQ[i] = total; total += (nQ[i] + 63) & ~size_t(63);
      offP[i] = total; total += (nP[i] + 63) & ~size_t(63);
    }
    size_t offOddP = total, offOddQ = total;
    if (odd) {
      offOddP = total; total += (P[c - 1].len + 63) & ~size_t(63);
      offOddQ = total; total += (Q[c - 1].len + 63) & ~size_t(63);
    }
    DevBuf next;
    if ((r = next.alloc(total * 4))) return r;
    uint32_t *nb = (uint32_t *)next.p;
    // products
    std::vector<bc_mul_desc> md(2 * np);
    for (size_t i = 0; i < np; i++) {
      md[2 * i] = {nb + offT[i], nT[i], P[2 * i].p, P[2 * i].len, Q[2 * i + 1].p, Q[2 * i + 1].len};
      md[2 * i + 1] = {nb + offQ[i], nQ[i], Q[2 * i].p, Q[2 * i].len, Q[2 * i + 1].p, Q[2 * i + 1].len};
    }
    auto tl0 = now();
    if ((r = mul_batch_locked(md.data(), md.size(), st, nullptr, BC_BATCH_DEVICE_OPERANDS))) return r;
    const double dm = secs(tl0);
    t_mul += dm;
    tl0 = now();
    // significant lengths of the products, then the additions
    std::vector<TrimDesc> td(2 * np);
    for (size_t i = 0; i < 2 * np; i++) td[i] = {md[i].C, md[i].CL};
    std::vector<AddDesc> ad(np);
    unsigned long long tiles = 0;  // bound from the untrimmed lengths; sizes the status words
    for (size_t i = 0; i < np; i++) {
      const unsigned long long n = std::max<unsigned long long>(nT[i], P[2 * i + 1].len);
      ad[i] = {nb + offT[i], P[2 * i + 1].p, nb + offP[i], nT[i], P[2 * i + 1].len, n, 0};
      tiles += n / ADD_TILE + 1;
    }
    // scratch: trim descs, product lengths, add descs, status, counter+flags, add lengths
    const size_t o_td = 0, o_tl = align256(o_td + td.size() * sizeof(TrimDesc));
    const size_t o_ad = align256(o_tl + 2 * np * 8), o_st = align256(o_ad + np * sizeof(AddDesc));
    const size_t o_ctr = align256(o_st + tiles * 4), o_al = o_ctr + 256, o_end = align256(o_al + np * 8);
    DevBuf meta;
    if ((r = meta.alloc(o_end))) return r;
    char *mb = (char *)meta.p;
    CK(cudaMemcpyAsync(mb + o_td, td.data(), td.size() * sizeof(TrimDesc), cudaMemcpyHostToDevice, g.stream));
    k_trim<<<(unsigned)((2 * np + 255) / 256), 256, 0, g.stream>>>((const TrimDesc *)(mb + o_td), (uint32_t)(2 * np),
                                                                 (unsigned long long *)(mb + o_tl));
    CK(cudaGetLastError());
    std::vector<unsigned long long> tl(2 * np);
    CK(cudaMemcpyAsync(tl.data(), mb + o_tl, tl.size() * 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    tiles = 0;
    for (size_t i = 0; i < np; i++) {
      ad[i].lx = tl[2 * i];
      ad[i].n = std::max<unsigned long long>(ad[i].lx, ad[i].ly);
      ad[i].tile0 = tiles;
      tiles += ad[i].n / ADD_TILE + 1;
    }
    CK(cudaMemcpyAsync(mb + o_ad, ad.data(), ad.size() * sizeof(AddDesc), cudaMemcpyHostToDevice, g.stream));
    CK(cudaMemsetAsync(mb + o_st, 0, o_al - o_st, g.stream));
    AddParams ap;
    ap.items = (const AddDesc *)(mb + o_ad);
    ap.nitems = (int)np;
    ap.tiles = tiles;
    ap.counter = (unsigned int *)(mb + o_ctr);
    ap.flags = (unsigned int *)(mb + o_ctr + 128);
    ap.status = (uint32_t *)(mb + o_st);
    ap.len = (unsigned long long *)(mb + o_al);
    const unsigned grid = (unsigned)std::min<unsigned long long>(tiles, (unsigned long long)g.sm_count * 4);
    k_add<<<grid, ADD_NT, 0, g.stream>>>(ap);
    CK(cudaGetLastError());
    std::vector<unsigned long long> al(np);
    unsigned int aflags = 0;
    CK(cudaMemcpyAsync(al.data(), ap.len, np * 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&aflags, ap.flags, 4, cudaMemcpyDeviceToHost, g.stream));
    if (odd) {
      CK(cudaMemcpyAsync(nb + offOddP, P[c - 1].p, P[c - 1].len * 4, cudaMemcpyDeviceToDevice, g.stream));
      CK(cudaMemcpyAsync(nb + offOddQ, Q[c - 1].p, Q[c - 1].len * 4, cudaMemcpyDeviceToDevice, g.stream));
    }
    CK(cudaStreamSynchronize(g.stream));
    if (aflags) return fail(BC_ERR_TIMEOUT);
    const double da = secs(tl0);
    t_add += da;
    if (stats && (dm + da > 0.05 || np < 4))
      fprintf(stderr, "      series level: %zu nodes, products %.3f s, lengths and sums %.3f s\n", np, dm, da);
    std::vector<DevNum> P2(np + odd), Q2(np + odd);
    for (size_t i = 0; i < np; i++) {
      P2[i] = {nb + offP[i], (size_t)al[i]};
      Q2[i] = {nb + offQ[i], (size_t)tl[2 * i + 1]};
    }
    if (odd) {
      P2[np] = {nb + offOddP, P[c - 1].len};
      Q2[np] = {nb + offOddQ, Q[c - 1].len};
    }
    P.swap(P2);
    Q.swap(Q2);
    std::swap(level.p, next.p);  // the old level is freed with `next`
  }
  // the root's P and Q into malloc'd host arrays, through the pinned ring
  const auto t_out = now();
  *hP = (uint32_t *)malloc(std::max<size_t>(P[0].len, 1) * 4);
  *hQ = (uint32_t *)malloc(std::max<size_t>(Q[0].len, 1) * 4);
  if (!*hP || !*hQ) {
    free(*hP);
    free(*hQ);
    *hP = *hQ = nullptr;
    return fail(BC_ERR_NOMEM);
  }
  std::vector<SpanJob> jp{{0, (char *)*hP, P[0].len * 4}}, jq{{0, (char *)*hQ, Q[0].len * 4}};
  if ((r = stage_d2h((const char *)P[0].p, jp, P[0].len * 4)) ||
      (r = stage_d2h((const char *)Q[0].p, jq, Q[0].len * 4))) {
    free(*hP);
    free(*hQ);
    *hP = *hQ = nullptr;
    return r;
  }
  *PL = P[0].len;
  *QL = Q[0].len;
  if (stats)
    fprintf(stderr, "      series: %u leaves %.3f s, products %.3f s, lengths and sums %.3f s, P and Q out %.3f s\n",
            nleaf, t_leaves, t_mul, t_add, secs(t_out));
  return BC_OK;
}

// ------------------------------------------------------------------ small exact products
// Products of at most SCHOOL_MAX limbs per operand, from and to host memory:
// descriptors and operands cross in one staged span, k_school computes all of
// them (one warp per product), the results come back in one span.
int mul_small_locked(const bc_mul_desc *items, size_t n) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (n && !items) return fail(BC_ERR_INVALID);
  std::vector<size_t> live;  // items with both operands nonempty
  live.reserve(n);
  for (size_t i = 0; i < n; i++) {
    const bc_mul_desc &d = items[i];
    if (d.CL > (size_t)SCHOOL_CMAX || d.AL > (size_t)SCHOOL_MAX || d.BL > (size_t)SCHOOL_MAX)
      return fail(BC_ERR_TOO_LARGE);
    if ((d.CL && !d.C) || (d.AL && !d.A) || (d.BL && !d.B)) return fail(BC_ERR_INVALID);
    if (is_device_ptr(d.C) || (d.AL && is_device_ptr(d.A)) || (d.BL && is_device_ptr(d.B)))
      return fail(BC_ERR_INVALID);
    if (d.CL && (!d.AL || !d.BL)) memset(d.C, 0, d.CL * 4);  // a zero operand
    else if (d.CL) live.push_back(i);
  }
  if (live.empty()) return BC_OK;
  // input span: descriptors, then every live item's A and B; output span: C
  const size_t m = live.size();
  std::vector<SchoolDesc> desc(m);
  const size_t desc_words = align256(m * sizeof(SchoolDesc)) / 4;
  size_t in_words = desc_words, out_words = 0;
  std::vector<SpanJob> in_jobs, out_jobs;
  in_jobs.reserve(2 * m + 1);
  out_jobs.reserve(m);
  in_jobs.push_back({0, (char *)desc.data(), m * sizeof(SchoolDesc)});
  for (size_t k = 0; k < m; k++) {
    const bc_mul_desc &d = items[live[k]];
    SchoolDesc &q = desc[k];
    q.AL = (uint32_t)d.AL;
    q.BL = (uint32_t)d.BL;
    q.CL = (uint32_t)d.CL;
    q.pad = 0;
    q.a = in_words - desc_words;
    in_jobs.push_back({in_words * 4, (char *)d.A, d.AL * 4});
    in_words += d.AL;
    q.b = in_words - desc_words;
    in_jobs.push_back({in_words * 4, (char *)d.B, d.BL * 4});
    in_words += d.BL;
    q.c = out_words;
    out_jobs.push_back({out_words * 4, (char *)d.C, d.CL * 4});
    out_words += d.CL;
  }
  DevBuf din, dout;
  int r;
  if ((r = din.alloc(in_words * 4)) || (r = dout.alloc(out_words * 4))) return r;
  if ((r = stage_h2d((char *)din.p, in_jobs, in_words * 4))) return r;
  const unsigned blocks =
      (unsigned)std::min<size_t>((m + SCHOOL_WARPS - 1) / SCHOOL_WARPS, (size_t)g.sm_count * 16);
  k_school<<<blocks, 32 * SCHOOL_WARPS, 0, g.stream>>>((const SchoolDesc *)din.p, (unsigned)m,
                                                        (const uint32_t *)din.p + desc_words, (uint32_t *)dout.p);
  CK(cudaGetLastError());
  if ((r = stage_d2h((const char *)dout.p, out_jobs, out_words * 4))) return r;
  CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

// ------------------------------------------------------------------ decimal text
// pwrite of [buf, buf + len) at file offset off, in pieces of at least 4 MiB
// on up to copy_threads() threads (the copy into the page cache is most of
// the time of a large write).
int par_pwrite(int fd, const char *buf, size_t len, long long off) {
  const unsigned nt = (unsigned)std::min<size_t>(copy_threads(), len / (size_t(4) << 20) + 1);
  const size_t piece = (len + nt - 1) / nt;
  std::atomic<int> bad{0};
  auto worker = [&](unsigned k) {
    size_t o = (size_t)k * piece;
    const size_t end = std::min(len, o + piece);
    while (o < end) {
      const ssize_t w = pwrite(fd, buf + o, end - o, (off_t)(off + (long long)o));
      if (w <= 0) {
        bad = 1;
        return;
      }
      o += (size_t)w;
    }
  };
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nt; k++) th.emplace_back(worker, k);
  worker(0);
  for (std::thread &t : th) t.join();
  return bad ? fail(BC_ERR_IO) : BC_OK;
}

// Nine decimal characters per limb for limbs[top], limbs[top-1], ...,
// limbs[top-n+1], cut at maxbytes, written at file offset off.  The text is
// rendered in device memory (k_decimal_text) and leaves through the pinned
// ring, each chunk written by several threads while the next one crosses.
int decimal_write_locked(const uint32_t *limbs, size_t top, size_t n, size_t maxbytes, int fd, long long off) {
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (fd < 0 || off < 0 || (n && (!limbs || top + 1 < n)) || n > (SIZE_MAX / 9)) return fail(BC_ERR_INVALID);
  const size_t bytes = std::min(maxbytes, 9 * n);
  if (!bytes) return BC_OK;
  const size_t nl = (bytes + 8) / 9;  // limbs whose text is written, whole or in part
  DevBuf din, dtext;
  int r;
  const uint32_t *dl = limbs;
  size_t dtop = top;
  if (!is_device_ptr(limbs)) {  // the nl limbs the text needs, limbs[top-nl+1 .. top]
    if ((r = din.alloc(nl * 4))) return r;
    std::vector<SpanJob> jobs{{0, (char *)(limbs + (top + 1 - nl)), nl * 4}};
    if ((r = stage_h2d((char *)din.p, jobs, nl * 4))) return r;
    dl = (const uint32_t *)din.p;
    dtop = nl - 1;
  }
  if ((r = dtext.alloc((9 * nl + 15) & ~size_t(15)))) return r;
  const unsigned long long blocks = (nl + TEXT_LIMBS - 1) / TEXT_LIMBS;
  if (blocks > 0x7fffffffULL) return fail(BC_ERR_TOO_LARGE);
  k_decimal_text<<<(unsigned)blocks, TEXT_THREADS, 0, g.stream>>>(dl, dtop, nl, (char *)dtext.p);
  CK(cudaGetLastError());
  if ((r = ring_ready())) return r;
  for (int h = 0; h < 2; h++)
    if (g_ring.pending[h]) { CK(cudaEventSynchronize(g_ring.ev[h])); g_ring.pending[h] = false; }
  const char *src = (const char *)dtext.p;
  const size_t nch = (bytes + kRingChunk - 1) / kRingChunk;
  auto issue = [&](size_t c) -> int {
    const int h = (int)(c & 1);
    const size_t w0 = c * kRingChunk, len = std::min(kRingChunk, bytes - w0);
    CK(cudaMemcpyAsync(g_ring.half[h], src + w0, len, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaEventRecord(g_ring.ev[h], g.stream));
    return BC_OK;
  };
  if ((r = issue(0))) return r;
  for (size_t c = 0; c < nch; c++) {
    if (c + 1 < nch && (r = issue(c + 1))) return r;
    const int h = (int)(c & 1);
    CK(cudaEventSynchronize(g_ring.ev[h]));
    const size_t w0 = c * kRingChunk, len = std::min(kRingChunk, bytes - w0);
    if ((r = par_pwrite(fd, g_ring.half[h], len, off + (long long)w0))) {
      CK(cudaStreamSynchronize(g.stream));  // the next chunk's copy is still in flight
      return r;
    }
  }
  return BC_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int bc_gpu_init(const bc_gpu_config *cfg) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (g.init) return BC_OK;
  bc_gpu_config c{};
  if (cfg) c = *cfg;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(BC_ERR_NO_DEVICE);
  }
  if (c.device < 0 || c.device >= ndev) return fail(BC_ERR_INVALID);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, c.device));
  if (prop.major != 10) return fail(BC_ERR_NO_DEVICE);
  CK(cudaSetDevice(c.device));
  g.device = c.device;
  g.sm_count = prop.multiProcessorCount;
  CK(cudaStreamCreateWithFlags(&g.own_stream, cudaStreamNonBlocking));
  g.stream = g.own_stream;
  {
    // the default pool backs the drivers' scratch (DevBuf): keep what they
    // free for the next level instead of returning it at every synchronisation
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, c.device));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  CK(cudaEventCreate(&g.ev0));
  CK(cudaEventCreate(&g.ev1));
  size_t fre = 0, tot = 0;
  CK(cudaMemGetInfo(&fre, &tot));
  g.arena_limit = c.arena_bytes ? c.arena_bytes : (size_t)(fre * 0.9);
  g.max_err = c.max_round_err > 0 ? c.max_round_err : 0.25;
  if (getenv("BC_PROFILE") && !g_prof_on) {
    g_prof_on = true;
    atexit(print_profile);
  }
  g.verbose = c.verbose || getenv("BC_VERBOSE") != nullptr;
  {
    const char *rw = getenv("BC_ROWS_WARP");
    g.rows_warp = !(rw && rw[0] == '0');
    const char *p16 = getenv("BC_PASS16");
    g.pass16 = !(p16 && p16[0] == '0');
    const char *fu = getenv("BC_FUSED");
    g.fused = fu && fu[0] == '1';
    const char *sb = getenv("BC_SHARE_B");
    g.share_b = !(sb && sb[0] == '0');
    const char *gr = getenv("BC_GRAPH");
    g.graph_all = gr && gr[0] == '1';
    const char *pd = getenv("BC_PDL");
    g.pdl = !(pd && pd[0] == '0');
  }
  load_width_file(c.tune_path);
  {
    // tuned decompositions: $BC_SHAPE_FILE, else shapes.txt beside the width table
    const char *sp = getenv("BC_SHAPE_FILE");
    std::string path = sp ? sp : "";
    const char *tp = c.tune_path ? c.tune_path : getenv("BC_TUNE_FILE");
    if (path.empty() && tp && *tp) {
      path = tp;
      const size_t slash = path.rfind('/');
      path = (slash == std::string::npos ? std::string() : path.substr(0, slash + 1)) + "shapes.txt";
    }
    if (!path.empty()) {
      FILE *f = fopen(path.c_str(), "r");
      if (f) {
        fclose(f);
        bc_gpu_load_shape_table(path.c_str());
      }
    }
  }
  g.init = true;
  return BC_OK;
}

int bc_gpu_shutdown(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g.init) return BC_OK;
  cudaStreamSynchronize(g.stream);
  for (auto &t : g.tables) cudaFree(t.second.dev);
  g.tables.clear();
  if (g.arena) cudaFree(g.arena);
  g.arena = nullptr;
  g.arena_cap = 0;
  for (auto e : g.kev_pool) cudaEventDestroy(e);
  g.kev_pool.clear();
  if (g.pin_small) cudaFreeHost(g.pin_small);
  g.pin_small = nullptr;
  g.pin_small_cap = 0;
  if (g.ev0) cudaEventDestroy(g.ev0);
  if (g.ev1) cudaEventDestroy(g.ev1);
  if (g.own_stream) cudaStreamDestroy(g.own_stream);
  if (g.copy_stream) cudaStreamDestroy(g.copy_stream);
  if (g.gexec) cudaGraphExecDestroy(g.gexec);
  if (g.cap_stream) cudaStreamDestroy(g.cap_stream);
  for (auto &cs : g.class_stream)
    if (cs) cudaStreamDestroy(cs);
  for (auto &e : g.class_ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : g.copy_ev)
    if (e) cudaEventDestroy(e);
  g_occ.clear();
  g = Ctx();
  return BC_OK;
}

int bc_gpu_mul(uint32_t *C, size_t CL, const uint32_t *A, size_t AL, const uint32_t *B, size_t BL,
               bc_mul_stats *stats) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  bc_mul_desc d{C, CL, A, AL, B, BL};
  bc_batch_stats st{};
  Plan pl;
  int r = mul_batch_locked(&d, 1, &st, &pl);
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->fft_points = pl.shape.M;
    stats->width = pl.b;
    stats->retries = st.retries;
    stats->max_round_err = st.max_round_err;
    stats->device_ms = st.device_ms;
    stats->total_ms = st.total_ms;
  }
  return r;
}

int bc_gpu_mul_batch(const bc_mul_desc *items, size_t n, bc_batch_stats *stats) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  bc_batch_stats st{};
  int r = mul_batch_locked(items, n, &st);
  if (stats) *stats = st;
  return r;
}

int bc_gpu_mul_batch_flags(const bc_mul_desc *items, size_t n, unsigned flags, bc_batch_stats *stats) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  bc_batch_stats st{};
  int r = mul_batch_locked(items, n, &st, nullptr, flags);
  if (stats) *stats = st;
  return r;
}

int bc_gpu_e_series(uint32_t a, uint32_t b, uint32_t **P, size_t *PL, uint32_t **Q, size_t *QL) {
  if (!P || !PL || !Q || !QL) return BC_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  bc_batch_stats st{};
  *P = *Q = nullptr;
  return e_series_locked(a, b, P, PL, Q, QL, &st);
}

int bc_gpu_radix_tree(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nnodes,
                      const uint32_t *const *table, const size_t *table_len, int ntable, double alpha,
                      uint32_t *out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return radix_tree_locked(y, ylen, nodes, nnodes, table, table_len, ntable, alpha, out);
}

int bc_gpu_radix_tree_pow(const uint32_t *y, size_t ylen, const bc_radix_node *nodes, size_t nnodes,
                          const uint32_t *t0, size_t t0len, const bc_radix_pow_step *steps, int ntable, double alpha,
                          uint32_t *out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return radix_tree_pow_locked(y, ylen, nodes, nnodes, t0, t0len, steps, ntable, alpha, out);
}

int bc_gpu_mul_small_batch(const bc_mul_desc *items, size_t n) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return mul_small_locked(items, n);
}

int bc_gpu_decimal_write(const uint32_t *limbs, size_t top, size_t n, size_t maxbytes, int fd, long long offset) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return decimal_write_locked(limbs, top, n, maxbytes, fd, offset);
}

int bc_gpu_device_alloc(size_t bytes, void **p) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!p) return fail(BC_ERR_INVALID);
  *p = nullptr;
  if (cudaMalloc(p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(BC_ERR_NOMEM);
  }
  return BC_OK;
}

int bc_gpu_device_free(void *p) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!p) return BC_OK;
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  CK(cudaStreamSynchronize(g.stream));
  CK(cudaFree(p));
  return BC_OK;
}

int bc_gpu_copy(void *dst, const void *src, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  if (!bytes) return BC_OK;
  if (!dst || !src) return fail(BC_ERR_INVALID);
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

int bc_gpu_selftest_wait(double *seconds) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return selftest_wait_locked(seconds);
}

int bc_gpu_newton(const bc_bignum *den, const bc_bignum *r0, const size_t *levels, int nlevels, const bc_bignum *num,
                  size_t pdiv, bc_bignum_out *out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return newton_locked(den, r0, levels, nlevels, num, pdiv, out);
}

int bc_gpu_radix_leaves(const bc_radix_leaf *leaves, size_t count, double alpha) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return radix_leaves_locked(leaves, count, alpha);
}

int bc_gpu_set_stream(void *stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  g.stream = stream ? (cudaStream_t)stream : g.own_stream;
  return BC_OK;
}

int bc_gpu_plan(size_t AL, size_t BL, size_t CL, int square, bc_plan_info *out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!out) return BC_ERR_INVALID;
  memset(out, 0, sizeof *out);
  if (!CL || !AL || !BL) return BC_OK;
  Plan pl;
  if (!make_plan(AL, BL, CL, square != 0, 24, pl)) return BC_ERR_TOO_LARGE;
  out->fft_points = pl.shape.M;
  out->width = pl.b;
  out->levels = pl.shape.levels;
  out->L1 = pl.shape.L1;
  out->L2 = pl.shape.L2;
  out->Lr = pl.shape.Lr;
  out->digits_a = pl.ndA;
  out->digits_b = pl.square ? pl.ndA : pl.ndB;
  out->out_words = pl.nwords;
  out->work_bytes = work_bytes(pl);
  return BC_OK;
}

int bc_gpu_width_limit(size_t fft_points) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return width_limit(fft_points);
}

int bc_gpu_set_width_limit(size_t fft_points, int width) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (width == 0) { g.width_override.erase(fft_points); return BC_OK; }
  if (width < 8 || width > 24) return BC_ERR_INVALID;
  g.width_override[fft_points] = width;
  return BC_OK;
}

int bc_gpu_force_width(int width) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (width != 0 && (width < 8 || width > 24)) return BC_ERR_INVALID;
  g.forced_width = width;
  return BC_OK;
}

int bc_gpu_load_width_table(const char *path) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!path) return BC_ERR_INVALID;
  FILE *f = fopen(path, "r");
  if (!f) return BC_ERR_INVALID;
  fclose(f);
  g.width_file.clear();
  load_width_file(path);
  return BC_OK;
}

int bc_gpu_check_shapes(void) {
  for (size_t M : lengths()) {
    Shape s;
    if (!shape_for(M, s)) return (int)std::min<size_t>(M, 0x7fffffff);
    for (int sq = 0; sq < 2; sq++)
      if (!shape_launch_ok(s, sq != 0)) return (int)std::min<size_t>(M, 0x7fffffff);
  }
  return BC_OK;
}

int bc_gpu_lengths(size_t *out, int cap) {
  const std::vector<size_t> &v = lengths();
  for (int i = 0; i < cap && i < (int)v.size(); i++) out[i] = v[i];
  return (int)v.size();
}

int bc_gpu_shape_candidates(size_t fft_points, int *out, int cap) {
  int n = 0;
  for (const Shape &s : shape_candidates(fft_points)) {
    if (!shape_launch_ok(s, false) || !shape_launch_ok(s, true)) continue;
    if (out && n < cap) {
      out[4 * n] = s.levels;
      out[4 * n + 1] = s.L1;
      out[4 * n + 2] = s.L2;
      out[4 * n + 3] = s.Lr;
    }
    n++;
  }
  return n;
}

int bc_gpu_set_shape(size_t fft_points, int L1, int L2, int Lr) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (L1 == 0 && L2 == 0 && Lr == 0) {
    g.shape_table.erase(fft_points);
    return BC_OK;
  }
  for (const Shape &s : shape_candidates(fft_points))
    if (s.L1 == L1 && s.L2 == L2 && s.Lr == Lr && shape_launch_ok(s, false) && shape_launch_ok(s, true)) {
      g.shape_table[fft_points] = s;
      return BC_OK;
    }
  return BC_ERR_INVALID;
}

int bc_gpu_load_shape_table(const char *path) {
  if (!path) return BC_ERR_INVALID;
  FILE *f = fopen(path, "r");
  if (!f) return BC_ERR_INVALID;
  char line[256];
  int bad = 0;
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    unsigned long long M = 0;
    int L1 = 0, L2 = 0, Lr = 0;
    if (sscanf(line, "%llu %d %d %d", &M, &L1, &L2, &Lr) == 4 && bc_gpu_set_shape((size_t)M, L1, L2, Lr) != BC_OK)
      bad++;
  }
  fclose(f);
  return bad ? BC_ERR_INVALID : BC_OK;
}

int bc_gpu_force_plan(size_t fft_points, int width) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (width != 0 && (width < 8 || width > 24)) return BC_ERR_INVALID;
  Shape s;
  if (fft_points && !shape_for(fft_points, s)) return BC_ERR_INVALID;
  g.forced_M = fft_points;
  g.forced_width = width;
  return BC_OK;
}

int bc_gpu_sync(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g.init) return fail(BC_ERR_NOT_INIT);
  CK(cudaStreamSynchronize(g.stream));
  return BC_OK;
}

int bc_gpu_last_error(void) { return g.last_error; }
int bc_gpu_last_cuda_error(void) { return g.last_cuda; }

const char *bc_gpu_strerror(int code) {
  switch (code) {
    case BC_OK: return "ok";
    case BC_ERR_INVALID: return "invalid argument";
    case BC_ERR_NOMEM: return "out of device memory";
    case BC_ERR_CUDA: return "CUDA runtime error";
    case BC_ERR_TIMEOUT: return "carry lookback timed out";
    case BC_ERR_PRECISION: return "rounding error above the limit at every width";
    case BC_ERR_NOT_INIT: return "library not initialised (bc_gpu_init)";
    case BC_ERR_TOO_LARGE: return "product too large for the supported transform lengths";
    case BC_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case BC_ERR_CARRY: return "carry out of the top word of an exact product";
    case BC_ERR_IO: return "writing the output file failed";
  }
  return "unknown error";
}

int bc_gpu_time_kernels(int on) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  g.time_kernels = on != 0;
  g.ktimes.clear();
  return BC_OK;
}

int bc_gpu_kernel_times(const char **names, double *ms, int cap) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int n = 0;
  for (auto &kt : g.ktimes) {
    if (n >= cap) break;
    if (names) names[n] = kt.first;
    if (ms) ms[n] = kt.second;
    n++;
  }
  return (int)g.ktimes.size();
}

}  // extern "C"

// ====================================================================== allocation-free entry point
// bc_gpu_mul_noalloc: the same exact product for callers that cannot
// allocate device memory themselves or let a library do it — a custom
// allocator or memory pool that owns the whole device, or an embedding host
// whose policy forbids cudaMalloc after start-up.  Its scratch (transform
// buffers, run records, lookback status, descriptor, error slots, twiddle
// tables) is one file-scope __device__ array; the caller passes device
// inputs and outputs.  Each call waits for its stream and reads the outcome
// back, so it cannot be called while that stream is being captured.
namespace {
constexpr size_t kNoAllocBytes = size_t(8) << 20;          // 8 MiB of scratch per GPU
constexpr size_t kNoAllocMaxPoints = size_t(1) << 17;       // transforms up to 2^17 points
constexpr size_t kNoAllocMaxLimbs = 131072;                 // AL + BL limit (fits 2^17 points at b = 16)
constexpr size_t kNoAllocTableBytes = size_t(256) << 10;
constexpr size_t kNoAllocDescOff = kNoAllocTableBytes;      // ItemDesc
constexpr size_t kNoAllocSlotsOff = kNoAllocDescOff + 256;  // err (8 B), flags (4 B), counter (4 B)
constexpr size_t kNoAllocStatusOff = kNoAllocSlotsOff + 256;
constexpr size_t kNoAllocStatusBytes = 4096;                // lookback tiles: (2M/8)/256 * 4 B
constexpr size_t kNoAllocWorkOff = kNoAllocStatusOff + kNoAllocStatusBytes;
static_assert(kNoAllocWorkOff + 2 * 16 * kNoAllocMaxPoints + kNoAllocMaxPoints / 4 * sizeof(RunRec) <= kNoAllocBytes,
              "no-alloc scratch too small");
static_assert(sizeof(ItemDesc) <= 256, "descriptor slot");
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocDevice {
  unsigned char *base;  // device address of the scratch array on this device
  size_t table_M;       // transform length and split whose tables are in the scratch
  int table_L1, table_L2, table_Lr;
  int ready;
};
NoAllocDevice g_noalloc[kNoAllocMaxDevices];
double2 g_noalloc_tables[kNoAllocTableBytes / sizeof(double2)];  // host staging for table uploads
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

extern "C" int bc_gpu_mul_noalloc(uint32_t *C, size_t CL, const uint32_t *A, size_t AL, const uint32_t *B,
                                  size_t BL, void *stream_ptr) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  if (CL == 0) return BC_OK;
  if (!C || (AL && !A) || (BL && !B)) return fail(BC_ERR_INVALID);
  if (overlaps(C, CL * 4, A, AL * 4) || overlaps(C, CL * 4, B, BL * 4)) return fail(BC_ERR_INVALID);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(BC_ERR_INVALID);
  NoAllocDevice &nd = g_noalloc[dev];
  if (!nd.ready) {
    // Set-up, once per device, with that device current: the array's name is
    // only a host-side stand-in, so fetch its device address.
    void *ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    nd.base = (unsigned char *)ptr;
    nd.table_M = 0;
    nd.ready = 1;
  }
  if (AL == 0 || BL == 0) {
    CK(cudaMemsetAsync(C, 0, CL * 4, stream));
    CK(cudaStreamSynchronize(stream));
    return BC_OK;
  }
  if (std::min(AL, CL) + std::min(BL, CL) > kNoAllocMaxLimbs) return fail(BC_ERR_TOO_LARGE);
  const bool square = A == B && AL == BL;
  int bcap = 24;
  for (int attempt = 0; attempt < 12; attempt++) {
    Plan pl;
    if (!make_plan(AL, BL, CL, square, bcap, pl, kNoAllocMaxPoints))
      return fail(attempt ? BC_ERR_PRECISION : BC_ERR_TOO_LARGE);
    const Shape &s = pl.shape;
    const TableLayout lay = table_layout(s);
    if (lay.total * sizeof(double2) > kNoAllocTableBytes || pl.ntiles * 4 > kNoAllocStatusBytes)
      return fail(BC_ERR_TOO_LARGE);
    if (nd.table_M != (size_t)s.M || nd.table_L1 != s.L1 || nd.table_L2 != s.L2 || nd.table_Lr != s.Lr) {
      CK(cudaStreamSynchronize(stream));  // the staging array and the old tables are no longer in use
      fill_tables(s, lay, g_noalloc_tables);
      CK(cudaMemcpyAsync(nd.base, g_noalloc_tables, lay.total * sizeof(double2), cudaMemcpyHostToDevice, stream));
      nd.table_M = s.M;
      nd.table_L1 = s.L1;
      nd.table_L2 = s.L2;
      nd.table_Lr = s.Lr;
    }
    unsigned char *w = nd.base + kNoAllocWorkOff;
    const size_t M = s.M;
    ItemDesc it{};
    it.A = A;
    it.B = square ? A : B;
    it.C = C;
    it.AL = pl.AL; it.BL = pl.BL; it.CL = CL;
    it.ndA = pl.ndA; it.ndB = square ? pl.ndA : pl.ndB;
    it.bufA = (double2 *)w;
    it.bufB = square ? nullptr : (double2 *)(w + 16 * M);
    it.rec = s.levels > 1 ? (RunRec *)(w + 32 * M) : nullptr;
    it.status = s.levels > 1 ? (uint32_t *)(nd.base + kNoAllocStatusOff) : nullptr;
    it.nwords = pl.nwords;
    it.nruns = pl.nruns;
    it.tile0 = 0;
    it.err = (unsigned long long *)(nd.base + kNoAllocSlotsOff);
    it.flags = (unsigned int *)(nd.base + kNoAllocSlotsOff + 8);
    it.b = pl.b;
    it.square = square ? 1 : 0;
    it.a16 = stage16_ok(it.A, pl);
    it.b16 = stage16_ok(it.B, pl);
    ItemDesc *ddesc = (ItemDesc *)(nd.base + kNoAllocDescOff);
    unsigned int *ctr = (unsigned int *)(nd.base + kNoAllocSlotsOff + 12);
    // every call reuses the array: clear what the kernels expect to start at zero
    CK(cudaMemcpyAsync(ddesc, &it, sizeof it, cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(nd.base + kNoAllocSlotsOff, 0, 256 + kNoAllocStatusBytes, stream));
    ClassParams p = class_params(s, tables_at(lay, (double2 *)nd.base));
    p.items = ddesc;
    p.nitems = 1;
    p.sq = square ? 1 : 0;
    p.counter = ctr;
    p.carry_tiles = pl.ntiles;
    p.nb = square ? 0 : 1;  // one B slot, its own (bowner null)
    size_t nl = 0;
    int r = launch_class(s, square, p, 1, pl.ntiles, it.bufA, it.bufB, stream, false, &nl);
    if (r) return r;
    unsigned long long errbits = 0;
    unsigned int flags = 0;
    CK(cudaMemcpyAsync(&errbits, it.err, 8, cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(&flags, it.flags, 4, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (flags & FLAG_TIMEOUT) return fail(BC_ERR_TIMEOUT);
    double e;
    memcpy(&e, &errbits, 8);
    if (e < g.max_err && !(flags & FLAG_TOPCARRY)) return BC_OK;
    bcap = pl.b - 1;  // narrower digits, as bc_gpu_mul retries
  }
  return fail(BC_ERR_PRECISION);
}
