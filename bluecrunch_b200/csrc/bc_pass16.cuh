// bc_pass16.cuh — outer column passes with 16 points per thread.
//
// Same arithmetic and data layout as k2_outer_fwd / k2_outer_inv
// (bc_pipe.cuh); the column transform is organised differently.  An L-point
// column (L = 16 R, R in {4, 8, 16}) is held by R threads with 16 points
// each, point t + R i in register i of thread t.  The transform is the
// four-step split L = 16 x R:
//   1. a 16-point DFT in registers over i (constant twiddles),
//   2. the twiddle e^{-+2 pi i t k2 / L},
//   3. ONE exchange through shared memory,
//   4. DFT-R over t for the 16/R values of k2 = t + R j a thread owns.
// Outputs land in the same register contract (frequency t + R i in register
// i), so the pass reads digits / tiles and writes results exactly as the
// 8-points-per-thread kernels do, with one exchange and two barriers per
// column transform instead of two exchanges and four barriers, and twice
// the independent work per thread between barriers.
#pragma once
#include "bc_pipe.cuh"
#include "bc_rows_warp.cuh"

namespace bc {

constexpr int P16 = 16;

// 16-point DFT in registers, natural order in and out: n = n1 + 4 n2,
// k = k2 + 4 k1; DFT-4 over n2, twiddle w16^(n1 k2), DFT-4 over n1.
template <bool INV>
__device__ __forceinline__ void dft16(double2 (&a)[P16]) {
#pragma unroll
  for (int n1 = 0; n1 < 4; n1++) {
    dft4<INV>(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);  // a[n1 + 4 k2] = y[n1][k2]
#pragma unroll
    for (int k2 = 1; k2 < 4; k2++) a[n1 + 4 * k2] = rot32<INV>(a[n1 + 4 * k2], 2 * n1 * k2);
  }
  double2 o[P16];
#pragma unroll
  for (int k2 = 0; k2 < 4; k2++) {
    double2 b0 = a[4 * k2], b1 = a[4 * k2 + 1], b2 = a[4 * k2 + 2], b3 = a[4 * k2 + 3];
    dft4<INV>(b0, b1, b2, b3);
    o[k2] = b0;
    o[k2 + 4] = b1;
    o[k2 + 8] = b2;
    o[k2 + 12] = b3;
  }
#pragma unroll
  for (int k = 0; k < P16; k++) a[k] = o[k];
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small16(double2 (&x)[R]) {
  static_assert(R == 4 || R == 8 || R == 16, "second-stage radix");
  if constexpr (R == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
  else if constexpr (R == 8) dft8<INV>(x);
  else dft16<INV>(x);
}

// Shared-memory twiddles of block16: tw[t*16 + k2] = e^{-2 pi i t k2 / L},
// t < L/16, k2 < 16, from the flat table flat[m] = e^{-2 pi i m/L}
// (m < 3L/4; above that e^{-2 pi i m/L} = -e^{-2 pi i (m - L/2)/L}).  All
// threads; the caller's next barrier publishes the table.
template <int L>
__device__ __forceinline__ void tw16_build(double2 *dst, const double2 *__restrict__ flat) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    const int m = (i >> 4) * (i & 15);
    const double2 w = __ldg(&flat[m < 3 * L / 4 ? m : m - L / 2]);
    dst[i] = m < 3 * L / 4 ? w : make_double2(-w.x, -w.y);
  }
}

// L-point transforms of W columns by R = L/16 threads per column.  On entry
// and exit v[i] = x[t + R i] of column s (natural order).  sm is the tile's
// shared memory (L x W, the swizzled layout of sidx); tw the table of
// tw16_build.  Ends past a barrier, so the CTA may reuse sm.
template <int L, int W, bool INV>
__device__ __forceinline__ void block16(double2 (&v)[P16], int t, int s, double2 *sm, const double2 *tw) {
  constexpr int R = L / P16, J = P16 / R;
  dft16<INV>(v);  // v[k2] = Y[t][k2]
#pragma unroll
  for (int k2 = 1; k2 < P16; k2++) v[k2] = ctw<INV>(v[k2], tw[t * P16 + k2]);
#pragma unroll
  for (int k2 = 0; k2 < P16; k2++) sm[sidx<L, W>(k2 * R + t, s)] = v[k2];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < J; j++) {
    const int k2 = t + R * j;
    double2 x[R];
#pragma unroll
    for (int tp = 0; tp < R; tp++) x[tp] = sm[sidx<L, W>(k2 * R + tp, s)];
    dft_small16<R, INV>(x);
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) v[j + J * k1] = x[k1];  // frequency k2 + 16 k1 = t + R (j + J k1)
  }
  __syncthreads();
}

// Tile geometry of the 16-point passes: same tiles as PassTile<L> (L rows x
// W columns, W = pass_tile_w(L)), R = L/16 threads per column.
template <int L> struct Pass16 {
  static constexpr int W = pass_tile_w(L);
  static constexpr int R = L / P16;
  static constexpr int NT = R * W;
  static_assert(L == 64 || L == 128 || L == 256, "16-point passes cover L1 = 64, 128, 256");
  // twelve warps per SM (at most 170 registers per thread)
  static constexpr int MINB = 384 / NT;
  // dynamic shared memory
  static constexpr size_t TWB = (size_t)L * 16;  // block16 twiddles
  static constexpr size_t SMEM_INV = 2 * (size_t)L * W * 16 + TWB + (size_t)L * 16 + 2 * 18 * 16 + 1024;
  static constexpr size_t SMEM_FWD = (size_t)L * W * 16 + (size_t)PackTile<L>::STAGE_WORDS * 4 + TWB +
                                     (size_t)L * 16 + 18 * 16 + 1024;
};

// Outer-pass twiddles e^{-2 pi i col (4 k1 - 1)/(4M)} of one thread, for
// k1 = t + R i (i = 0..15) and col = tile W + s, as two runs of 8 (a base
// and a step, then products).  With T(m) = e^{-2 pi i m/(4M)} (m signed) and
// T(col x) = T(tile W x) T(s x):
//   base of the first run   T(col (4t - 1))     = F_t       * T(s (4t - 1))
//   step                    T(col 4R)           = G         * T(s 4R)
//   base of the second run  T(col (4t + 32R - 1)) = base1 * H * T(s 32R)
// The tile factors F_t (t < 16), G = T(tile W 4R), H = T(tile W 32R) are
// computed once per unit by 18 threads (sincospi) into shared memory; the
// column factors depend only on the thread (s, t fixed by tid) and stay in
// registers.  No global twiddle loads remain on the unit's path.
constexpr int TILE_TW = 18;  // tile factors per unit

// T(m) = e^{-2 pi i m/(4M)}: t4m(m, 2M) (bc_pipe.cuh).

struct ColTw16 {
  double2 c0, cst, cb1;
};
template <int R>
__device__ __forceinline__ ColTw16 col_tw16(int s, int t, double twoM) {
  ColTw16 c;
  c.c0 = t4m((long long)s * (4 * t - 1), twoM);
  c.cst = t4m((long long)s * 4 * R, twoM);
  c.cb1 = t4m((long long)s * 32 * R, twoM);
  return c;
}

// The tile factors of `tile` into fac[0..17], spread over the CTA's warps
// (a few lanes of each).  The caller's next barrier publishes them.
template <int R, int W, int NT>
__device__ __forceinline__ void tile_tw16(double2 *fac, int tile, double twoM) {
  constexpr int NW = NT / 32, PER = (TILE_TW + NW - 1) / NW;
  const int lane = threadIdx.x & 31, j = (threadIdx.x >> 5) * PER + lane;
  if (lane < PER && j < TILE_TW) {
    const long long tw = (long long)tile * W;
    const long long x = j < 16 ? 4 * j - 1 : (j == 16 ? 4 * R : 32 * R);
    fac[j] = t4m(tw * x, twoM);
  }
}

struct OuterRun16 {
  double2 b0, b1, st;
};
__device__ __forceinline__ OuterRun16 outer_run16(const double2 *fac, const ColTw16 &c, int t) {
  OuterRun16 o;
  o.b0 = cmul(fac[t], c.c0);
  o.st = cmul(fac[16], c.cst);
  o.b1 = cmul(o.b0, cmul(fac[17], c.cb1));
  return o;
}

// ------------------------------------------------------------------ outer forward (pack)
// Units: (item, operand, column tile), as k2_outer_fwd.  One limb stage: the
// next unit's words are copied (cp.async) as soon as this unit's digits are
// cut, and land while this unit is transformed and stored.
template <int L>
__global__ void __launch_bounds__(Pass16<L>::NT, Pass16<L>::MINB) k3_outer_fwd(ClassParams p) {
  pdl_trigger();  // the first pass of a class: launched normally, lets the next one start early
  using T = Pass16<L>;
  using K = PackTile<L>;
  constexpr int W = T::W, R = T::R, NT = T::NT;
  static_assert(K::W == W, "pack tile geometry");
  extern __shared__ unsigned char smraw[];
  double2 *tile = align1024(smraw);
  uint32_t *stg = reinterpret_cast<uint32_t *>(tile + L * W);  // one stage of STAGE_WORDS
  double2 *twS = reinterpret_cast<double2 *>(stg + K::STAGE_WORDS);
  double2 *pwS = twS + L;
  double2 *fac = pwS + L;  // tile factors of the current unit
  tw16_build<L>(twS, p.twL1);
  table_to_smem(pwS, p.pw_fwd, L);
  const int tid = threadIdx.x, s = tid % W, t = tid / W;
  const double twoM = 2.0 * (double)p.M;
  const ColTw16 ct = col_tw16<R>(s, t, twoM);
  const int tiles = p.S1 / W;
  const unsigned nA = fwd_units_a(p, (unsigned)tiles);
  const unsigned total = nA + fwd_units_b(p, (unsigned)tiles);  // far below 2^32
  const FastDiv fd_tile((unsigned)tiles);
  // limb staging: as k2_outer_fwd (every row segment of a tile shares one
  // alignment below a 16-byte boundary)
  auto seg_shift = [&](int tl, int b, bool al16) -> int {
    return al16 ? (int)((((long long)tl * W * b >> 5) - 1) & 3) : 0;
  };
  auto stage_copy = [&](unsigned u) {
    const FwdUnit f = fwd_unit(p, u, nA, fd_tile, (unsigned)tiles);
    const int tl = (int)f.rest, op = f.op;
    const ItemDesc &it = p.items[f.item];
    const uint32_t *X = op ? it.B : it.A;
    const int XL = (int)(op ? it.BL : it.AL);
    const int b = it.b;
    const bool al16 = op ? it.b16 : it.a16;
    const int RW = (int)((unsigned)p.S1 * (unsigned)b / 32), PW = (int)((unsigned)p.M * (unsigned)b / 32);
    const int wbase = ((tl * W * b) >> 5) - 1 - seg_shift(tl, b, al16);
    const int parts = (op ? it.ndB : it.ndA) > (unsigned long long)p.M ? 2 : 1;
    if (al16) {
      constexpr int CH = K::SEGW4 / 4;
      const int NCH = parts * L * CH;
      for (int idx = tid; idx < NCH; idx += NT) {
        const int segi = idx / CH, k = idx - segi * CH;
        const int part = segi >= L, row = segi - (part ? L : 0);
        const int w = row * RW + (part ? PW : 0) + wbase + 4 * k;  // multiple of 4
        int nv = XL - w;
        nv = nv < 0 ? 0 : (nv > 4 ? 4 : nv);
        if (w < 0) nv = 0;
        cp_async16(stg + segi * K::SEGW4 + 4 * k, X + (nv ? w : 0), nv * 4);
      }
    } else {
      for (int idx = tid; idx < parts * (K::STAGE_WORDS / 2); idx += NT) {
        const int segi = idx / K::SEGW4, k = idx - segi * K::SEGW4;
        const int part = segi >= L, row = segi - (part ? L : 0);
        const int w = row * RW + (part ? PW : 0) + wbase + k;
        const bool in = w >= 0 && w < XL;
        cp_async4(stg + idx, X + (in ? w : 0), in ? 4 : 0);
      }
    }
  };
  unsigned u = blockIdx.x;
  if (u < total) stage_copy(u);
  cp_async_commit();
  for (; u < total; u += gridDim.x) {
    const FwdUnit f = fwd_unit(p, u, nA, fd_tile, (unsigned)tiles);
    const int tl = (int)f.rest, op = f.op;
    const ItemDesc &it = p.items[f.item];
    const int col = tl * W + s;
    cp_async_wait<0>();
    __syncthreads();  // the stage (every thread's copies) has landed; the last unit's factors are read
    tile_tw16<R, W, NT>(fac, tl, twoM);  // read after block16's barriers
    const unsigned nd = (unsigned)(op ? it.ndB : it.ndA);  // below 2^30
    double2 *gbuf = op ? it.bufB : it.bufA;
    const int b = it.b;
    const bool al16 = op ? it.b16 : it.a16;
    const unsigned rel = 32u * (1u + (unsigned)seg_shift(tl, b, al16)) + (unsigned)((tl * W * b) & 31) +
                         (unsigned)(s * b);  // bit of digit j0+s in its staged segment
    const unsigned wi = (rel - 1) >> 5, sh = (rel - 1) & 31;
    const unsigned mask = (1u << b) - 1;
    const bool imag = nd > (unsigned)p.M;
    auto digit = [&](int part, int n1) -> double {
      const unsigned j = (unsigned)n1 * (unsigned)p.S1 + col + (part ? (unsigned)p.M : 0u);
      const uint32_t *rw = stg + (part * L + n1) * K::SEGW4 + wi;
      const unsigned x = __funnelshift_r(rw[0], rw[1], sh);
      const int r = (int)((x >> 1) & mask);
      const int top = (j + 1 >= nd) ? 0 : (r >> (b - 1));
      return j < nd ? (double)(r - (top << b) + (int)(x & 1u)) : 0.0;
    };
    double2 v[P16];
    if (imag) {
#pragma unroll
      for (int i = 0; i < P16; i++) {
        const int n1 = t + i * R;
        v[i] = cmul(make_double2(digit(0, n1), digit(1, n1)), pwS[n1]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < P16; i++) {
        const int n1 = t + i * R;
        const double d = digit(0, n1);
        const double2 w = pwS[n1];
        v[i] = make_double2(d * w.x, d * w.y);
      }
    }
    __syncthreads();  // every thread has cut its digits: the stage is free
    const unsigned un = u + gridDim.x;
    if (un < total) stage_copy(un);
    cp_async_commit();
    block16<L, W, false>(v, t, s, tile, twS);
    const OuterRun16 tw = outer_run16(fac, ct, t);
    double2 w = tw.b0;
#pragma unroll
    for (int i = 0; i < P16; i++) {
      if (i == 8) w = tw.b1;
      gbuf[(unsigned)(t + i * R) * (unsigned)p.S1 + col] = cmul(v[i], w);
      w = cmul(w, tw.st);
    }
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------------ outer inverse
// Units: (item, column tile), as k2_outer_inv; tiles by TMA one unit ahead.
template <int L>
__global__ void __launch_bounds__(Pass16<L>::NT, Pass16<L>::MINB)
    k3_outer_inv(ClassParams p, const __grid_constant__ CUtensorMap mA) {
  using T = Pass16<L>;
  constexpr int W = T::W, R = T::R, NT = T::NT, G = W / 8;
  extern __shared__ unsigned char smraw[];
  __shared__ uint64_t bars[2];
  double2 *const buf0 = align1024(smraw);  // stage st's tile at buf0 + st * L * W
  double2 *twS = buf0 + 2 * L * W;
  double2 *pwS = twS + L;
  double2 *fac = pwS + L;  // tile factors of unit parity st at fac + st * TILE_TW
  tw16_build<L>(twS, p.twL1);
  table_to_smem(pwS, p.pw_inv, L);
  const int tid = threadIdx.x, s = tid % W, t = tid / W;
  const unsigned tiles = p.S1 / W;
  const unsigned total = (unsigned)p.nitems * tiles;  // far below 2^32
  const FastDiv fd_tiles(tiles);
  const double twoM = 2.0 * (double)p.M;
  const ColTw16 ct = col_tw16<R>(s, t, twoM);
  if (blockIdx.x < total) tile_tw16<R, W, NT>(fac, (int)(blockIdx.x % tiles), twoM);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  // largest rounding error of this thread's units of the current item,
  // published (one atomic per warp) when the item changes and at the end
  double err_acc = 0.0;
  int err_item = -1;
  unsigned phases = 0;  // bit st: parity to wait for on bars[st]
  int st = 0;
  unsigned u = blockIdx.x;
  if (tid == 0 && u < total) {
    fence_proxy_async_smem();
    const unsigned q0 = fd_tiles.div(u);
    tile_load_3d<L, W>(buf0, &mA, &bars[0], (int)(u - q0 * tiles) * W, (int)q0);
  }
  for (; u < total; u += gridDim.x) {
    const unsigned un = u + gridDim.x;
    if (tid == 0 && un < total) {
      fence_proxy_async_smem();
      const unsigned qn = fd_tiles.div(un);
      tile_load_3d<L, W>(buf0 + (st ^ 1) * L * W, &mA, &bars[st ^ 1], (int)(un - qn * tiles) * W, (int)qn);
    }
    const int item = (int)fd_tiles.div(u), tile = (int)(u - (unsigned)item * tiles);
    if (item != err_item) {  // uniform over the CTA: every thread is on unit u
      if (err_item >= 0) atomic_max_err(p.items[err_item].err, err_acc);
      err_acc = 0.0;
      err_item = item;
    }
    const ItemDesc &it = p.items[item];
    const unsigned par = (phases >> st) & 1u;
    const bool ok = mbar_wait(&bars[st], par);
    phases ^= 1u << st;
    double2 *bf = buf0 + st * L * W;
    double2 v[P16];
    {
      const OuterRun16 tw = outer_run16(fac + st * TILE_TW, ct, t);
      double2 w = tw.b0;
#pragma unroll
      for (int i = 0; i < P16; i++) {
        if (i == 8) w = tw.b1;
        v[i] = cmulc(bf[bidx<L>(t + i * R, s)], w);
        w = cmul(w, tw.st);
      }
    }
    if (__syncthreads_or(!ok)) {  // a wait gave up: flag, drain, leave
      if (tid == 0) {
        atomicOr(it.flags, FLAG_TIMEOUT);
        mbar_drain(&bars[st], par);
        if (un < total) mbar_drain(&bars[st ^ 1], (phases >> (st ^ 1)) & 1u);
      }
      return;
    }
    // the next unit's tile factors (read after this unit's last barrier)
    if (un < total) tile_tw16<R, W, NT>(fac + (st ^ 1) * TILE_TW, (int)(un % tiles), twoM);
    block16<L, W, true>(v, t, s, bf, twS);
#pragma unroll
    for (int i = 0; i < P16; i++) {
      const int n1 = t + i * R;
      double2 z = cmul(v[i], pwS[n1]);
      double re = rint(z.x), im = rint(z.y);
      err_acc = fmax(err_acc, round_check(z, re, im));
      bf[bidx<L>(n1, s)] = make_double2(re, im);
    }
    __syncthreads();
    // run records: one 8-column group of one row per (thread, q); L*G rows x
    // groups over NT threads
#pragma unroll
    for (int q = 0; q < (L * G) / NT; q++) {
      const int idx = tid + q * NT, row = idx % L, gi = idx / L;
      double cre[8], cim[8];
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const double2 z = bf[bidx<L>(row, 8 * gi + c)];
        cre[c] = z.x;
        cim[c] = z.y;
      }
      const unsigned n0 = (unsigned)row * (unsigned)p.S1 + (unsigned)tile * W + 8 * gi;
      store_rec(&it.rec[n0 >> 3], make_run(cre, it.b));
      store_rec(&it.rec[(n0 + p.M) >> 3], make_run(cim, it.b));
    }
    static_assert((L * G) % NT == 0, "run pairs per thread");
    __syncthreads();  // the tile buffer is reloaded next iteration
    st ^= 1;
  }
  if (err_item >= 0) atomic_max_err(p.items[err_item].err, err_acc);
}

}  // namespace bc
