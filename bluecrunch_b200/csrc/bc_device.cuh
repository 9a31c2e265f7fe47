// bc_device.cuh — device building blocks for the exact FP64 FFT multiply.
//
// Arithmetic follows the reference's product C = A*B (bigfloat/mul.c:108-174)
// but the transform is designed for sm_100a:
//   * balanced b-bit digits (d_j in [-2^(b-1), 2^(b-1)]) computed without a
//     carry chain: d_j = r_j - 2^b*top(r_j) + top(r_{j-1});
//   * "right-angle" packing: point n holds digits n (real) and n+M (imag),
//     weighted by w^n, w = e^{i pi/(2M)}, so a length-M complex cyclic
//     convolution gives the 2M-coefficient acyclic product with no real-FFT
//     untangling step;
//   * Stockham auto-sort block FFTs (natural order in and out) with radix-8
//     register butterflies and one shared-memory exchange per stage; lengths
//     2^k and 3*2^k (the radix-3 stage runs from shared memory);
//   * all twiddles from tables computed on the host in long double.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bc {

// ------------------------------------------------------------------ complex
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
template <bool INV>
__device__ __forceinline__ double2 ctw(double2 a, double2 w) { return INV ? cmulc(a, w) : cmul(a, w); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 cmul_mi(double2 a) { return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x); }

// ------------------------------------------------------------------ small DFTs
// Forward uses e^{-2 pi i/R}; inverse e^{+2 pi i/R}; both unscaled.
template <bool INV>
__device__ __forceinline__ void dft2(double2 &a, double2 &b) {
  double2 t = a; a = cadd(t, b); b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3) {
  double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = cmul_mi<INV>(csub(a1, a3));
  a0 = cadd(t0, t2); a2 = csub(t0, t2); a1 = cadd(t1, t3); a3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft8(double2 *x) {
  constexpr double H = 0.70710678118654752440084436210484903928483593768847;
  double2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
  double2 o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // o_k *= W8^k
  double2 w1, w2, w3;
  if (!INV) {
    w1 = make_double2(H * (o1.x + o1.y), H * (o1.y - o1.x));
    w3 = make_double2(H * (o3.y - o3.x), -H * (o3.x + o3.y));
  } else {
    w1 = make_double2(H * (o1.x - o1.y), H * (o1.x + o1.y));
    w3 = make_double2(-H * (o3.x + o3.y), H * (o3.x - o3.y));
  }
  w2 = cmul_mi<INV>(o2);
  x[0] = cadd(e0, o0); x[4] = csub(e0, o0);
  x[1] = cadd(e1, w1); x[5] = csub(e1, w1);
  x[2] = cadd(e2, w2); x[6] = csub(e2, w2);
  x[3] = cadd(e3, w3); x[7] = csub(e3, w3);
}

template <bool INV>
__device__ __forceinline__ void dft3(double2 &a, double2 &b, double2 &c) {
  constexpr double S = 0.86602540378443864676372317075293618347140262690519;
  double2 s = cadd(b, c), d = csub(b, c);
  double2 m = make_double2(fma(-0.5, s.x, a.x), fma(-0.5, s.y, a.y));
  // forward: -i*S*d ; inverse: +i*S*d
  double2 r = INV ? make_double2(-S * d.y, S * d.x) : make_double2(S * d.y, -S * d.x);
  a = cadd(a, s);
  b = cadd(m, r);
  c = csub(m, r);
}

// 5-point DFT: with s1 = x1+x4, d1 = x1-x4, s2 = x2+x3, d2 = x2-x3 and
// c_k = cos(2 pi k/5), s_k = sin(2 pi k/5):
//   X0 = x0 + s1 + s2
//   X1, X4 = x0 + c1 s1 + c2 s2 -+ i (s1' d1 + s2' d2)
//   X2, X3 = x0 + c2 s1 + c1 s2 -+ i (s2' d1 - s1' d2)
// (forward: the upper signs, e^{-2 pi i/5}; inverse: the lower).  Constants
// are cos/sin of 2 pi/5 and 4 pi/5 rounded to double.
template <bool INV>
__device__ __forceinline__ void dft5(double2 &x0, double2 &x1, double2 &x2, double2 &x3, double2 &x4) {
  constexpr double C1 = 0.30901699437494745, C2 = -0.8090169943749475;
  constexpr double S1 = 0.9510565162951535, S2 = 0.5877852522924731;
  const double2 s1 = cadd(x1, x4), d1 = csub(x1, x4), s2 = cadd(x2, x3), d2 = csub(x2, x3);
  const double2 t1 = make_double2(fma(C2, s2.x, fma(C1, s1.x, x0.x)), fma(C2, s2.y, fma(C1, s1.y, x0.y)));
  const double2 t2 = make_double2(fma(C1, s2.x, fma(C2, s1.x, x0.x)), fma(C1, s2.y, fma(C2, s1.y, x0.y)));
  // u = S1 d1 + S2 d2, v = S2 d1 - S1 d2 (real combinations), then times -i (forward) or +i
  const double2 u = make_double2(fma(S2, d2.x, S1 * d1.x), fma(S2, d2.y, S1 * d1.y));
  const double2 v = make_double2(fma(-S1, d2.x, S2 * d1.x), fma(-S1, d2.y, S2 * d1.y));
  const double2 iu = cmul_mi<INV>(u), iv = cmul_mi<INV>(v);
  x0 = cadd(x0, cadd(s1, s2));
  x1 = cadd(t1, iu);
  x4 = csub(t1, iu);
  x2 = cadd(t2, iv);
  x3 = csub(t2, iv);
}

template <int R, bool INV>
__device__ __forceinline__ void dftR(double2 *x) {
  if constexpr (R == 2) dft2<INV>(x[0], x[1]);
  else if constexpr (R == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
  else if constexpr (R == 8) dft8<INV>(x);
  else if constexpr (R == 3) dft3<INV>(x[0], x[1], x[2]);
  else if constexpr (R == 5) dft5<INV>(x[0], x[1], x[2], x[3], x[4]);
}

// ------------------------------------------------------------------ block FFT
// An L-point FFT of W independent columns held by NT = (L/8)*W threads, 8
// points per thread.  Thread (t, s): column s in [0,W), t in [0, L/8).
// Register contract on entry and exit: v[i] = x[t + i*(L/8)] of column s
// (natural order), so the first stage reads straight from global memory and
// the last stage writes straight back, both coalesced across s.
//
// Shared-memory layout of a tile (the layout a TMA load with 128-byte
// swizzle writes): W >= 8 columns are W/8 boxes of L rows x 8 columns; the
// 16-byte chunk of column c in row r of a box sits at chunk c ^ (r & 7).
// A single row of L points (W == 1) is one box of L/8 lines of 8.  Any 8
// lanes touching 8 columns of one row, one column of 8 consecutive rows, or
// the Stockham scatter pattern land on distinct banks.

constexpr int PTS = 8;

// Division of 32-bit values by a divisor fixed for a whole kernel, by one
// multiply-high, a subtract, an add and two shifts (Granlund and
// Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994, fig. 4.1): for 1 <= d < 2^32, l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, q = (t + ((n - t) >> min(l,1))) >> max(l-1,0)
// with t = mulhi(m, n).  Built once per CTA; exact for every n < 2^32.
struct FastDiv {
  uint32_t d, m;
  int s1, s2;
  __host__ __device__ explicit FastDiv(uint32_t div) : d(div) {
    int l = 0;
    while (l < 32 && (1ull << l) < (unsigned long long)div) l++;
    m = (uint32_t)((((1ull << l) - div) << 32) / div + 1);
    s1 = l < 1 ? l : 1;
    s2 = l - 1 > 0 ? l - 1 : 0;
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const {
    const uint32_t t = __umulhi(m, n);
    return (t + ((n - t) >> s1)) >> s2;
  }
};

// Barrier policies for block_fft: the threads that exchange data through
// shared memory in one transform.  CtaSync: the whole CTA.  GroupSync<N>:
// the N threads (N a multiple of 32) of group g, on named barrier 1 + g;
// N == 32 is a single warp (__syncwarp).  Groups must not share shared
// memory while a transform runs.
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
template <int N> struct GroupSync {
  static_assert(N % 32 == 0, "named barriers count whole warps");
  int id;
  __device__ __forceinline__ void operator()() const {
    if constexpr (N == 32) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(N) : "memory");
  }
};

constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x / 2); }

template <int L> struct Radices {
  // odd factor of L (3 or 5), done as a first stage from shared memory
  static constexpr int F = (L % 3) == 0 ? 3 : ((L % 5) == 0 ? 5 : 1);
  static constexpr bool has3 = F != 1;  // an odd first stage (radix 3 or 5)
  static constexpr int L2 = L / F;       // power of two part
  static constexpr int log2L2 = ilog2(L2);
  static constexpr int n8 = log2L2 / 3;               // radix-8 stages
  static constexpr int rem = 1 << (log2L2 % 3);       // 1, 2 or 4
};

template <int L, int W>
__device__ __forceinline__ int sidx(int row, int s) {
  static_assert(W == 1 || W % 8 == 0, "tile width must be 1 or a multiple of 8");
  if constexpr (W == 1) return (row & ~7) + ((row & 7) ^ ((row >> 3) & 7));
  else return (s >> 3) * (L * 8) + row * 8 + ((s & 7) ^ (row & 7));
}

template <int L, int W> struct TileSmem {
  static constexpr int elems = (W == 1) ? (L + L / 8) : (L * W);
};

// Per-stage twiddle tables for single-row transforms.  In a row transform
// the lanes of a warp hold consecutive j, so a flat table read at
// k*step (k = j mod NS) strides by multiples of 128 bytes and every lane of a
// quarter-warp hits the same banks.  The staged layout stores, for each
// radix-8 register stage with NS > 1, the twiddles w^1, w^2, w^4 it reads
// for k = 0..NS-1 contiguously at offset(NS) + 3k.  The remainder stage
// (radix 2 or 4) reads the flat table at k*r*L/(NS R) with consecutive k,
// which is conflict-free already (and coalesced from global memory).
template <int L> struct StagedTw {
  using RX = Radices<L>;
  static constexpr int NS0 = RX::F;
  __host__ __device__ static constexpr int offset(int NS) {
    int off = 0, ns = NS0;
    for (int k = 0; k < RX::n8; k++, ns *= 8) {
      if (ns == NS) return off;
      if (ns > 1) off += ns * 3;
    }
    return off;
  }
  __host__ __device__ static constexpr int entries() {
    int off = 0, ns = NS0;
    for (int k = 0; k < RX::n8; k++, ns *= 8)
      if (ns > 1) off += ns * 3;
    return off > 0 ? off : 1;
  }
};

// Fill a staged table from the flat one (flat[m] = e^{-2 pi i m/L}); all
// threads of the CTA, published by the caller's next barrier.
template <int L>
__device__ __forceinline__ void staged_tw_build(double2 *dst, const double2 *__restrict__ flat) {
  using ST = StagedTw<L>;
  using RX = Radices<L>;
  constexpr int n = ST::entries();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int off = 0, ns = ST::NS0, k = 0, e = 0;
    bool found = false;
    for (int st = 0; st < RX::n8; st++, ns *= 8) {
      if (ns == 1) continue;
      if (i < off + 3 * ns) {
        k = (i - off) / 3;
        e = (i - off) - 3 * k;
        found = true;
        break;
      }
      off += 3 * ns;
    }
    dst[i] = found ? flat[k * (1 << e) * (L / (ns * 8))] : make_double2(1.0, 0.0);
  }
}

// Twiddle sources of a transform: `flat` (e^{-2 pi i m/L}, global or shared
// memory) and, for STAGED transforms, the radix-8 stage tables.
struct TwSrc {
  const double2 *flat;
  const double2 *staged;
};

// One register stage of radix R at span NS (Stockham, twiddle before the
// butterfly: x_r *= w^{(j mod NS) r}, w = e^{-+2 pi i/(NS R)}).  Flat
// tables: tw[m] holds e^{-2 pi i m/L}; the largest m any stage reads is
// below 3L/4 (radix 8 reads r*k*L/(8 NS) for r <= 4, radix 4 up to
// 3*k*L/(4 NS), radix 2 k*L/(2 NS), k < NS), so tw_entries<L>() entries
// suffice.  STAGED: radix-8 stages read StagedTw<L> tables.  Outputs stay in
// registers at v[q + r*(8/R)], whose destination row is
// (j/NS)*NS*R + j%NS + r*NS.
template <int L, int R, int NS, bool INV, bool STAGED>
__device__ __forceinline__ void reg_stage(double2 (&v)[PTS], int t, const TwSrc &ts) {
  constexpr int TC = L / PTS, Q = PTS / R;
  const double2 *__restrict__ tw = ts.flat;
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const int j = t + q * TC;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; r++) x[r] = v[q + r * Q];
    if constexpr (NS > 1) {
      const int k = j % NS;
      constexpr int step = L / (NS * R);
      if constexpr (R == 8) {
        // w^1, w^2, w^4 from the table, the other powers by one product each
        double2 w1, w2, w4;
        if constexpr (STAGED) {
          constexpr int off = StagedTw<L>::offset(NS);
          const double2 *b = ts.staged + off + 3 * k;
          w1 = b[0]; w2 = b[1]; w4 = b[2];
        } else {
          w1 = tw[k * step]; w2 = tw[2 * k * step]; w4 = tw[4 * k * step];
        }
        const double2 w3 = cmul(w1, w2), w5 = cmul(w1, w4), w6 = cmul(w2, w4), w7 = cmul(w3, w4);
        x[1] = ctw<INV>(x[1], w1); x[2] = ctw<INV>(x[2], w2); x[3] = ctw<INV>(x[3], w3);
        x[4] = ctw<INV>(x[4], w4); x[5] = ctw<INV>(x[5], w5); x[6] = ctw<INV>(x[6], w6);
        x[7] = ctw<INV>(x[7], w7);
      } else {
#pragma unroll
        for (int r = 1; r < R; r++) x[r] = ctw<INV>(x[r], tw[k * r * step]);
      }
    }
    dftR<R, INV>(x);
#pragma unroll
    for (int r = 0; r < R; r++) v[q + r * Q] = x[r];
  }
}

template <int L> __host__ __device__ constexpr int tw_entries() { return (3 * L) / 4; }

template <int L, int R, int NS, int W>
__device__ __forceinline__ void reg_stage_store(const double2 (&v)[PTS], int t, int s, double2 *sm) {
  constexpr int TC = L / PTS, Q = PTS / R;
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const int j = t + q * TC;
    const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
    for (int r = 0; r < R; r++) sm[sidx<L, W>(base + r * NS, s)] = v[q + r * Q];
  }
}

template <int L, int W>
__device__ __forceinline__ void load_regs(double2 (&v)[PTS], int t, int s, const double2 *sm) {
  constexpr int TC = L / PTS;
#pragma unroll
  for (int i = 0; i < PTS; i++) v[i] = sm[sidx<L, W>(t + i * TC, s)];
}

template <int L, int W>
__device__ __forceinline__ void store_regs(const double2 (&v)[PTS], int t, int s, double2 *sm) {
  constexpr int TC = L / PTS;
#pragma unroll
  for (int i = 0; i < PTS; i++) sm[sidx<L, W>(t + i * TC, s)] = v[i];
}

// Odd first stage (radix F = 3 or 5, NS = 1, no twiddles) run from shared
// memory: the L/F butterflies of each column are spread over the column's
// L/8 threads.
template <int L, int W, bool INV, class Sync>
__device__ __forceinline__ void smem_odd_stage(int t, int s, double2 *sm, const Sync &sync) {
  constexpr int F = Radices<L>::F;
  constexpr int TC = L / PTS, NB = L / F;
  constexpr int MAXB = (NB + TC - 1) / TC;
  double2 a[MAXB][F];
#pragma unroll
  for (int q = 0; q < MAXB; q++) {
    const int j = t + q * TC;
    if (j < NB) {
#pragma unroll
      for (int r = 0; r < F; r++) a[q][r] = sm[sidx<L, W>(j + r * NB, s)];
      dftR<F, INV>(a[q]);
    }
  }
  sync();
#pragma unroll
  for (int q = 0; q < MAXB; q++) {
    const int j = t + q * TC;
    if (j < NB) {
#pragma unroll
      for (int r = 0; r < F; r++) sm[sidx<L, W>(F * j + r, s)] = a[q][r];
    }
  }
  sync();
}

// Radix-8 stages k..n8-1, then the remainder stage; NS is the span so far.
template <int L, int W, bool INV, int NS, int K, bool STAGED, class Sync>
__device__ __forceinline__ void run_pow2_stages(double2 (&v)[PTS], int t, int s, double2 *sm, const TwSrc &tw,
                                                const Sync &sync) {
  using RX = Radices<L>;
  if constexpr (K < RX::n8) {
    reg_stage<L, 8, NS, INV, STAGED>(v, t, tw);
    constexpr bool last = (K + 1 == RX::n8) && (RX::rem == 1);
    if constexpr (!last) {
      reg_stage_store<L, 8, NS, W>(v, t, s, sm);
      sync();
      load_regs<L, W>(v, t, s, sm);
      sync();
      run_pow2_stages<L, W, INV, NS * 8, K + 1, STAGED>(v, t, s, sm, tw, sync);
    }
  } else if constexpr (RX::rem > 1) {
    reg_stage<L, RX::rem, NS, INV, STAGED>(v, t, tw);
  }
}
// Full block FFT.  v in/out per the register contract; sm is this tile's
// shared memory; flat = e^{-2 pi i m/L}, m < tw_entries<L>().  STAGED: the
// radix-8 stages read `staged` (StagedTw<L> layout) instead.  Ends with the
// threads of the sync group past a barrier, so the group may reuse sm.
template <int L, int W, bool INV, class Sync = CtaSync, bool STAGED = false>
__device__ __forceinline__ void block_fft(double2 (&v)[PTS], int t, int s, double2 *sm,
                                          const double2 *__restrict__ flat, const Sync &sync = Sync{},
                                          const double2 *staged = nullptr) {
  const TwSrc tw{flat, staged};
  using RX = Radices<L>;
  static_assert(L % PTS == 0, "block length must be a multiple of 8");
  if constexpr (RX::has3) {
    store_regs<L, W>(v, t, s, sm);
    sync();
    smem_odd_stage<L, W, INV>(t, s, sm, sync);
    load_regs<L, W>(v, t, s, sm);
    sync();
    run_pow2_stages<L, W, INV, RX::F, 0, STAGED>(v, t, s, sm, tw, sync);
  } else {
    run_pow2_stages<L, W, INV, 1, 0, STAGED>(v, t, s, sm, tw, sync);
  }
}

// ------------------------------------------------------------------ twiddles
// e^{-2 pi i m / N} for m < N from a two-level table: lo[m & (2^h-1)] *
// hi[m >> h].  (Host computes both tables in long double.)
struct Tw2 {
  const double2 *lo;
  const double2 *hi;
  uint64_t mask;  // 2^h - 1
  int h;
};
__device__ __forceinline__ double2 tw2_get(const Tw2 &T, uint64_t m) {
  return cmul(__ldg(&T.lo[m & T.mask]), __ldg(&T.hi[m >> T.h]));
}

// ------------------------------------------------------------------ digits
// Balanced digit j of the operand X[0..XL) at width b: r = bits[jb, jb+b),
// top(r) its bit b-1, d = r - 2^b*top(r) + top(r_{j-1}).  The most
// significant digit (j = nd-1, nd = ceil(32 XL / b)) stays unbalanced so the
// sum telescopes without an extra digit.  Zero for j >= nd.
__device__ __forceinline__ double digit_at(const uint32_t *__restrict__ X, uint64_t XL, int b, uint64_t j,
                                           uint64_t nd) {
  if (j >= nd) return 0.0;
  const uint64_t pos = j * (uint64_t)b;
  uint64_t lo_bit = pos == 0 ? 0 : pos - 1;
  const uint64_t w0 = lo_bit >> 5;
  const unsigned sh = (unsigned)(lo_bit & 31);
  uint64_t win = 0;
  if (w0 < XL) win = __ldg(&X[w0]);
  if (w0 + 1 < XL) win |= (uint64_t)__ldg(&X[w0 + 1]) << 32;
  win >>= sh;
  int64_t prevtop, r;
  if (pos == 0) {
    prevtop = 0;
    r = (int64_t)(win & ((1ull << b) - 1));
  } else {
    prevtop = (int64_t)(win & 1);
    r = (int64_t)((win >> 1) & ((1ull << b) - 1));
  }
  const int64_t top = (j + 1 == nd) ? 0 : (r >> (b - 1));
  return (double)(r - (top << b) + prevtop);
}

// ------------------------------------------------------------------ carry
// Run records: 8 consecutive coefficients form one run with value
//   V = sum_u c_u 2^{b u} = H + C * 2^{8b},  0 <= H < 2^{8b}, C signed.
// H is kept in 3 64-bit words (8b <= 192).
struct RunRec {
  unsigned long long h0, h1, h2;
  long long c;
};

// Carry resolution between runs: with X_r = C_{r-1} + delta_{r-1}, the carry
// delta_r out of H_r + X_r beyond C_{r-1} is in {-1,0,1}.  The map
// delta_{r-1} -> delta_r is kept as three 2-bit fields (value+1) for inputs
// -1, 0, +1; composition gives a scan.
__host__ __device__ __forceinline__ int fn_apply(uint32_t f, int d) { return (int)((f >> (2 * (d + 1))) & 3) - 1; }
__host__ __device__ __forceinline__ uint32_t fn_make(int vm, int v0, int vp) {
  return (uint32_t)(vm + 1) | ((uint32_t)(v0 + 1) << 2) | ((uint32_t)(vp + 1) << 4);
}
constexpr uint32_t FN_ID = 0u | (1u << 2) | (2u << 4);
__host__ __device__ __forceinline__ bool fn_is_const(uint32_t f) {
  return (f & 3u) == ((f >> 2) & 3u) && (f & 3u) == ((f >> 4) & 3u);
}
// result = second(first(x))
__host__ __device__ __forceinline__ uint32_t fn_compose(uint32_t first, uint32_t second) {
  return fn_make(fn_apply(second, fn_apply(first, -1)), fn_apply(second, fn_apply(first, 0)),
                 fn_apply(second, fn_apply(first, 1)));
}

// 192-bit helpers (little-endian words).
struct U192 { unsigned long long w[3]; };

// H + v (v signed 64-bit) modulo 2^nbits; returns the carry out in {-1,0,1}.
__host__ __device__ __forceinline__ int u192_add_s64(U192 &h, long long v, int nbits) {
  unsigned long long add = (unsigned long long)v;
  unsigned long long ext = v < 0 ? ~0ull : 0ull;
  unsigned long long s0 = h.w[0] + add;
  unsigned long long c0 = s0 < add;
  unsigned long long s1 = h.w[1] + ext;
  unsigned long long c1 = s1 < ext;
  unsigned long long s1b = s1 + c0;
  c1 += s1b < c0;
  unsigned long long s2 = h.w[2] + ext;
  unsigned long long c2 = s2 < ext;
  unsigned long long s2b = s2 + c1;
  c2 += s2b < c1;
  // full result = s0 + s1b*2^64 + s2b*2^128 + (c2 - (v<0 ? 1 : 0)) * 2^192 ... reduce by nbits
  h.w[0] = s0; h.w[1] = s1b; h.w[2] = s2b;
  // value bits above nbits (as a signed quantity): compute via top word
  // Since |v| < 2^63 and H < 2^nbits with nbits >= 64, the true sum lies in
  // (-2^63, 2^nbits + 2^63); the carry is decided by the bits at >= nbits.
  int carry;
  if (nbits == 192) {
    long long hi = (long long)(c2) - (v < 0 ? 1 : 0);
    carry = (int)hi;
  } else {
    const int wi = nbits >> 6, bi = nbits & 63;
    unsigned long long above;
    if (wi == 1) above = (bi == 0) ? h.w[1] : ((h.w[1] >> bi) | (h.w[2] << (64 - bi)));
    else above = (bi == 0) ? h.w[2] : (h.w[2] >> bi);
    // 'above' is the (wrapped) value of floor(sum / 2^nbits) modulo 2^(192-nbits):
    // it is 0, 1 or all-ones (= -1) in that field.
    carry = (above == 0) ? 0 : ((above & 1) && (above >> 1) == 0 ? 1 : -1);
    // clear bits >= nbits
    if (wi == 1) {
      if (bi == 0) { h.w[1] = 0; h.w[2] = 0; }
      else { h.w[1] &= (1ull << bi) - 1; h.w[2] = 0; }
    } else {
      h.w[2] = bi ? (h.w[2] & ((1ull << bi) - 1)) : 0;
    }
  }
  return carry;
}

__host__ __device__ __forceinline__ bool u192_is_zero(const U192 &h) { return (h.w[0] | h.w[1] | h.w[2]) == 0; }
__host__ __device__ __forceinline__ bool u192_is_ones(const U192 &h, int nbits) {
  const int wi = nbits >> 6, bi = nbits & 63;
  unsigned long long m2 = 0, m1 = ~0ull;
  if (wi == 1) { m1 = bi ? ((1ull << bi) - 1) : 0; m2 = 0; }
  else if (wi == 2) { m2 = bi ? ((1ull << bi) - 1) : 0; }
  else { m2 = ~0ull; }
  if (nbits < 64) return false;  // not used (8b >= 64)
  return h.w[0] == ~0ull && h.w[1] == m1 && h.w[2] == m2;
}

// Bits [off, off+32) of a 192-bit value (off may exceed 192 -> 0).
__host__ __device__ __forceinline__ uint32_t u192_bits32(const U192 &h, int off) {
  if (off >= 192) return 0;
  const int wi = off >> 6, bi = off & 63;
  // selects instead of a runtime word index, so h stays in registers
  const unsigned long long a = wi == 0 ? h.w[0] : (wi == 1 ? h.w[1] : h.w[2]);
  const unsigned long long b = wi == 0 ? h.w[1] : (wi == 1 ? h.w[2] : 0ull);
  unsigned long long lo = a >> bi;
  if (bi > 32) lo |= b << (64 - bi);
  return (uint32_t)lo;
}

// Map for one run: given H_r (8b bits) and C_{r-1}, produce H'_r, G_r and
// the transfer function delta_{r-1} -> delta_r.
__host__ __device__ __forceinline__ uint32_t run_transfer(U192 &h, long long cprev, int nbits) {
  int g = u192_add_s64(h, cprev, nbits);
  bool z = u192_is_zero(h), o = u192_is_ones(h, nbits);
  return fn_make(g - (z ? 1 : 0), g, g + (o ? 1 : 0));
}

// Add a delta in {-1,0,1} modulo 2^nbits.
__host__ __device__ __forceinline__ void u192_add_delta(U192 &h, int d, int nbits) {
  if (d != 0) (void)u192_add_s64(h, (long long)d, nbits);
}

}  // namespace bc
