// Shared-memory Stockham FFT building blocks for sm_100a.
//
// A length-N transform is executed by T = N/P threads that each hold P points in registers.
// On entry and on exit thread j holds the elements at positions j + m*T (m = 0..P-1), so an
// inverse transform followed by a point-wise multiply and a forward transform never leaves
// registers between the two transforms.
//
// Plans (radices per stage, first stage first):
//   N   :  64    128     256      512      1024     2048       4096
//   P   :  8     16      16       32       32       32         32
//   R   :  8x8   16x8    16x16    32x16    32x32    32x8x8     32x16x8
// so N <= 1024 needs one shared-memory exchange per transform.  Radix-16 and radix-32
// butterflies run in registers as 4x4 and 8x4 Cooley-Tukey splits whose internal twiddles are
// compile-time constants.  Mixed-radix windows (96 .. 1600, TOTEM_PLAN below) add radices with
// a factor 3, 5 or 7 (odd primes from the DFT definition folded over conjugate pairs, composites
// such as 24 = 8 x 3 by the same Cooley-Tukey split); their T = N / P need not be a power of two.
// Inter-stage twiddles W_N^e = exp(-2 pi i e / N) come from per-stage
// tables (index (r-1)*Ns + k) computed on the host in FP64, rounded once to FP32 and staged in
// shared memory; lanes with consecutive k read consecutive entries, so the reads are free of bank
// conflicts.  Exchanges use XOR-swizzled addresses chosen so that every 64-bit store and load of
// a half-warp hits distinct banks.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace totem {

// Complex arithmetic on (re, im) pairs with sm_100's packed FP32 instructions (two IEEE FP32
// operations per lane, round-to-nearest, the same results as the scalar forms).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// a * b = a.x * (b.x, b.y) + a.y * (-b.y, b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x)));
}
// a * conj(b) = a.x * (b.x, -b.y) + a.y * (b.y, b.x)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), make_float2(b.x, -b.y), __fmul2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x)));
}
// a + s * (-i b) for s = +1 / -1 (forward) or a + s * (+i b) (inverse): the radix-4 cross term
template <bool INV, int S>
__device__ __forceinline__ float2 cadd_rot(float2 a, float2 b) {
  // -i b = (b.y, -b.x), +i b = (-b.y, b.x)
  constexpr float sx = (INV ? -1.f : 1.f) * S, sy = (INV ? 1.f : -1.f) * S;
  return __ffma2_rn(make_float2(b.y, b.x), make_float2(sx, sy), a);
}

// ---------------------------------------------------------------------------------------------
// Compile-time trigonometry for the butterflies' internal twiddles (Taylor series in double,
// argument reduced to |x| <= pi/4; exact multiples of 2 pi / R only).
// ---------------------------------------------------------------------------------------------
constexpr double kPi = 3.14159265358979323846;
constexpr double ce_poly_sin(double x) {
  double t = x, s = x;
  for (int k = 1; k < 12; ++k) {
    t = -t * x * x / ((2 * k) * (2 * k + 1));
    s += t;
  }
  return s;
}
constexpr double ce_poly_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int k = 1; k < 12; ++k) {
    t = -t * x * x / ((2 * k - 1) * (2 * k));
    s += t;
  }
  return s;
}
// cos / sin of 2 pi e / R via octant symmetry
constexpr double ce_cos_frac(int e, int R) {
  e = ((e % R) + R) % R;
  const int o8 = (8 * e) / R;  // octant index 0..7
  const double x = 2 * kPi * e / R;
  switch (o8) {
    case 0: return ce_poly_cos(x);
    case 1: return ce_poly_sin(kPi / 2 - x);
    case 2: return -ce_poly_sin(x - kPi / 2);
    case 3: return -ce_poly_cos(kPi - x);
    case 4: return -ce_poly_cos(x - kPi);
    case 5: return -ce_poly_sin(3 * kPi / 2 - x);
    case 6: return ce_poly_sin(x - 3 * kPi / 2);
    default: return ce_poly_cos(2 * kPi - x);
  }
}
// sin(2 pi e / R) = cos(2 pi (4 e - R) / (4 R)), exact in integers for every R
constexpr double ce_sin_frac(int e, int R) { return ce_cos_frac(4 * (e % R) - R, 4 * R); }

// x * W_R^e (forward: exp(-2 pi i e/R)); inverse uses the conjugate.  Trivial angles are exact.
template <int E, int R, bool INV>
__device__ __forceinline__ float2 twiddle_const(float2 x) {
  constexpr int e = ((E % R) + R) % R;
  constexpr float r2 = 0.70710678118654752440f;
  if constexpr (e == 0) {
    return x;
  } else if constexpr (4 * e == R) {  // -i (forward)
    return INV ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
  } else if constexpr (2 * e == R) {
    return make_float2(-x.x, -x.y);
  } else if constexpr (4 * e == 3 * R) {  // +i (forward)
    return INV ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
  } else if constexpr (8 * e == R) {  // (1 -/+ i)/sqrt2 = (x + rot x) / sqrt2
    return cscale(cadd_rot<INV, 1>(x, x), r2);
  } else if constexpr (8 * e == 3 * R) {  // (-1 -/+ i)/sqrt2
    return cscale(cadd_rot<INV, 1>(make_float2(-x.x, -x.y), x), r2);
  } else if constexpr (8 * e == 5 * R) {  // (-1 +/- i)/sqrt2
    return cscale(cadd_rot<INV, -1>(make_float2(-x.x, -x.y), x), r2);
  } else if constexpr (8 * e == 7 * R) {  // (1 +/- i)/sqrt2
    return cscale(cadd_rot<INV, -1>(x, x), r2);
  } else {
    constexpr float c = (float)ce_cos_frac(e, R);
    constexpr float s = INV ? (float)ce_sin_frac(e, R) : -(float)ce_sin_frac(e, R);
    return cmul(x, make_float2(c, s));
  }
}

// ---------------------------------------------------------------------------------------------
// Register DFTs, natural order in and out.
// ---------------------------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2* x) {
  const float2 t = x[0];
  x[0] = cadd(t, x[1]);
  x[1] = csub(t, x[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* y) {
  const float2 b0 = cadd(y[0], y[2]), b1 = csub(y[0], y[2]);
  const float2 b2 = cadd(y[1], y[3]);
  const float2 d = csub(y[1], y[3]);
  y[0] = cadd(b0, b2);
  y[2] = csub(b0, b2);
  y[1] = cadd_rot<INV, 1>(b1, d);   // b1 + (-/+ i) d
  y[3] = cadd_rot<INV, -1>(b1, d);  // b1 - (-/+ i) d
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* x) {
  float2 u[4], w[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    u[n] = cadd(x[n], x[n + 4]);
    w[n] = csub(x[n], x[n + 4]);
  }
  w[1] = twiddle_const<1, 8, INV>(w[1]);
  w[2] = twiddle_const<2, 8, INV>(w[2]);
  w[3] = twiddle_const<3, 8, INV>(w[3]);
  dft4<INV>(u);
  dft4<INV>(w);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[2 * k] = u[k];
    x[2 * k + 1] = w[k];
  }
}

template <int R, bool INV>
__device__ __forceinline__ void dft_r(float2* x);

template <int I>
struct IntC {
  static constexpr int value = I;
};
template <int I, int END, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < END) {
    f(IntC<I>{});
    static_for<I + 1, END>(f);
  }
}

// Cooley-Tukey split R = A * B: n = n1 + A n2, X[k2 + B k1] = sum_n1 W_A^{n1 k1} W_R^{n1 k2} DFT_B(x[n1 + A .])[k2]
template <int A, int B, bool INV>
__device__ __forceinline__ void dft_split(float2* x) {
  float2 y[A][B];
  static_for<0, A>([&](auto n1c) {
    constexpr int n1 = decltype(n1c)::value;
    float2 z[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) z[n2] = x[n1 + A * n2];
    dft_r<B, INV>(z);
    static_for<0, B>([&](auto k2c) {
      constexpr int k2 = decltype(k2c)::value;
      y[n1][k2] = twiddle_const<n1 * k2, A * B, INV>(z[k2]);
    });
  });
#pragma unroll
  for (int k2 = 0; k2 < B; ++k2) {
    float2 w[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) w[n1] = y[n1][k2];
    dft_r<A, INV>(w);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) x[k2 + B * k1] = w[k1];
  }
}

// Odd prime R straight from the definition, folded over conjugate pairs: with
// a_m = x_m + x_{R-m}, b_m = x_m - x_{R-m} (m = 1 .. (R-1)/2) and theta = 2 pi m k / R,
//   X_k     = x_0 + sum_m a_m cos(theta) - i sum_m b_m sin(theta)
//   X_{R-k} = x_0 + sum_m a_m cos(theta) + i sum_m b_m sin(theta)
// (forward; the inverse swaps the two signs of i).  The cosines and sines are compile-time
// constants of the series above.
template <int R, bool INV>
__device__ __forceinline__ void dft_odd_prime(float2* x) {
  constexpr int H = (R - 1) / 2;
  float2 a[H], b[H];
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    a[m - 1] = cadd(x[m], x[R - m]);
    b[m - 1] = csub(x[m], x[R - m]);
  }
  float2 out[R];
  float2 s = x[0];
#pragma unroll
  for (int m = 0; m < H; ++m) s = cadd(s, a[m]);
  out[0] = s;
  static_for<1, H + 1>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    float2 re = x[0], im = make_float2(0.f, 0.f);
    static_for<1, H + 1>([&](auto mc) {
      constexpr int m = decltype(mc)::value;
      constexpr float c = (float)ce_cos_frac(m * k, R), sn = (float)ce_sin_frac(m * k, R);
      re = __ffma2_rn(make_float2(c, c), a[m - 1], re);
      im = __ffma2_rn(make_float2(sn, sn), b[m - 1], im);
    });
    out[k] = cadd_rot<INV, 1>(re, im);       // re - i im (forward)
    out[R - k] = cadd_rot<INV, -1>(re, im);  // re + i im (forward)
  });
#pragma unroll
  for (int k = 0; k < R; ++k) x[k] = out[k];
}

constexpr bool ce_pow2(int r) { return r > 0 && (r & (r - 1)) == 0; }
constexpr int ce_odd_factor(int r) {  // smallest odd prime factor (r not a power of two)
  for (int p = 3; p <= r; p += 2)
    if (r % p == 0) return p;
  return r;
}

template <int R, bool INV>
__device__ __forceinline__ void dft_r(float2* x) {
  if constexpr (R == 2) dft2<INV>(x);
  else if constexpr (R == 4) dft4<INV>(x);
  else if constexpr (R == 8) dft8<INV>(x);
  else if constexpr (R == 16) dft_split<4, 4, INV>(x);
  else if constexpr (R == 32) dft_split<8, 4, INV>(x);
  else if constexpr (!ce_pow2(R) && ce_odd_factor(R) == R) dft_odd_prime<R, INV>(x);
  else if constexpr (!ce_pow2(R)) dft_split<R / ce_odd_factor(R), ce_odd_factor(R), INV>(x);  // e.g. 24 = 8 x 3
  else static_assert(R <= 32, "radix");
}

// ---------------------------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------------------------
template <int N>
struct Plan;
template <> struct Plan<64> { static constexpr int P = 8, S = 2; static constexpr int R[3] = {8, 8, 1}; };
template <> struct Plan<128> { static constexpr int P = 16, S = 2; static constexpr int R[3] = {16, 8, 1}; };
template <> struct Plan<256> { static constexpr int P = 16, S = 2; static constexpr int R[3] = {16, 16, 1}; };
template <> struct Plan<512> { static constexpr int P = 32, S = 2; static constexpr int R[3] = {32, 16, 1}; };
template <> struct Plan<1024> { static constexpr int P = 32, S = 2; static constexpr int R[3] = {32, 32, 1}; };
#ifndef TOTEM_PLAN2048_P16
#define TOTEM_PLAN2048_P16 0
#endif
#if TOTEM_PLAN2048_P16  // 16 points per thread: half the registers, twice the threads per transform
template <> struct Plan<2048> { static constexpr int P = 16, S = 3; static constexpr int R[3] = {16, 16, 8}; };
#else
template <> struct Plan<2048> { static constexpr int P = 32, S = 3; static constexpr int R[3] = {32, 8, 8}; };
#endif
template <> struct Plan<4096> { static constexpr int P = 32, S = 3; static constexpr int R[3] = {32, 16, 8}; };

// Windows of 2^a x 3, 5, 7, 9 or 25 (multiples of 16, the window sizes the reference's STEM
// driver can pack): every radix divides P, so T = N / P need not be a power of two (transform
// groups that do not fit a warp evenly synchronise the whole CTA, see group_sync).
#define TOTEM_PLAN(NN, PP, SS, R0_, R1_, R2_)                        \
  template <>                                                        \
  struct Plan<NN> {                                                  \
    static constexpr int P = PP, S = SS;                             \
    static constexpr int R[3] = {R0_, R1_, R2_};                     \
  };
TOTEM_PLAN(96, 24, 2, 24, 4, 1)
TOTEM_PLAN(160, 20, 3, 20, 4, 2)
TOTEM_PLAN(192, 24, 2, 24, 8, 1)
TOTEM_PLAN(288, 24, 2, 24, 12, 1)
TOTEM_PLAN(320, 20, 3, 20, 4, 4)
TOTEM_PLAN(384, 24, 3, 24, 4, 4)
TOTEM_PLAN(400, 20, 2, 20, 20, 1)
TOTEM_PLAN(448, 28, 3, 28, 4, 4)
TOTEM_PLAN(576, 24, 2, 24, 24, 1)
TOTEM_PLAN(640, 40, 3, 40, 8, 2)
TOTEM_PLAN(768, 24, 3, 24, 8, 4)
TOTEM_PLAN(800, 20, 3, 20, 20, 2)
TOTEM_PLAN(1152, 24, 3, 24, 24, 2)
TOTEM_PLAN(1280, 40, 3, 40, 8, 4)
TOTEM_PLAN(1536, 24, 3, 24, 8, 8)
TOTEM_PLAN(1600, 20, 3, 20, 20, 4)
#undef TOTEM_PLAN
// The window edges above, in four quarters compiled apart (windows_mr_a.cu .. windows_mr_d.cu).
#define TOTEM_MR_WINDOWS_A(X) X(96) X(320) X(576) X(1152)
#define TOTEM_MR_WINDOWS_B(X) X(160) X(384) X(640) X(1280)
#define TOTEM_MR_WINDOWS_C(X) X(192) X(400) X(768) X(1536)
#define TOTEM_MR_WINDOWS_D(X) X(288) X(448) X(800) X(1600)
#define TOTEM_MR_WINDOWS(X) TOTEM_MR_WINDOWS_A(X) TOTEM_MR_WINDOWS_B(X) TOTEM_MR_WINDOWS_C(X) TOTEM_MR_WINDOWS_D(X)

template <int N>
struct Fft {
  static constexpr int P = Plan<N>::P;
  static constexpr int T = N / P;
  static constexpr int stages = Plan<N>::S;
  static constexpr int R0 = Plan<N>::R[0];
  static_assert(P % Plan<N>::R[0] == 0 && P % Plan<N>::R[1] == 0 && P % Plan<N>::R[2] == 0, "radices divide P");
  static_assert(Plan<N>::R[0] * Plan<N>::R[1] * (Plan<N>::S == 3 ? Plan<N>::R[2] : 1) == N, "radices multiply to N");
  // twiddle-table size: sum over stages s >= 1 of Ns * (R_s - 1)
  static constexpr int tw_size = (stages == 2) ? R0 * (Plan<N>::R[1] - 1)
                                               : R0 * (Plan<N>::R[1] - 1) + R0 * Plan<N>::R[1] * (Plan<N>::R[2] - 1);
};

template <int N, int S>
struct StageInfo {
  static constexpr int R = Plan<N>::R[S];
  static constexpr int Ns = (S == 0) ? 1 : StageInfo<N, S - 1>::Ns * StageInfo<N, S - 1>::R;
  static constexpr int tw_off =
      (S <= 1) ? 0 : StageInfo<N, S - 1>::tw_off + StageInfo<N, S - 1>::Ns * (StageInfo<N, S - 1>::R - 1);
};
template <int N>
struct StageInfo<N, -1> {
  static constexpr int R = 1, Ns = 1, tw_off = 0;
};

// ---------------------------------------------------------------------------------------------
// Shared-memory address maps (float2 units) for transform g's element p
// ---------------------------------------------------------------------------------------------
// Both maps pad one slot after every R0 elements (R0 = the first radix): p -> p + p / R0.  With
// that padding every 64-bit store and load of the exchanges hits distinct banks for all plans
// (checked by simulation of each stage's access pattern and by ncu), and because the stage
// patterns decompose as p = lo + hi * R0 with lo < R0 known by construction, every address is a
// per-thread base plus a compile-time offset (``split``), with no index arithmetic per element.
template <int N>
struct PadMap {
  static constexpr int R0 = Fft<N>::R0;
  __device__ __forceinline__ static int pad(int p) { return p + p / R0; }
  __device__ __forceinline__ static int split(int hi, int lo) { return hi * (R0 + 1) + lo; }
  // padded index of position p = j + m*T (the register layout of a thread)
  __device__ __forceinline__ static int pos(int j, int m) {
    constexpr int T = Fft<N>::T;
    if constexpr (T <= R0 && R0 % T == 0) {
      constexpr int per = R0 / T;  // register slots per R0 block
      return split(m / per, j + (m % per) * T);
    } else if constexpr (T > R0 && T % R0 == 0) {
      return split(j / R0 + m * (T / R0), j % R0);
    } else {
      return pad(j + m * T);  // mixed-radix plans where neither of T, R0 divides the other
    }
  }
};
// Contiguous per-transform regions (row pass, builder rows).
template <int N>
struct RowLayout {
  static constexpr int stride = N + N / Fft<N>::R0;
  __device__ __forceinline__ int operator()(int g, int p) const { return g * stride + PadMap<N>::pad(p); }
  __device__ __forceinline__ int split(int g, int hi, int lo) const { return g * stride + PadMap<N>::split(hi, lo); }
  __device__ __forceinline__ int pos(int g, int j, int m) const { return g * stride + PadMap<N>::pos(j, m); }
  static constexpr int size(int G) { return G * stride; }
};
// G transforms interleaved element by element (column pass): element p of transform g at
// pad(p) * G + g.
template <int N, int G>
struct ColLayout {
  __device__ __forceinline__ int operator()(int g, int p) const { return PadMap<N>::pad(p) * G + g; }
  __device__ __forceinline__ int split(int g, int hi, int lo) const { return PadMap<N>::split(hi, lo) * G + g; }
  __device__ __forceinline__ int pos(int g, int j, int m) const { return PadMap<N>::pos(j, m) * G + g; }
  static constexpr int size(int) { return (N + N / Fft<N>::R0) * G; }
};

// Barrier over the threads that share one transform.
struct SyncWarp {  // transform groups never straddle a warp
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct SyncBlock {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
template <int NT>
struct SyncNamed {  // one named barrier per group of NT threads (NT a multiple of 32)
  int id;
  __device__ __forceinline__ void operator()() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(NT) : "memory"); }
};

// ---------------------------------------------------------------------------------------------
// One Stockham stage.  Register layout at stage input: v[q*R + r] = x[(j + q*T) + r*N/R];
// for stage 0 that is the entry layout v[m] = x[j + m*T] permuted at compile time.
// ---------------------------------------------------------------------------------------------
// Derive the twiddles of a thread's later sub-sequences from the first by constant rotations
// (fewer shared-memory loads, a few more FMAs); see StageLoop.
#ifndef TOTEM_TW_DERIVE
#define TOTEM_TW_DERIVE 1
#endif
constexpr bool kTwiddleDerive = TOTEM_TW_DERIVE != 0;

template <int N, int S, bool INV, class Layout, class Sync, class Hook>
struct StageLoop {
  __device__ __forceinline__ static void run(float2 (&v)[Fft<N>::P], int j, int g, const float2* __restrict__ tw,
                                             float2* sm, const Layout& L, const Sync& sync, Hook& hook) {
    constexpr int P = Fft<N>::P, T = Fft<N>::T;
    constexpr int R = StageInfo<N, S>::R, Ns = StageInfo<N, S>::Ns;
    constexpr int Q = P / R;
    constexpr bool LAST = (S == Fft<N>::stages - 1);
    __builtin_assume(j >= 0 && j < T);
    if constexpr (S == 0 && Q > 1) {
      // entry layout v[m], m = q + r*Q  ->  stage layout v[q*R + r]
      float2 t[P];
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) t[q * R + r] = v[q + r * Q];
#pragma unroll
      for (int m = 0; m < P; ++m) v[m] = t[m];
    }
    if constexpr (kTwiddleDerive && Ns > 1 && Q > 1 && T * Q <= Ns) {
      // The thread's sub-sequences are b = j + q*T < Ns, so their twiddles are
      // W^(r (j + q T)) = W^(r j) * W^(r q T): one table load per r, and a compile-time rotation
      // for q > 0 (one shared-memory load instead of Q).
      const float2* twr = tw + StageInfo<N, S>::tw_off + j;
      static_for<1, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        const float2 w = twr[(r - 1) * Ns];
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          const float2 x = INV ? cmulc(v[q * R + r], w) : cmul(v[q * R + r], w);
          v[q * R + r] = twiddle_const<r * q * T, Ns * R, INV>(x);
        });
      });
#pragma unroll
      for (int q = 0; q < Q; ++q) dft_r<R, INV>(&v[q * R]);
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int b = j + q * T;
        if constexpr (Ns > 1) {
          const int k = b % Ns;
          const float2* twr = tw + StageInfo<N, S>::tw_off + k;
#pragma unroll
          for (int r = 1; r < R; ++r) {
            const float2 w = twr[(r - 1) * Ns];
            v[q * R + r] = INV ? cmulc(v[q * R + r], w) : cmul(v[q * R + r], w);
          }
        }
        dft_r<R, INV>(&v[q * R]);
      }
    }
    if constexpr (LAST) {
      // outputs at b + r*N/R = j + T*(q + r*Q): back to v[m] = x[j + m*T]
      if constexpr (Q > 1) {
        float2 t[P];
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
          for (int r = 0; r < R; ++r) t[q + r * Q] = v[q * R + r];
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = t[m];
      }
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int b = j + q * T;
        if constexpr (S == 0) {
          // p = R0 * b + r with r < R0
#pragma unroll
          for (int r = 0; r < R; ++r) sm[L.split(g, b, r)] = v[q * R + r];
        } else {
          const int idxD = (b / Ns) * Ns * R + (b % Ns);
#pragma unroll
          for (int r = 0; r < R; ++r) sm[L(g, idxD + r * Ns)] = v[q * R + r];
        }
      }
      sync();
      constexpr int Rn = StageInfo<N, S + 1>::R;
      constexpr int Qn = P / Rn;
#pragma unroll
      for (int q = 0; q < Qn; ++q)
#pragma unroll
        for (int r = 0; r < Rn; ++r) {
          if constexpr (N / Rn == Fft<N>::R0) {
            // p = (j + q*T) + r * R0 with j + q*T < N / Rn = R0
            v[q * Rn + r] = sm[L.split(g, r, j + q * T)];
          } else {
            v[q * Rn + r] = sm[L(g, j + q * T + r * (N / Rn))];
          }
        }
      sync();  // the region is free for the next exchange
      if constexpr (S + 2 == Fft<N>::stages) hook();  // last exchange done: the region is free
      StageLoop<N, S + 1, INV, Layout, Sync, Hook>::run(v, j, g, tw, sm, L, sync, hook);
    }
  }
};

struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

// Unnormalised transform of one length-N sequence held as v[m] = x[j + m*T].  Every thread of
// the transform group must call it (it synchronises through ``sync``).  ``hook()`` runs once,
// right after the last shared-memory exchange, when this transform's region is no longer read
// by the transform (used to prefetch the next operand into it).
template <int N, bool INV, class Layout, class Sync, class Hook = NoHook>
__device__ __forceinline__ void fft_regs(float2 (&v)[Fft<N>::P], int j, int g, const float2* tw, float2* sm,
                                         const Layout& L, const Sync& sync, Hook&& hook = Hook()) {
  StageLoop<N, 0, INV, Layout, Sync, std::remove_reference_t<Hook>>::run(v, j, g, tw, sm, L, sync, hook);
}

// 8-byte asynchronous global -> shared copies (each thread later reads only what it copied).
__device__ __forceinline__ void cp_async8(float2* smem_dst, const float2* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 4-byte variant (a bfloat16 pair).
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Launch shapes shared by the kernels that transform whole rows or whole columns.
// Rows: G transforms of T threads per CTA (each transform inside one warp, or a named barrier
// per transform when T > 32), at most 32 KB of exchange space per CTA.
// Rows per CTA: the largest g up to the cap (256 threads below N = 256, 128 from there, or 4096
// elements) that divides N (a CTA's rows belong to one probe) and makes whole warps; for
// power-of-two N the cap itself.  At 256^2 the 128-thread CTA (8 rows) made the slice loop 3.7 %
// faster than 16 rows (0.364 against 0.378 us per probe*slice); halving the rows at 512, 1024 and
// 2048 made it 4, 4 and 14 % slower.
template <int N>
constexpr int row_group_count() {
  constexpr int T = Fft<N>::T;
  constexpr int threads = N >= 256 ? 128 : 256;
  constexpr int cap = (threads / T < 4096 / N) ? threads / T : (4096 / N > 0 ? 4096 / N : 1);
  for (int g = cap > 0 ? cap : 1; g >= 1; --g)
    if (N % g == 0 && (g * T) % 32 == 0) return g;
  for (int g = (cap > 0 ? cap : 1) + 1; g <= 64; ++g)
    if (N % g == 0 && (g * T) % 32 == 0) return g;
  return 1;
}
template <int N, int CTAS = 0>
struct RowCfg {
  static constexpr int P = Fft<N>::P, T = Fft<N>::T;
  static constexpr int G = row_group_count<N>();
  static_assert((G * T) % 32 == 0 && N % G == 0, "row tile: whole warps, whole probes");
  // resident CTAs of 128 threads requested per SM: 5 caps registers at 96 per thread, which
  // the padded exchange addressing fits without spilling up to N = 1024 (and 5 CTAs is also
  // what the row pass's shared memory allows).  At 1024 a 128-register cap (4 CTAs) made the
  // row pass 12 % faster (3.51 against 4.01 us per probe; no change at 512); from N = 2048
  // (three-stage transforms) 3, i.e. ~170 registers: the 2048 row pass spilled 200 B at 128
  // and ran 22 % slower
  // CTAS != 0 (a row-pass variant) replaces the default
  static constexpr int CTAS128 = CTAS ? CTAS : ((N <= 512) ? 5 : (N <= 1024 ? 4 : 3));
  static constexpr int MINB = (CTAS128 * 128 / (G * T) > 0) ? CTAS128 * 128 / (G * T) : 1;
};
// Columns: G adjacent columns per CTA, thread (j, g) = (tid / G, tid % G), so a warp's loads
// cover 32 / G rows x G columns.
template <int N, int CTAS128 = 4, int GW = 0>
struct ColCfg {
  static constexpr int P = Fft<N>::P, T = Fft<N>::T;
  // GW = 0: the default width, 16 columns (one 128-byte segment per row) up to N = 512, 8 (64
  // bytes) up to 2048 (at 2048 one 512-thread CTA per SM; 4 columns at two CTAs was 10 % slower;
  // at 1024 4-column tiles at four 128-thread CTAs per SM made the column pass 23 % slower)
  static constexpr int G0 = (N <= 512) ? 16 : (N <= 2048 ? 8 : 2);
  // Mixed-radix windows whose tile would exceed 256 threads take half the columns when the half
  // tile is still at most 256 threads (two CTAs per SM): 800^2 12 %, 1152^2 and 1536^2 3 % faster
  // slice loops; at 1600^2 the half tile (320 threads, one CTA per SM) was 8 % slower.
  static constexpr int G = GW ? GW : (((N & (N - 1)) && G0 * T > 256 && (G0 / 2) * T <= 256) ? G0 / 2 : G0);
  static_assert((G * T) % 32 == 0 && N % G == 0, "column tile: whole warps, whole tiles");
  // resident CTAs of 128 threads requested per SM (4 = a 128-register cap)
  static constexpr int MINB = (CTAS128 * 128 / (G * T) > 0) ? CTAS128 * 128 / (G * T) : 1;
};

constexpr int gcd_c(int a, int b) { return b ? gcd_c(b, a % b) : a; }
// Columns [lo, hi) of an N x N window that lie beyond the reference's 2/3-of-Nyquist propagator
// cut (index distance from DC above N / 3, ToTEM_submit_v1.m:1558-1564), rounded inward to whole
// groups of T row-pass elements and whole default column tiles.  When the propagator is zero on
// them (checked per request), every column pass turns them into zeros, so the row pass neither
// loads nor stores them (a compile-time choice: those loads and stores are not emitted) and the
// column pass leaves their tiles out (lo = hi: nothing to leave out).
template <int N>
struct BandCols {
  static constexpr int T = Fft<N>::T, G = ColCfg<N>::G;
  static constexpr int L = T / gcd_c(T, G) * G;
  static constexpr int K = N / 3;
  static constexpr int lo = (K + 1 + L - 1) / L * L;
  static constexpr int hi = ((N - K) / L * L > lo) ? (N - K) / L * L : lo;
};

// Transform groups of T threads: within a warp when T divides 32, whole warps with a named barrier
// when 32 divides T, else (mixed-radix T such as 12 or 20) the whole CTA, whose groups all run
// the same sequence of barriers.
template <int N>
__device__ __forceinline__ auto group_sync(int g) {
  constexpr int T = Fft<N>::T;
  if constexpr (T <= 32 && 32 % T == 0) return SyncWarp{};
  else if constexpr (T % 32 == 0) return SyncNamed<T>{1 + g};
  else return SyncBlock{};
}

// Cooperative copy of the twiddle tables into shared memory (caller synchronises afterwards).
template <int N>
__device__ __forceinline__ void load_twiddles(float2* dst, const float2* __restrict__ src) {
  for (int i = threadIdx.x; i < Fft<N>::tw_size; i += blockDim.x) dst[i] = src[i];
}

}  // namespace totem
