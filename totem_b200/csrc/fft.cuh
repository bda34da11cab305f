// Shared-memory Stockham FFT building blocks for sm_100a.
//
// A length-N transform (N = 8^k * {1,2,4}, 64 <= N <= 4096) is executed by T = N/8 threads.
// Each thread holds 8 points in registers.  On entry and on exit thread j holds the elements
// at positions j + m*T (m = 0..7), so an inverse transform followed by a point-wise multiply and
// a forward transform never leaves registers between the two transforms.  Stages exchange data
// through a caller-provided shared-memory region; the caller chooses the region's address map
// (row-major with padding for contiguous rows, column-interleaved for strided columns).
//
// Radix sequence: radix-8 stages first, then one radix-2 or radix-4 stage when N is not a power
// of 8.  Twiddles W_N^e = exp(-2 pi i e / N) come from a table computed on the host in FP64 and
// rounded once to FP32 (table index e in [0, N)); the inverse uses their conjugates.
#pragma once
#include <cuda_runtime.h>

namespace totem {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---------------------------------------------------------------------------------------------
// Small DFTs on registers, natural order in and out.
// ---------------------------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& y0, float2& y1, float2& y2, float2& y3) {
  float2 b0 = cadd(y0, y2), b1 = csub(y0, y2);
  float2 b2 = cadd(y1, y3), b3 = mul_mi<INV>(csub(y1, y3));
  y0 = cadd(b0, b2);
  y2 = csub(b0, b2);
  y1 = cadd(b1, b3);
  y3 = csub(b1, b3);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* x) {
  const float r = 0.70710678118654752440f;
  // split into even/odd outputs: u = x[n] + x[n+4], w = (x[n] - x[n+4]) * W8^n
  float2 u0 = cadd(x[0], x[4]), w0 = csub(x[0], x[4]);
  float2 u1 = cadd(x[1], x[5]), w1 = csub(x[1], x[5]);
  float2 u2 = cadd(x[2], x[6]), w2 = csub(x[2], x[6]);
  float2 u3 = cadd(x[3], x[7]), w3 = csub(x[3], x[7]);
  // W8^1 = (1 -/+ i)/sqrt2, W8^2 = -/+ i, W8^3 = (-1 -/+ i)/sqrt2
  if (INV) {
    w1 = make_float2((w1.x - w1.y) * r, (w1.x + w1.y) * r);
    w3 = make_float2((-w3.x - w3.y) * r, (w3.x - w3.y) * r);
  } else {
    w1 = make_float2((w1.x + w1.y) * r, (w1.y - w1.x) * r);
    w3 = make_float2((w3.y - w3.x) * r, (-w3.x - w3.y) * r);
  }
  w2 = mul_mi<INV>(w2);
  dft4<INV>(u0, u1, u2, u3);
  dft4<INV>(w0, w1, w2, w3);
  x[0] = u0; x[2] = u1; x[4] = u2; x[6] = u3;
  x[1] = w0; x[3] = w1; x[5] = w2; x[7] = w3;
}

template <int R, bool INV>
__device__ __forceinline__ void dft_r(float2* x) {
  if (R == 8) dft8<INV>(x);
  else if (R == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
  else dft2<INV>(x[0], x[1]);
}

// ---------------------------------------------------------------------------------------------
// Stage bookkeeping
// ---------------------------------------------------------------------------------------------
template <int N>
struct Fft {
  static_assert(N >= 64 && N <= 4096 && (N & (N - 1)) == 0, "N must be a power of two in [64, 4096]");
  static constexpr int T = N / 8;
  static constexpr int log2N = (N == 64) ? 6 : (N == 128) ? 7 : (N == 256) ? 8 : (N == 512) ? 9
                             : (N == 1024) ? 10 : (N == 2048) ? 11 : 12;
  static constexpr int n8 = log2N / 3;                 // radix-8 stages
  static constexpr int tail = 1 << (log2N - 3 * n8);   // 1, 2 or 4
  static constexpr int stages = n8 + (tail > 1 ? 1 : 0);
};

template <int N, int S>
struct StageInfo {
  static constexpr int R = (S < Fft<N>::n8) ? 8 : Fft<N>::tail;
  static constexpr int Ns = (S == 0) ? 1 : StageInfo<N, S - 1>::Ns * StageInfo<N, S - 1>::R;
};
template <int N>
struct StageInfo<N, -1> {
  static constexpr int R = 1;
  static constexpr int Ns = 1;
};

// Layout functors: map (fft index g, element position n) to a float2 offset in shared memory.
// RowLayout: each FFT owns a contiguous padded region (one pad slot every 16 elements).
template <int N>
struct RowLayout {
  static constexpr int stride = N + N / 16;
  __device__ __forceinline__ int operator()(int g, int n) const { return g * stride + n + (n >> 4); }
  static constexpr int size(int G) { return G * stride; }
};
// ColLayout: G transforms interleaved element by element (position n of transform g at n*G+g),
// plus one pad slot every 16 float2 when G < 8.
template <int N, int G>
struct ColLayout {
  __device__ __forceinline__ int operator()(int g, int n) const {
    int o = n * G + g;
    return (G >= 8) ? o : o + (o >> 4);
  }
  static constexpr int size(int) { return (G >= 8) ? N * G : N * G + (N * G) / 16 + 1; }
};

// One Stockham stage on registers + shared memory.
//   v: registers, layout for this stage: v[q*R + r] = element (j + q*T) + r*N/R (stage input).
//   On return (unless LAST) v holds the inputs of stage S+1 in that stage's layout.
template <int N, int S, bool INV, class Layout>
__device__ __forceinline__ void stockham_stage(float2 (&v)[8], int j, int g, const float2* __restrict__ tw,
                                               float2* sm, const Layout& L) {
  constexpr int R = StageInfo<N, S>::R;
  constexpr int Ns = StageInfo<N, S>::Ns;
  constexpr int T = Fft<N>::T;
  constexpr int Q = 8 / R;
  constexpr bool LAST = (S == Fft<N>::stages - 1);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = j + q * T;
    if (Ns > 1) {
      const int k = b % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = tw[(k * r) * (N / (Ns * R))];
        v[q * R + r] = INV ? cmulc(v[q * R + r], w) : cmul(v[q * R + r], w);
      }
    }
    dft_r<R, INV>(&v[q * R]);
  }
  if (LAST) {
    // outputs at b + r*N/R = j + T*(q + r*Q): renumber to v[m] = element j + m*T
    if (Q > 1) {
      float2 t[8];
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) t[q + r * Q] = v[q * R + r];
#pragma unroll
      for (int m = 0; m < 8; ++m) v[m] = t[m];
    }
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int b = j + q * T;
      const int idxD = (b / Ns) * Ns * R + (b % Ns);
#pragma unroll
      for (int r = 0; r < R; ++r) sm[L(g, idxD + r * Ns)] = v[q * R + r];
    }
    __syncthreads();
    constexpr int Rn = StageInfo<N, S + 1>::R;
    constexpr int Qn = 8 / Rn;
#pragma unroll
    for (int q = 0; q < Qn; ++q)
#pragma unroll
      for (int r = 0; r < Rn; ++r) v[q * Rn + r] = sm[L(g, j + q * T + r * (N / Rn))];
    __syncthreads();
  }
}

template <int N, int S, bool INV, class Layout>
struct StageLoop {
  __device__ __forceinline__ static void run(float2 (&v)[8], int j, int g, const float2* tw, float2* sm,
                                             const Layout& L) {
    stockham_stage<N, S, INV, Layout>(v, j, g, tw, sm, L);
    StageLoop<N, S + 1, INV, Layout>::run(v, j, g, tw, sm, L);
  }
};
template <int N, bool INV, class Layout>
struct StageLoop<N, Fft<N>::stages, INV, Layout> {
  __device__ __forceinline__ static void run(float2 (&)[8], int, int, const float2*, float2*, const Layout&) {}
};

// Unnormalised transform of one length-N sequence held as v[m] = x[j + m*T].
// All threads of the CTA must call it (it contains __syncthreads()).
template <int N, bool INV, class Layout>
__device__ __forceinline__ void fft_regs(float2 (&v)[8], int j, int g, const float2* tw, float2* sm,
                                         const Layout& L) {
  StageLoop<N, 0, INV, Layout>::run(v, j, g, tw, sm, L);
}

// Cooperative copy of the twiddle table (N entries) into shared memory.
template <int N>
__device__ __forceinline__ void load_twiddles(float2* dst, const float2* __restrict__ src) {
  for (int i = threadIdx.x; i < N; i += blockDim.x) dst[i] = src[i];
}

}  // namespace totem
