// HRTEM imaging kernels (fused transforms) from the exit-wave spectrum: the exit wave itself and the partially coherent
// image  I = sum_k w_k |IFFT2(FFT2(psi_exit) .* tf_k)|^2  (ToTEM_submit_v1.m:1355-1369, where
// tf_k = ifftshift(tcc_k .* objective aperture) and ifft2 is normalised by 1/N^2).
//
// Two passes over N x N, as in the slice loop: k_img_cols takes column tiles of the spectrum,
// multiplies by tf_k and inverse-transforms them (one plane per k); k_img_rows inverse-transforms
// the rows and either stores the complex result or accumulates w_k |.|^2 over k inside the
// thread that owns the pixels, so the sum has a fixed order.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace totem {

namespace {


template <int N>
__global__ void __launch_bounds__(ColCfg<N>::G * ColCfg<N>::T, ColCfg<N>::MINB)
    k_img_cols(const float2* __restrict__ spec, const float2* __restrict__ tf, float2* __restrict__ work,
               const float2* __restrict__ tw) {
  constexpr int P = ColCfg<N>::P, T = ColCfg<N>::T, G = ColCfg<N>::G, nblk = N / G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int j = threadIdx.x / G, g = threadIdx.x - j * G;
  const int k = blockIdx.x / nblk, cb = blockIdx.x - k * nblk;
  const int c = cb * G + g;
  load_twiddles<N>(s_tw, tw);
  const long plane = (long)N * N;
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const long idx = (long)(j + m * T) * N + c;
    v[m] = spec[idx];
    if (tf != nullptr) v[m] = cmul(v[m], __ldg(tf + k * plane + idx));
  }
  __syncthreads();
  fft_regs<N, true>(v, j, g, s_tw, s_x, ColLayout<N, G>(), SyncBlock());
  float2* dst = work + k * plane + c;
#pragma unroll
  for (int m = 0; m < P; ++m) dst[(long)(j + m * T) * N] = v[m];
}

// MODE 0: out_c = rows of plane 0, inverse-transformed and scaled by 1/N^2.
// MODE 1: out_i = sum over k of w_k |row IFFT(plane k) / N^2|^2.
template <int N, int MODE>
__global__ void __launch_bounds__(RowCfg<N>::G * RowCfg<N>::T, RowCfg<N>::MINB)
    k_img_rows(const float2* __restrict__ work, int planes, const double* __restrict__ w, float2* __restrict__ out_c,
               float* __restrict__ out_i, const float2* __restrict__ tw) {
  constexpr int P = RowCfg<N>::P, T = RowCfg<N>::T, G = RowCfg<N>::G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int g = threadIdx.x / T, j = threadIdx.x - g * T;
  const long row = (long)blockIdx.x * G + g;
  load_twiddles<N>(s_tw, tw);
  __syncthreads();
  const float scale = 1.f / ((float)N * (float)N);
  const long plane = (long)N * N;
  float acc[P];
#pragma unroll
  for (int m = 0; m < P; ++m) acc[m] = 0.f;
  for (int k = 0; k < planes; ++k) {
    float2 v[P];
    const float2* src = work + k * plane + row * N;
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = src[j + m * T];
    fft_regs<N, true>(v, j, g, s_tw, s_x, RowLayout<N>(), group_sync<N>(g));
    if (MODE == 0) {
#pragma unroll
      for (int m = 0; m < P; ++m) out_c[row * N + j + m * T] = cscale(v[m], scale);
    } else {
      const float wk = (float)w[k];
#pragma unroll
      for (int m = 0; m < P; ++m) {
        const float2 u = cscale(v[m], scale);
        acc[m] = fmaf(wk, fmaf(u.x, u.x, u.y * u.y), acc[m]);
      }
    }
  }
  if (MODE == 1) {
#pragma unroll
    for (int m = 0; m < P; ++m) out_i[row * N + j + m * T] = acc[m];
  }
}

template <int N>
Status image_n(const float2* spec, const float2* tf, int planes, const double* w, float2* work, float2* out_c,
               float* out_i, const float2* tw, cudaStream_t st) {
  {
    constexpr int G = ColCfg<N>::G, T = ColCfg<N>::T;
    const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
    TOTEM_TRY(ensure_smem((const void*)k_img_cols<N>, smem));
    k_img_cols<N><<<(unsigned)(planes * (N / G)), G * T, smem, st>>>(spec, tf, work, tw);
    TOTEM_TRY(cuda_status(cudaGetLastError(), "k_img_cols"));
  }
  constexpr int G = RowCfg<N>::G, T = RowCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  if (out_i == nullptr) {
    TOTEM_TRY(ensure_smem((const void*)k_img_rows<N, 0>, smem));
    k_img_rows<N, 0><<<N / G, G * T, smem, st>>>(work, 1, w, out_c, out_i, tw);
  } else {
    TOTEM_TRY(ensure_smem((const void*)k_img_rows<N, 1>, smem));
    k_img_rows<N, 1><<<N / G, G * T, smem, st>>>(work, planes, w, out_c, out_i, tw);
  }
  return cuda_status(cudaGetLastError(), "k_img_rows");
}

}  // namespace

}  // namespace totem
