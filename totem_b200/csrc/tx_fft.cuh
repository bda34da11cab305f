// The transmission's inverse 2-D FFT with the ifftshift sign and exp(i sigma V) (rows, then
// columns), instantiated per grid size by transmission.cu (powers of two) and windows_mr_*.cu
// (mixed-radix sizes).
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace totem {

namespace {

// Column shape of the builder's transforms: columns of 4096 take four per CTA (32-byte row
// segments, whole sectors; 168 KB of shared memory), shorter ones the default width.
template <int N>
using GridColCfg = ColCfg<N, 4, (N == 4096) ? 4 : 0>;

// In-place inverse FFT of rows of length N (RowCfg<N>::G rows per CTA).
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::G * RowCfg<N>::T, RowCfg<N>::MINB) k_fft_rows_inv(float2* __restrict__ data,
                                                                             const float2* __restrict__ tw) {
  constexpr int P = RowCfg<N>::P, T = RowCfg<N>::T, G = RowCfg<N>::G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int g = threadIdx.x / T, j = threadIdx.x - g * T;
  const long row = (long)blockIdx.x * G + g;
  load_twiddles<N>(s_tw, tw);
  float2* p = data + row * N;
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) v[m] = p[j + m * T];
  __syncthreads();
  fft_regs<N, true>(v, j, g, s_tw, s_x, RowLayout<N>(), group_sync<N>(g));
#pragma unroll
  for (int m = 0; m < P; ++m) p[j + m * T] = v[m];
}

// Column inverse FFT of length N over a p_w-wide plane, (-1)^(r+c), exp(i s V).
template <int N>
__global__ void __launch_bounds__(GridColCfg<N>::G * GridColCfg<N>::T, GridColCfg<N>::MINB) k_fft_cols_exp(float2* __restrict__ data, int p_w,
                                                                             const float2* __restrict__ tw, float sig) {
  constexpr int P = GridColCfg<N>::P, T = GridColCfg<N>::T, G = GridColCfg<N>::G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int j = threadIdx.x / G, g = threadIdx.x - j * G;
  const int nblk = p_w / G;
  const int slice = blockIdx.x / nblk, cb = blockIdx.x - slice * nblk;
  const int c = cb * G + g;
  load_twiddles<N>(s_tw, tw);
  float2* p = data + (long)slice * N * p_w + c;
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) v[m] = p[(long)(j + m * T) * p_w];
  __syncthreads();
  fft_regs<N, true>(v, j, g, s_tw, s_x, ColLayout<N, G>(), SyncBlock());
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int r = j + m * T;
    const float sgn = ((r + c) & 1) ? -1.f : 1.f;
    const float re = sgn * v[m].x * sig, im = sgn * v[m].y * sig;
    const float amp = expf(-im);
    float sn, cs;
    sincosf(re, &sn, &cs);
    p[(long)r * p_w] = make_float2(amp * cs, amp * sn);
  }
}

template <int N>
Status rows_inv(float2* data, long nrows, const float2* tw, cudaStream_t st) {
  constexpr int T = RowCfg<N>::T, G = RowCfg<N>::G;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_fft_rows_inv<N>, smem));
  if (nrows % G) return Status::Err(TOTEM_ERR_UNSUPPORTED, "row count not a multiple of the row tile");
  k_fft_rows_inv<N><<<(unsigned)(nrows / G), G * T, smem, st>>>(data, tw);
  return cuda_status(cudaGetLastError(), "k_fft_rows_inv");
}

template <int N>
Status cols_exp(float2* data, int slices, int p_w, const float2* tw, float sig, cudaStream_t st) {
  constexpr int T = GridColCfg<N>::T, G = GridColCfg<N>::G;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_fft_cols_exp<N>, smem));
  if (p_w % G) return Status::Err(TOTEM_ERR_UNSUPPORTED, "potential width not a multiple of the column tile");
  k_fft_cols_exp<N><<<(unsigned)((long)slices * (p_w / G)), G * T, smem, st>>>(data, p_w, tw, sig);
  return cuda_status(cudaGetLastError(), "k_fft_cols_exp");
}

}  // namespace

}  // namespace totem
