// Row pass of the fused slice loop (single request): row IFFT -> * T[window] / N^2 -> row FFT
// (the first pass: probe * T -> row FFT), every register-cap variant and the zero-band skip.
#include "slice_tiles.cuh"

namespace totem {

namespace {

// CTAS: resident 128-thread CTAs per SM the register allocation is sized for (0 = the default
// of RowCfg; the row-pass variants 3, 4, 5).  SKIP: leave out the zero-band columns.
template <int N, bool FIRST, bool TB16, int CTAS = 0, bool SKIP = false>
__global__ void __launch_bounds__(RowCfg<N, CTAS>::G * RowCfg<N, CTAS>::T, RowCfg<N, CTAS>::MINB)
    k_row_pass(SliceLoopArgs a, const void* __restrict__ tslice, float scale) {
  constexpr int G = RowCfg<N>::G;
  using TElem = std::conditional_t<TB16, __nv_bfloat162, float2>;
  const long grow0 = (long)blockIdx.x * G;  // G divides N: the CTA's rows belong to one item
  const int item = (int)(grow0 / N), row0 = (int)(grow0 % N);
  const int gi = a.item0 + item;
  const int w = gi / a.geo.depth, pos = gi - w * a.geo.depth;
  const int x0 = a.geo.begin_row + (pos / a.geo.width_red) * a.geo.step;
  const int y0 = a.geo.begin_col + (pos % a.geo.width_red) * a.geo.step;
  row_tile<N, FIRST, TB16, SKIP>(a.psi + (long)item * N * N,
                                 static_cast<const TElem*>(tslice) + (long)x0 * a.geo.p_width + y0, a.geo.p_width,
                                 a.probe + (long)w * N * N, row0, scale, a.tw);
}

template <int N, bool FIRST, bool TB16, int CTAS = 0, bool SKIP = false>
Status row_pass_launch(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  constexpr int G = RowCfg<N>::G, T = RowCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_row_pass<N, FIRST, TB16, CTAS, SKIP>, smem));
  const long rows = (long)a.items * N;
  const float scale = FIRST ? 1.f : 1.f / ((float)N * (float)N);
  k_row_pass<N, FIRST, TB16, CTAS, SKIP><<<(unsigned)(rows / G), G * T, smem, st>>>(a, tslice, scale);
  return cuda_status(cudaGetLastError(), "k_row_pass");
}

// the zero-band skip (a.skip_band) chosen at launch; windows without a band skip nothing
template <int N, bool FIRST, bool TB16, int CTAS = 0>
Status row_pass_t(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  if constexpr (!TB16 && BandCols<N>::hi > BandCols<N>::lo)
    if (a.skip_band) return row_pass_launch<N, FIRST, TB16, CTAS, true>(a, tslice, st);
  return row_pass_launch<N, FIRST, TB16, CTAS, false>(a, tslice, st);
}

// Row-pass variants (register caps) for windows of 512 and more: 3 (N >= 1024), 4 or 5 (N <= 1024)
// resident 128-thread CTAs per SM, i.e. about 168, 128 and 96 registers per thread; any other
// value (0, 1, or a cap that is the default already) = the default of RowCfg.  The bfloat16
// trial always uses the default.
template <int N, bool FIRST>
Status row_pass(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  if (a.t_bf16) {
    if (a.skip_band) return Status::Err(TOTEM_ERR_STATE, "the bfloat16 trial computes every column");
    return row_pass_t<N, FIRST, true>(a, tslice, st);
  }
  if constexpr (N >= 1024 && RowCfg<N>::CTAS128 != 3)
    if (a.row_variant == 3) return row_pass_t<N, FIRST, false, 3>(a, tslice, st);
  if constexpr (N >= 512 && RowCfg<N>::CTAS128 != 4)
    if (a.row_variant == 4) return row_pass_t<N, FIRST, false, 4>(a, tslice, st);
  if constexpr (N >= 512 && N <= 1024 && RowCfg<N>::CTAS128 != 5)
    if (a.row_variant == 5) return row_pass_t<N, FIRST, false, 5>(a, tslice, st);
  return row_pass_t<N, FIRST, false>(a, tslice, st);
}

}  // namespace

Status launch_row_pass(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st) {
  switch (a.n) {
#define TOTEM_ROW(NN) \
  case NN: return first ? row_pass<NN, true>(a, tslice, st) : row_pass<NN, false>(a, tslice, st);
    TOTEM_ROW(64) TOTEM_ROW(128) TOTEM_ROW(256) TOTEM_ROW(512) TOTEM_ROW(1024) TOTEM_ROW(2048)
#undef TOTEM_ROW
  }
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused slice loop needs a power-of-two window 64..2048");
}

}  // namespace totem
