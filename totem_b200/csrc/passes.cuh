// Kernel templates of the fused slice loop and of continuous batching, instantiated per window
// size by the files that dispatch on it (power-of-two windows: rowpass.cu, multislice.cu,
// groups.cu; mixed-radix windows: windows_mixed_*.cu).
#pragma once
#include "hrtem_kernels.cuh"
#include "tx_fft.cuh"
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

// Column-pass variants, per 2048-probe launch on the SrTiO3 512^2 workload (microseconds per
// probe): 16-column tiles with the propagator read from global memory (L2-resident) at a
// 128-register cap, 0.98 (the default); 8-column tiles 1.11; 32-column tiles 1.32; 16-column
// tiles at an 80-register cap 1.10 (it spills).  A persistent column pass streaming the next
// tile into shared memory with cp.async while transforming the current one (one 256-thread CTA
// per SM for its 134 KB of shared memory) measured 1.22, with 8-column tiles (3 CTAs per SM)
// 1.24: the pass needs warps more than it needs its loads hidden.  With 8-column tiles,
// prefetching the propagator into shared memory (4.6 ms against 4.3 ms per 4096 probes) and an
// 80-register cap (5.8 ms) were slower.
// The launch covers the tiles outside [skip.z0, skip.z0 + skip.nskip) only.
template <int N, bool PREFETCH, int CTAS128, int GW>
__global__ void __launch_bounds__(ColCfg<N, CTAS128, GW>::G * ColCfg<N, CTAS128, GW>::T, ColCfg<N, CTAS128, GW>::MINB)
    k_col_pass(SliceLoopArgs a, int flags, TileSkip skip) {
  constexpr int G = ColCfg<N, CTAS128, GW>::G;
  constexpr int nblk = N / G;
  const int active = nblk - skip.nskip;
  const int item = blockIdx.x / active, t = blockIdx.x - item * active;
  const int cb = t < skip.z0 ? t : t + skip.nskip;
  const ColInputs in{a.prop, a.mask_mid, a.mask_exit, a.aper_num, a.part_mid, a.part_exit};
  col_tile<N, PREFETCH, G>(a.psi + (long)item * N * N, in, item, cb, flags, a.tw);
}

template <int N, bool PREFETCH, int CTAS128, int GW>
Status col_pass_v(const SliceLoopArgs& a, int flags, cudaStream_t st) {
  constexpr int G = ColCfg<N, CTAS128, GW>::G, T = ColCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_col_pass<N, PREFETCH, CTAS128, GW>, smem));
  const TileSkip skip = a.skip_band ? band_tiles(N, N / G) : TileSkip();
  k_col_pass<N, PREFETCH, CTAS128, GW>
      <<<(unsigned)((long)a.items * (N / G - skip.nskip)), G * T, smem, st>>>(a, flags, skip);
  TOTEM_TRY(cuda_status(cudaGetLastError(), "k_col_pass"));
  if ((flags & 8) && skip.nskip) {
    // a kept spectrum is stored whole: on the skipped columns it is exactly zero (the propagator is)
    const size_t pitch = (size_t)N * sizeof(float2);
    TOTEM_CUDA(cudaMemset2DAsync(a.psi + (size_t)skip.z0 * G, pitch, 0, (size_t)skip.nskip * G * sizeof(float2),
                                 (size_t)a.items * N, st));
  }
  return Status::Ok();
}

// Column-pass variants: 0/1 default; 2 propagator prefetched to shared memory; 3 a cap of
// 6 x 128 threads per SM (80 registers at 16 columns); 5 tiles of 8 columns (up to N = 2048);
// 6 tiles of 32 columns (up to N = 512).  col_blocks() gives the number of column tiles, i.e. of
// detector partial sums per probe, of each variant.
template <int N>
Status col_pass(const SliceLoopArgs& a, int flags, cudaStream_t st) {
  switch (a.col_variant) {
    case 2: return col_pass_v<N, true, 4, 0>(a, flags, st);
    case 3: return col_pass_v<N, false, (N <= 1024 ? 6 : 4), 0>(a, flags, st);
    case 5: return col_pass_v<N, false, 4, (N <= 2048 ? 8 : 0)>(a, flags, st);
    case 6: return col_pass_v<N, false, 4, (N <= 512 ? 32 : 0)>(a, flags, st);
    default: return col_pass_v<N, false, 4, 0>(a, flags, st);
  }
}

template <int N>
int col_tiles(int variant) {
  if (N <= 2048 && variant == 5) return N / 8;
  if (N <= 512 && variant == 6) return N / 32;
  return N / ColCfg<N>::G;
}

template <int N, int S>
void fill_stage(std::vector<float2>& out) {
  if constexpr (S < Fft<N>::stages) {
    constexpr int R = StageInfo<N, S>::R, Ns = StageInfo<N, S>::Ns;
    if constexpr (S >= 1) {
      for (int r = 1; r < R; ++r)
        for (int k = 0; k < Ns; ++k) {
          const long e = (long)k * r * (N / (Ns * R));
          const double ang = -2.0 * kPi * (double)e / (double)N;
          out[StageInfo<N, S>::tw_off + (r - 1) * Ns + k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
    }
    fill_stage<N, S + 1>(out);
  }
}

template <int N>
std::vector<float2> tables() {
  std::vector<float2> t(Fft<N>::tw_size > 0 ? Fft<N>::tw_size : 1);
  fill_stage<N, 0>(t);
  return t;
}

// Row pass of a continuous batch over groups of one window size.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::G * RowCfg<N>::T, RowCfg<N>::MINB)
    k_row_groups(const GroupDesc* __restrict__ groups, const int* __restrict__ item_begin, int ngroups, int tick,
                 const float2* __restrict__ tw) {
  constexpr int G = RowCfg<N>::G, per_item = N / G;
  const int li = blockIdx.x / per_item;
  const int row0 = (blockIdx.x - li * per_item) * G;
  const int gidx = find_group(item_begin, ngroups, li);
  row_group_tile<N>(groups[gidx], li - __ldg(item_begin + gidx), row0, tick, tw);
}

// Column pass of a continuous batch over groups of one window size.
template <int N>
__global__ void __launch_bounds__(ColCfg<N>::G * ColCfg<N>::T, ColCfg<N>::MINB)
    k_col_groups(const GroupDesc* __restrict__ groups, const int* __restrict__ item_begin, int ngroups, int tick,
                 const float2* __restrict__ tw, TileSkip skip) {
  constexpr int G = ColCfg<N>::G, nblk = N / G;
  const int active = nblk - skip.nskip;
  const int li = blockIdx.x / active, t = blockIdx.x - li * active;
  const int cb = t < skip.z0 ? t : t + skip.nskip;
  const int gidx = find_group(item_begin, ngroups, li);
  col_group_tile<N, G>(groups[gidx], li - __ldg(item_begin + gidx), cb, tick, tw);
}

template <int N>
Status row_groups(const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick, const float2* tw,
                  cudaStream_t st) {
  constexpr int G = RowCfg<N>::G, T = RowCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_row_groups<N>, smem));
  k_row_groups<N><<<(unsigned)(items * (N / G)), G * T, smem, st>>>(groups, item_begin, ngroups, tick, tw);
  return cuda_status(cudaGetLastError(), "k_row_groups");
}

template <int N>
Status col_groups(const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick, const float2* tw,
                  TileSkip skip, cudaStream_t st) {
  constexpr int G = ColCfg<N>::G, T = ColCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_col_groups<N>, smem));
  if (skip.nskip < 0 || skip.z0 < 0 || skip.z0 + skip.nskip > N / G)
    return Status::Err(TOTEM_ERR_STATE, "column tiles to skip out of range");
  k_col_groups<N><<<(unsigned)(items * (N / G - skip.nskip)), G * T, smem, st>>>(groups, item_begin, ngroups, tick,
                                                                                 tw, skip);
  return cuda_status(cudaGetLastError(), "k_col_groups");
}

// ---------------------------------------------------------------------------------------------
// Mixed-radix windows (the TOTEM_MR_WINDOWS sizes): the default launch shapes only (no row-pass
// register caps, no column-pass variants, no bfloat16 trial), reached through a WindowOps table.
// ---------------------------------------------------------------------------------------------
template <int N, bool FIRST>
Status row_pass_mr(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  if (a.t_bf16) return Status::Err(TOTEM_ERR_UNSUPPORTED, "the bfloat16 trial runs power-of-two windows");
  return row_pass_t<N, FIRST, false>(a, tslice, st);
}

template <int N>
Status row_pass_mr_any(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st) {
  return first ? row_pass_mr<N, true>(a, tslice, st) : row_pass_mr<N, false>(a, tslice, st);
}

template <int N>
Status col_pass_mr(const SliceLoopArgs& a, int flags, cudaStream_t st) {
  return col_pass_v<N, false, 4, 0>(a, flags, st);
}

template <int N>
const WindowOps* window_ops() {
  static const WindowOps ops{N,
                             N / ColCfg<N>::G,
                             BandCols<N>::lo,
                             BandCols<N>::hi,
                             &row_pass_mr_any<N>,
                             &col_pass_mr<N>,
                             &row_groups<N>,
                             &col_groups<N>,
                             &tables<N>,
                             &image_n<N>,
                             RowCfg<N>::G,
                             GridColCfg<N>::G,
                             &rows_inv<N>,
                             &cols_exp<N>};
  return &ops;
}

}  // namespace

}  // namespace totem
