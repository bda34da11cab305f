// Per-tile device code of the fused multislice passes, shared by the single-request kernels
// (multislice.cu, rowpass.cu) and the continuous-batching kernels (groups.cu).
//
// Fused multislice: the propagate-and-transmit loop as alternating row and column passes.
//
// Reference loop (cuda_source_lobato.cu:1313-1398, CPU form cuda_STEM_CPU_Mcore_lobato_peng.m
// :60-73), per slice k:  psi *= T_k[window];  Psi = FFT2(psi);  Psi *= H;  [mid detectors];
// psi = IFFT2(Psi) / N^2.  After the last slice: Psi = FFT2(psi); I_a = sum |Psi|^2 * aper_a.
//
// With FFT2 = (row FFT) o (column FFT), consecutive slices regroup into
//   column pass k : column FFT -> *H -> [detectors] -> column IFFT           (one column at a time)
//   row pass k+1  : row IFFT -> * T_{k+1}[window] / N^2 -> row FFT           (one row at a time)
// so every pass reads and writes psi once and keeps a whole row / column in registers and shared
// memory.  The final FFT2 of the reference cancels the last IFFT2: the exit detectors read the
// spectrum of the last column pass (after *H), which skips one column IFFT and one row pass.
//
// Layout in HBM: psi[item][row][col] complex64, item = w * depth + pos (probe-major, as the
// reference's w_series loop); T[slice][P_H][P_W]; H[N][N] and the masks [A][N][N] in natural
// FFT order (the masks for the exit detector are ifftshift(aper), computed at upload).
#pragma once
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace totem {

namespace {

// One CTA's share of a row pass: rows row0 .. row0+G-1 of one probe's wave.
//   psi_item  the probe's wave [N][N];  t_origin  T at the window origin (row stride p_w),
//   complex64 or, with TB16, bfloat16 pairs;  probe_item  the probe [N][N] (FIRST only: the first
//   pass starts from the probe).  SKIP: the columns BandCols<N>::lo .. hi-1 are zero after every
//   column pass and no column pass reads them, so they are neither loaded (zeros instead) nor
//   stored; they are whole groups of T elements, so this is decided per register slot m at compile
//   time.
template <int N, bool FIRST, bool TB16 = false, bool SKIP = false>
__device__ __forceinline__ void row_tile(float2* __restrict__ psi_item, const void* __restrict__ t_origin, long p_w,
                                         const float2* __restrict__ probe_item, int row0, float scale,
                                         const float2* __restrict__ tw) {
  using TElem = std::conditional_t<TB16, __nv_bfloat162, float2>;
  constexpr int P = RowCfg<N>::P, T = RowCfg<N>::T;
  constexpr int mlo = SKIP ? BandCols<N>::lo / T : P, mhi = SKIP ? BandCols<N>::hi / T : P;  // skipped slots
  static_assert(!SKIP || (BandCols<N>::lo % T == 0 && BandCols<N>::hi % T == 0), "band in whole element groups");
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int g = threadIdx.x / T, j = threadIdx.x - g * T;
  const int row = row0 + g;
  load_twiddles<N>(s_tw, tw);
  const TElem* __restrict__ trow = static_cast<const TElem*>(t_origin) + (long)row * p_w;
  float2* prow = psi_item + (long)row * N;
  const RowLayout<N> L;
  const auto sync = group_sync<N>(g);
  // The transmission window row is copied asynchronously into this row's exchange region as soon
  // as the region is free (kernel start for the first pass, after the inverse transform's last
  // exchange otherwise), so its latency overlaps the transform.  Each thread copies and later
  // reads only its own elements.
  auto prefetch_t = [&]() {
#pragma unroll
    for (int m = 0; m < P; ++m) {
      if constexpr (TB16) cp_async4(&s_x[L.pos(g, j, m)], trow + j + m * T);
      else cp_async8(&s_x[L.pos(g, j, m)], trow + j + m * T);
    }
    cp_async_commit();
  };
  float2 v[P];
  if (FIRST) {
    prefetch_t();
    const float2* src = probe_item + (long)row * N;
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = __ldg(src + j + m * T);
  } else {
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = (m >= mlo && m < mhi) ? make_float2(0.f, 0.f) : prow[j + m * T];
  }
  __syncthreads();  // twiddles staged
  if (!FIRST) fft_regs<N, true>(v, j, g, s_tw, s_x, L, sync, prefetch_t);
  cp_async_wait_all();
#pragma unroll
  for (int m = 0; m < P; ++m) {
    float2 t;
    if constexpr (TB16) t = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&s_x[L.pos(g, j, m)]));
    else t = s_x[L.pos(g, j, m)];
    v[m] = cscale(cmul(v[m], t), scale);
  }
  sync();  // every thread of the transform has read its window values before the region is reused
  fft_regs<N, false>(v, j, g, s_tw, s_x, L, sync);
#pragma unroll
  for (int m = 0; m < P; ++m)
    if (m < mlo || m >= mhi) prow[j + m * T] = v[m];
}

// Deterministic block sum of one double per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double x, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) s += red[i];
  }
  return s;
}

template <int N>
__device__ __forceinline__ void detect(const float (&inten)[Fft<N>::P], const float* __restrict__ masks, int aper_num,
                                       int j, int c, double* __restrict__ part, int item, int cb, int nblk,
                                       double* red) {
  constexpr int P = Fft<N>::P, T = Fft<N>::T;
  for (int a = 0; a < aper_num; ++a) {
    const float* mk = masks + (long)a * N * N + c;
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < P; ++m) acc += (double)inten[m] * (double)__ldg(mk + (long)(j + m * T) * N);
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) part[((long)item * aper_num + a) * nblk + cb] = s;
  }
}

// Inputs of the column pass shared by every item of a launch (or of a group).
struct ColInputs {
  const float2* prop;
  const float* mask_mid;
  const float* mask_exit;
  int aper_num;
  double* part_mid;   // [items][aper_num][nblk] when flags & 1
  double* part_exit;  // [items][aper_num][nblk] when flags & 2
};

// One CTA's share of a column pass: columns cb*G .. cb*G+G-1 of one probe's wave.  ``item`` is
// the item's index in the partial-sum arrays.  flags: 1 mid detectors, 2 exit detectors,
// 4 final pass (no inverse transform), 8 (with 4) store the spectrum.
template <int N, bool PREFETCH, int G>
__device__ __forceinline__ void col_tile(float2* __restrict__ psi_item, const ColInputs& in, int item, int cb, int flags,
                                         const float2* __restrict__ tw) {
  constexpr int P = ColCfg<N>::P, T = ColCfg<N>::T;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  __shared__ double red[32];
  constexpr int nblk = N / G;
  const int j = threadIdx.x / G, g = threadIdx.x - j * G;
  const int c = cb * G + g;
  load_twiddles<N>(s_tw, tw);
  float2* base = psi_item + c;
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) v[m] = base[(long)(j + m * T) * N];
  __syncthreads();
  const ColLayout<N, G> L;
  const SyncBlock sync;
  // PREFETCH: the propagator column is copied into the exchange region once the forward
  // transform has finished with it (each thread copies and reads only its own elements)
  if constexpr (!PREFETCH) {
    fft_regs<N, false>(v, j, g, s_tw, s_x, L, sync);
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = cmul(v[m], __ldg(in.prop + (long)(j + m * T) * N + c));
  } else {
    auto prefetch_h = [&]() {
#pragma unroll
      for (int m = 0; m < P; ++m) cp_async8(&s_x[L.pos(g, j, m)], in.prop + (long)(j + m * T) * N + c);
      cp_async_commit();
    };
    fft_regs<N, false>(v, j, g, s_tw, s_x, L, sync, prefetch_h);
    cp_async_wait_all();
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = cmul(v[m], s_x[L.pos(g, j, m)]);
    sync();  // all propagator values read before the inverse transform reuses the region
  }
  if (flags & 3) {
    float inten[P];
#pragma unroll
    for (int m = 0; m < P; ++m) inten[m] = fmaf(v[m].x, v[m].x, v[m].y * v[m].y);
    if (flags & 1) detect<N>(inten, in.mask_mid, in.aper_num, j, c, in.part_mid, item, cb, nblk, red);
    if (flags & 2) detect<N>(inten, in.mask_exit, in.aper_num, j, c, in.part_exit, item, cb, nblk, red);
  }
  if (flags & 4) {
    if (flags & 8) {  // keep the spectrum (HRTEM: the exit wave and image are taken from it)
#pragma unroll
      for (int m = 0; m < P; ++m) base[(long)(j + m * T) * N] = v[m];
    }
    return;
  }
  fft_regs<N, true>(v, j, g, s_tw, s_x, L, sync);
#pragma unroll
  for (int m = 0; m < P; ++m) base[(long)(j + m * T) * N] = v[m];
}

// Group of launch item ``li``: the last g with item_begin[g] <= li.
__device__ __forceinline__ int find_group(const int* __restrict__ item_begin, int ngroups, int li) {
  int lo = 0, hi = ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(item_begin + mid) <= li) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Rows row0 .. row0 + blockDim.x / T - 1 of item ``item`` of group ``d`` at this tick: the same
// tile as k_row_pass, with the probe, transmission slice and window taken from the group.
template <int N, bool SKIP>
__device__ __forceinline__ void row_group_tile_t(const GroupDesc& d, int item, int row0, int tick,
                                                 const float2* __restrict__ tw) {
  const int slice = tick - d.start_tick;
  const int gi = d.item0 + item;
  const int w = gi / d.geo.depth, pos = gi - w * d.geo.depth;
  const int x0 = d.geo.begin_row + (pos / d.geo.width_red) * d.geo.step;
  const int y0 = d.geo.begin_col + (pos % d.geo.width_red) * d.geo.step;
  const long p_w = d.geo.p_width;
  const float2* t_origin = d.t_stack + (long)slice * d.p_h * p_w + (long)x0 * p_w + y0;
  float2* psi_item = d.psi + (long)item * N * N;
  if (slice == 0)
    row_tile<N, true, false, SKIP>(psi_item, t_origin, p_w, d.probe + (long)w * N * N, row0, 1.f, tw);
  else
    row_tile<N, false, false, SKIP>(psi_item, t_origin, p_w, nullptr, row0, 1.f / ((float)N * (float)N), tw);
}

// A group that skips the zero band (d.skip_band) does so in every pass of every tick.
template <int N>
__device__ __forceinline__ void row_group_tile(const GroupDesc& d, int item, int row0, int tick,
                                               const float2* __restrict__ tw) {
  if constexpr (BandCols<N>::hi > BandCols<N>::lo) {
    if (d.skip_band) {
      row_group_tile_t<N, true>(d, item, row0, tick, tw);
      return;
    }
  }
  row_group_tile_t<N, false>(d, item, row0, tick, tw);
}

// Column tile ``cb`` of item ``item`` of group ``d`` at this tick: detectors at the group's
// mid-layer slices, exit detectors and no inverse transform at its last slice.  A tile inside a
// skipping group's zero band (left in the launch for another group) does nothing: its columns
// were not written, and the group's detector sums leave the tile out.
template <int N, int G>
__device__ __forceinline__ void col_group_tile(const GroupDesc& d, int item, int cb, int tick,
                                               const float2* __restrict__ tw) {
  constexpr int nblk = N / G;
  if (d.skip_band && cb >= d.skip.z0 && cb < d.skip.z0 + d.skip.nskip) return;
  const int slice = tick - d.start_tick;
  const long estride = (long)d.items * d.aper_num * nblk;
  ColInputs in{d.prop, d.mask_mid, d.mask_exit, d.aper_num, nullptr, nullptr};
  int flags = 0;
  const int ev = __ldg(d.event_of_slice + slice + 1);
  if (ev >= 0) {
    flags |= 1;
    in.part_mid = d.part + ev * estride;
  }
  if (slice == d.slices - 1) {
    flags |= 2 | 4;
    in.part_exit = d.part + d.exit_event * estride;
  }
  col_tile<N, false, G>(d.psi + (long)item * N * N, in, item, cb, flags, tw);
}

}  // namespace

}  // namespace totem
