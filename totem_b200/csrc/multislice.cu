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
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace totem {

namespace {

// One CTA's share of a row pass: rows row0 .. row0+G-1 of one probe's wave.
//   psi_item  the probe's wave [N][N];  t_origin  T at the window origin (row stride p_w),
//   complex64 or, with TB16, bfloat16 pairs;  probe_item  the probe [N][N] (FIRST only: the first
//   pass starts from the probe);  band  the zero band of the propagator: the wave's columns
//   band < c < N - band are zero after the column pass, so they are neither loaded (zeros
//   instead) nor stored (the column pass does not read them).
template <int N, bool FIRST, bool TB16 = false>
__device__ __forceinline__ void row_tile(float2* __restrict__ psi_item, const void* __restrict__ t_origin, long p_w,
                                         const float2* __restrict__ probe_item, int row0, float scale,
                                         const float2* __restrict__ tw, int band) {
  using TElem = std::conditional_t<TB16, __nv_bfloat162, float2>;
  constexpr int P = RowCfg<N>::P, T = RowCfg<N>::T;
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
    for (int m = 0; m < P; ++m) v[m] = in_zero_band(j + m * T, band, N) ? make_float2(0.f, 0.f) : prow[j + m * T];
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
    if (!in_zero_band(j + m * T, band, N)) prow[j + m * T] = v[m];
}

template <int N, bool FIRST, bool TB16>
__global__ void __launch_bounds__(RowCfg<N>::G * RowCfg<N>::T, RowCfg<N>::MINB)
    k_row_pass(SliceLoopArgs a, const void* __restrict__ tslice, float scale) {
  constexpr int G = RowCfg<N>::G;
  using TElem = std::conditional_t<TB16, __nv_bfloat162, float2>;
  const long grow0 = (long)blockIdx.x * G;  // G divides N: the CTA's rows belong to one item
  const int item = (int)(grow0 / N), row0 = (int)(grow0 % N);
  const int gi = a.item0 + item;
  const int w = gi / a.geo.depth, pos = gi - w * a.geo.depth;
  const int x0 = a.geo.begin_row + (pos / a.geo.width_red) * a.geo.step;
  const int y0 = a.geo.begin_col + (pos % a.geo.width_red) * a.geo.step;
  row_tile<N, FIRST, TB16>(a.psi + (long)item * N * N,
                           static_cast<const TElem*>(tslice) + (long)x0 * a.geo.p_width + y0, a.geo.p_width,
                           a.probe + (long)w * N * N, row0, scale, a.tw, a.band);
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
// 4 final pass (no inverse transform), 8 (with 4) store the spectrum.  A column inside the zero
// band (band < c < N - band; the propagator is zero on it) is taken as zero, not loaded, and not
// stored, except that a kept spectrum (flag 8) is stored whole.
template <int N, bool PREFETCH, int G>
__device__ __forceinline__ void col_tile(float2* __restrict__ psi_item, const ColInputs& in, int item, int cb, int flags,
                                         const float2* __restrict__ tw, int band) {
  constexpr int P = ColCfg<N>::P, T = ColCfg<N>::T;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  __shared__ double red[32];
  constexpr int nblk = N / G;
  const int j = threadIdx.x / G, g = threadIdx.x - j * G;
  const int c = cb * G + g;
  const bool zc = in_zero_band(c, band, N);
  load_twiddles<N>(s_tw, tw);
  float2* base = psi_item + c;
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) v[m] = zc ? make_float2(0.f, 0.f) : base[(long)(j + m * T) * N];
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
  if (!zc) {
#pragma unroll
    for (int m = 0; m < P; ++m) base[(long)(j + m * T) * N] = v[m];
  }
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
  col_tile<N, PREFETCH, G>(a.psi + (long)item * N * N, in, item, cb, flags, a.tw, a.band);
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

// Row pass of a continuous batch: the same tile as k_row_pass, with the probe, transmission slice
// and window of each item taken from its group.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::G * RowCfg<N>::T, RowCfg<N>::MINB)
    k_row_groups(const GroupDesc* __restrict__ groups, const int* __restrict__ item_begin, int ngroups, int tick,
                 const float2* __restrict__ tw) {
  constexpr int G = RowCfg<N>::G, per_item = N / G;
  const int li = blockIdx.x / per_item;
  const int row0 = (blockIdx.x - li * per_item) * G;
  const int gidx = find_group(item_begin, ngroups, li);
  const GroupDesc& d = groups[gidx];
  const int item = li - __ldg(item_begin + gidx);
  const int slice = tick - d.start_tick;
  const int gi = d.item0 + item;
  const int w = gi / d.geo.depth, pos = gi - w * d.geo.depth;
  const int x0 = d.geo.begin_row + (pos / d.geo.width_red) * d.geo.step;
  const int y0 = d.geo.begin_col + (pos % d.geo.width_red) * d.geo.step;
  const long p_w = d.geo.p_width;
  const float2* t_origin = d.t_stack + (long)slice * d.p_h * p_w + (long)x0 * p_w + y0;
  float2* psi_item = d.psi + (long)item * N * N;
  if (slice == 0)
    row_tile<N, true>(psi_item, t_origin, p_w, d.probe + (long)w * N * N, row0, 1.f, tw, d.band);
  else
    row_tile<N, false>(psi_item, t_origin, p_w, nullptr, row0, 1.f / ((float)N * (float)N), tw, d.band);
}

// Column pass of a continuous batch: detectors at the group's mid-layer slices, exit detectors
// and no inverse transform at its last slice.
template <int N>
__global__ void __launch_bounds__(ColCfg<N>::G * ColCfg<N>::T, ColCfg<N>::MINB)
    k_col_groups(const GroupDesc* __restrict__ groups, const int* __restrict__ item_begin, int ngroups, int tick,
                 const float2* __restrict__ tw, TileSkip skip) {
  constexpr int G = ColCfg<N>::G, nblk = N / G;
  const int active = nblk - skip.nskip;
  const int li = blockIdx.x / active, t = blockIdx.x - li * active;
  const int cb = t < skip.z0 ? t : t + skip.nskip;
  const int gidx = find_group(item_begin, ngroups, li);
  const GroupDesc& d = groups[gidx];
  const int item = li - __ldg(item_begin + gidx);
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
  col_tile<N, false, G>(d.psi + (long)item * N * N, in, item, cb, flags, tw, d.band);
}

__global__ void k_det_reduce(const double* __restrict__ part, int nblk, int aper_num, int items, int item0,
                             int depth, double* __restrict__ acc, TileSkip skip) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= items * aper_num) return;
  const int item = t / aper_num, a = t - item * aper_num;
  const double* p = part + (long)t * nblk;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b)
    if (b < skip.z0 || b >= skip.z0 + skip.nskip) s += p[b];
  const int gi = item0 + item;
  const int w = gi / depth, pos = gi - w * depth;
  acc[((long)w * aper_num + a) * depth + pos] = s;
}

__global__ void k_combine(const double* __restrict__ acc, const double* __restrict__ gfsf, int w_num, long ad,
                          double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= ad) return;
  double s = 0.0;
  for (int w = 0; w < w_num; ++w) s += acc[(long)w * ad + i] * gfsf[w];
  out[i] = s;
}

template <int N, bool FIRST, bool TB16>
Status row_pass_t(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  constexpr int G = RowCfg<N>::G, T = RowCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_row_pass<N, FIRST, TB16>, smem));
  const long rows = (long)a.items * N;
  const float scale = FIRST ? 1.f : 1.f / ((float)N * (float)N);
  k_row_pass<N, FIRST, TB16><<<(unsigned)(rows / G), G * T, smem, st>>>(a, tslice, scale);
  return cuda_status(cudaGetLastError(), "k_row_pass");
}

template <int N, bool FIRST>
Status row_pass(const SliceLoopArgs& a, const void* tslice, cudaStream_t st) {
  return a.t_bf16 ? row_pass_t<N, FIRST, true>(a, tslice, st) : row_pass_t<N, FIRST, false>(a, tslice, st);
}

template <int N, bool PREFETCH, int CTAS128, int GW>
Status col_pass_v(const SliceLoopArgs& a, int flags, cudaStream_t st) {
  constexpr int G = ColCfg<N, CTAS128, GW>::G, T = ColCfg<N>::T;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_col_pass<N, PREFETCH, CTAS128, GW>, smem));
  // a kept spectrum is stored whole: no tile is left out then
  const TileSkip skip = (flags & 8) ? TileSkip() : zero_tiles(N, N / G, a.band);
  k_col_pass<N, PREFETCH, CTAS128, GW>
      <<<(unsigned)((long)a.items * (N / G - skip.nskip)), G * T, smem, st>>>(a, flags, skip);
  return cuda_status(cudaGetLastError(), "k_col_pass");
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

}  // namespace

std::vector<float2> stage_twiddles(int n) {
  switch (n) {
    case 64: return tables<64>();
    case 128: return tables<128>();
    case 256: return tables<256>();
    case 512: return tables<512>();
    case 1024: return tables<1024>();
    case 2048: return tables<2048>();
    case 4096: return tables<4096>();
  }
  return {};
}

int col_blocks(int n, int variant) {
  switch (n) {
    case 64: return col_tiles<64>(variant);
    case 128: return col_tiles<128>(variant);
    case 256: return col_tiles<256>(variant);
    case 512: return col_tiles<512>(variant);
    case 1024: return col_tiles<1024>(variant);
    case 2048: return col_tiles<2048>(variant);
  }
  return 0;
}

Status launch_row_pass(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st) {
  switch (a.n) {
#define TOTEM_ROW(NN) \
  case NN: return first ? row_pass<NN, true>(a, tslice, st) : row_pass<NN, false>(a, tslice, st);
    TOTEM_ROW(64) TOTEM_ROW(128) TOTEM_ROW(256) TOTEM_ROW(512) TOTEM_ROW(1024) TOTEM_ROW(2048)
#undef TOTEM_ROW
  }
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused slice loop needs a power-of-two window 64..2048");
}

Status launch_col_pass(const SliceLoopArgs& a, int flags, cudaStream_t st) {
  switch (a.n) {
    case 64: return col_pass<64>(a, flags, st);
    case 128: return col_pass<128>(a, flags, st);
    case 256: return col_pass<256>(a, flags, st);
    case 512: return col_pass<512>(a, flags, st);
    case 1024: return col_pass<1024>(a, flags, st);
    case 2048: return col_pass<2048>(a, flags, st);
  }
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused slice loop needs a power-of-two window 64..2048");
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

Status launch_row_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, cudaStream_t st) {
  if (items <= 0 || ngroups <= 0) return Status::Ok();
  switch (n) {
    case 64: return row_groups<64>(groups, item_begin, ngroups, items, tick, tw, st);
    case 128: return row_groups<128>(groups, item_begin, ngroups, items, tick, tw, st);
    case 256: return row_groups<256>(groups, item_begin, ngroups, items, tick, tw, st);
    case 512: return row_groups<512>(groups, item_begin, ngroups, items, tick, tw, st);
    case 1024: return row_groups<1024>(groups, item_begin, ngroups, items, tick, tw, st);
    case 2048: return row_groups<2048>(groups, item_begin, ngroups, items, tick, tw, st);
  }
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "continuous batching needs a power-of-two window 64..2048");
}

Status launch_col_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, TileSkip skip, cudaStream_t st) {
  if (items <= 0 || ngroups <= 0) return Status::Ok();
  switch (n) {
    case 64: return col_groups<64>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 128: return col_groups<128>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 256: return col_groups<256>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 512: return col_groups<512>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 1024: return col_groups<1024>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 2048: return col_groups<2048>(groups, item_begin, ngroups, items, tick, tw, skip, st);
  }
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "continuous batching needs a power-of-two window 64..2048");
}

Status launch_det_reduce(const double* part, int nblk, int aper_num, int items, int item0, int depth, double* acc,
                         cudaStream_t st, TileSkip skip) {
  const int n = items * aper_num;
  if (n == 0) return Status::Ok();
  k_det_reduce<<<(n + 127) / 128, 128, 0, st>>>(part, nblk, aper_num, items, item0, depth, acc, skip);
  return cuda_status(cudaGetLastError(), "k_det_reduce");
}

int spectral_band(const double* re, const double* im, int h, int w) {
  int band = 0;
  for (int c = 0; c < w; ++c) {
    const int dist = c < w - c ? c : w - c;
    if (dist <= band) continue;
    for (int r = 0; r < h; ++r)
      if (re[(size_t)r * w + c] != 0.0 || im[(size_t)r * w + c] != 0.0) {
        band = dist;
        break;
      }
  }
  return band;
}

Status launch_combine(const double* acc, const double* gfsf, int w_num, long ad, double* out, cudaStream_t st) {
  if (ad == 0) return Status::Ok();
  k_combine<<<(unsigned)((ad + 255) / 256), 256, 0, st>>>(acc, gfsf, w_num, ad, out);
  return cuda_status(cudaGetLastError(), "k_combine");
}

}  // namespace totem
