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
#include "slice_tiles.cuh"

namespace totem {

namespace {

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

Status launch_det_reduce(const double* part, int nblk, int aper_num, int items, int item0, int depth, double* acc,
                         cudaStream_t st, TileSkip skip) {
  const int n = items * aper_num;
  if (n == 0) return Status::Ok();
  k_det_reduce<<<(n + 127) / 128, 128, 0, st>>>(part, nblk, aper_num, items, item0, depth, acc, skip);
  return cuda_status(cudaGetLastError(), "k_det_reduce");
}

void band_columns(int n, int* lo, int* hi) {
  switch (n) {
#define TOTEM_BAND(NN) \
  case NN: *lo = BandCols<NN>::lo; *hi = BandCols<NN>::hi; return;
    TOTEM_BAND(64) TOTEM_BAND(128) TOTEM_BAND(256) TOTEM_BAND(512) TOTEM_BAND(1024) TOTEM_BAND(2048)
#undef TOTEM_BAND
  }
  *lo = *hi = 0;
}

bool band_skip_ok(int n, int band, int col_variant) {
  int lo = 0, hi = 0;
  band_columns(n, &lo, &hi);
  const int nblk = col_blocks(n, col_variant);
  if (hi <= lo || nblk <= 0) return false;
  const int g = n / nblk;
  // the columns lie inside the zero band (band, n - band) and are whole tiles of the variant
  return lo > band && hi <= n - band && lo % g == 0 && hi % g == 0;
}

TileSkip band_tiles(int n, int nblk) {
  int lo = 0, hi = 0;
  band_columns(n, &lo, &hi);
  TileSkip t;
  if (nblk <= 0 || hi <= lo) return t;
  const int g = n / nblk;
  if (lo % g || hi % g) return t;
  t.z0 = lo / g;
  t.nskip = (hi - lo) / g;
  return t;
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
