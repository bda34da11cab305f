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
#include "passes.cuh"

namespace totem {

namespace {

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
  if (const WindowOps* o = radix_window_ops(n)) return o->twiddles();
  return {};
}

const WindowOps* radix_window_ops_a(int n);
const WindowOps* radix_window_ops_b(int n);
const WindowOps* radix_window_ops_c(int n);
const WindowOps* radix_window_ops_d(int n);

const WindowOps* radix_window_ops(int n) {
  for (auto f : {radix_window_ops_a, radix_window_ops_b, radix_window_ops_c, radix_window_ops_d})
    if (const WindowOps* o = f(n)) return o;
  return nullptr;
}

bool fused_window_ok(int n) {
  if (n >= 64 && n <= 2048 && (n & (n - 1)) == 0) return true;
  return radix_window_ops(n) != nullptr;
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
  if (const WindowOps* o = radix_window_ops(n)) return o->col_tiles;  // one tile width for every variant
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
  if (const WindowOps* o = radix_window_ops(a.n)) return o->col_pass(a, flags, st);
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused slice loop: unsupported window edge");
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
  if (const WindowOps* o = radix_window_ops(n)) {
    *lo = o->band_lo;
    *hi = o->band_hi;
    return;
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
