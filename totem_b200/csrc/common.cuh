// Shared declarations of the engine's device code and its host-side launchers.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/totem_b200.h"

namespace totem {

// Host-side status carrier used across the engine's C++ code.
struct Status {
  int code = TOTEM_OK;
  std::string msg;
  bool ok() const { return code == TOTEM_OK; }
  static Status Ok() { return Status(); }
  static Status Err(int c, std::string m) {
    Status s;
    s.code = c;
    s.msg = std::move(m);
    return s;
  }
};

Status cuda_status(cudaError_t e, const char* what);
Status cufft_status(cufftResult r, const char* what);
// Raise a kernel's dynamic shared-memory limit once (cached per function pointer).
Status ensure_smem(const void* func, size_t bytes);
// Set the calling thread's message returned by totem_last_error().
void set_last_error(const std::string& msg);

#define TOTEM_CUDA(call)                                              \
  do {                                                                \
    cudaError_t _e = (call);                                          \
    if (_e != cudaSuccess) return ::totem::cuda_status(_e, #call);    \
  } while (0)
#define TOTEM_CUFFT(call)                                             \
  do {                                                                \
    cufftResult _r = (call);                                          \
    if (_r != CUFFT_SUCCESS) return ::totem::cufft_status(_r, #call); \
  } while (0)
#define TOTEM_TRY(expr)                    \
  do {                                     \
    ::totem::Status _s = (expr);           \
    if (!_s.ok()) return _s;               \
  } while (0)

// Window placement of scan position ``pos``: row offset begin_row + (pos / width_red) * step,
// column offset begin_col + (pos % width_red) * step (cuda_source_lobato.cu:344-345).
struct ScanGeom {
  int begin_row, begin_col, step, width_red, depth, p_width;
};

// ---------------------------------------------------------------------------------------------
// Transmission builder
// ---------------------------------------------------------------------------------------------
struct AtomRowsDev {
  const double* pos = nullptr;     // [n][2] x, y in Angstrom (FP64: used for the phase)
  const float* coef = nullptr;     // [n][ncoef]: the row without x, y (occ, a1, b1, ...)
  const float* absorp = nullptr;   // [n][10] or null
  const int* beg = nullptr;        // [slices + 1] first row of every slice
  int ncoef = 0;
};

struct TxGrid {
  int p_h = 0, p_w = 0, slices = 0;
  int separable = 0;               // kx depends on the column only, ky on the row only
  const double* kx_axis = nullptr; // [p_w]  (separable)
  const double* ky_axis = nullptr; // [p_h]
  const double* kx = nullptr;      // [p_h*p_w] (general)
  const double* ky = nullptr;
  const float* s2 = nullptr;       // [p_h*p_w]
  const float* aper_true = nullptr;// [p_h*p_w] or null (all ones)
  float parameter = 0.f;
  int lobato = 0;
  const float* cim = nullptr;      // [cim_len][p_h*p_w] correction planes or null
  int cim_len = 0;
};

// Atoms of one kind grouped by species, i.e. by identical coefficient (and absorptive) rows, so
// that V(g) = sum_species f_species(s^2) * sum_atoms exp(-2 pi i g.r).
struct SpeciesDev {
  const double* pos = nullptr;     // [n][2] x, y, ordered by (slice, species, row order)
  const float* coef = nullptr;     // [species][ncoef]
  const float* absorp = nullptr;   // [species][10] or null
  const int* seg_beg = nullptr;    // [slices + 1] first segment of every slice
  const int* seg = nullptr;        // [segments][3]: species, first atom, end atom
  int ncoef = 0;
};

// The four kinds of coefficient rows by species: 0 neutral, 1 ionic, 2 Peng-extended correction
// (neutral, [B, amplitude, plane]), 3 correction (ionic, [B, amplitude, w1, plane1, w2, plane2]).
struct SpeciesSet {
  SpeciesDev k[4];
};

// V_k(g) * PARAMETER * APERTURE for all slices into out[slice][p_h][p_w] (complex64), one
// thread per pixel and atom row.  accumulate: add to out instead of overwriting it.
Status launch_tx_structure(const TxGrid& g, const AtomRowsDev& neutral, const AtomRowsDev& ion,
                           const AtomRowsDev& corr_n, const AtomRowsDev& corr_i, float2* out,
                           cudaStream_t st, bool accumulate = false);
// The same sums on separable grids, by species (all four kinds): a complex rank-K update per
// species (no exponential per atom and pixel), then the form factor once per species and pixel.
// Overwrites out.
Status launch_tx_species(const TxGrid& g, const SpeciesSet& sp, float2* out, cudaStream_t st);
// The same sums by Gaussian gridding (a type-1 non-uniform FFT) on uniform separable grids.
// Work is grouped in jobs, one per (slice, kind, species) segment, ordered by slice; a batch
// runs the jobs [j_lo, j_hi) in scratch memory and writes slices [s_lo, s_hi) (the last may be
// partial, finished by the next batch).
struct GridPlanDev {
  double dkx = 0, dky = 0;         // spacing of the kx / ky axes
  double sx = 0, sy = 0;           // kx(p_w / 2), ky(p_h / 2): the shift folded into each atom's weight
  const float2* ax = nullptr;      // [p_w][2]: Gaussian deconvolution x half-bin phase (parity 0, 1)
  const float2* ay = nullptr;      // [p_h][2]
  const int4* jobs = nullptr;      // [jobs]: kind (SpeciesSet index), species, first atom, end atom
  const int* job_beg = nullptr;    // [slices + 1] first job of every slice
};
struct GridBatch {
  int s_lo, s_hi, j_lo, j_hi;
};
std::vector<GridBatch> grid_batches(const std::vector<int>& job_beg, int jobs_per_batch);
// Scratch of one job: four p_h x p_w planes of 16-byte points and a flag per fine row.
inline size_t grid_job_bytes(int p_h, int p_w) { return (size_t)p_h * p_w * 64 + (size_t)p_h * 8; }
// Overwrites out like launch_tx_species; ``scratch`` holds at least one job.  ``scratch_zero``:
// the scratch is as an earlier call left it (otherwise it is cleared whole first).
Status launch_tx_gridding(const TxGrid& g, const SpeciesSet& sp, const GridPlanDev& gp,
                          const std::vector<int>& job_beg, const std::vector<int4>& jobs, const float2* tw_w,
                          const float2* tw_h, void* scratch, size_t scratch_bytes, bool scratch_zero, float2* out,
                          cudaStream_t st, int* launches);
// Per-axis factors of the gridding builder for an axis of n points: [c][parity] = the inverse
// of the spreading Gaussian's transform (normalised) times exp(-i pi k parity / n), k = c - n/2.
std::vector<float2> grid_deconvolution(int n);
// Process-wide builder choice for separable grids (TOTEM_TX_*) and gridding scratch bytes.
int tx_builder_mode();
// Process-wide: repeated fused slice loops replay as CUDA graphs (totem_set_slice_graphs).
bool slice_graphs_enabled();
size_t tx_gridding_scratch();
// In-place unnormalised inverse 2-D FFT of every slice, times (-1)^(r+c) (the ifftshift of the
// input), then T = exp(i * sigma_scaled * V).  Powers of two only; returns
// TOTEM_ERR_UNSUPPORTED otherwise.
Status launch_tx_fft_exp(float2* data, int slices, int p_h, int p_w, float sigma_scaled,
                         const float2* tw_w, const float2* tw_h, cudaStream_t st);
// Element-wise (-1)^(r+c) and exp for the cuFFT builder.
Status launch_sign_exp(float2* data, long total, int p_h, int p_w, float sigma_scaled, cudaStream_t st);

// Grid edges of the fused transmission FFT (powers of two 64..4096 and the mixed-radix edges of
// TOTEM_MR_WINDOWS), and of the gridding builder (powers of two 64..4096).
bool fused_fft_size_ok(int n);
bool gridding_size_ok(int n);
// Whether the fused transmission FFT takes a p_h x p_w grid of ``slices`` slices: both edges
// fused_fft_size_ok, the rows of all slices whole row tiles of p_w and the width whole column
// tiles of p_h.
bool tx_fft_shape_ok(int p_h, int p_w, int slices);
// Per-stage twiddle tables of the shared-memory FFT of length n (empty if n is unsupported).
std::vector<float2> stage_twiddles(int n);

// ---------------------------------------------------------------------------------------------
// Fused multislice
// ---------------------------------------------------------------------------------------------
// Spectral band of a propagator H [N][N] (FFT order): the largest index distance from DC,
// min(c, N - c), of a column holding a non-zero entry.  The columns c with band < c < N - band are
// zero in every row, so after the column pass's multiply by H those columns of the wave are zero
// whatever the wave was.  The reference's propagator is cut at 2/3 of Nyquist
// (ToTEM_submit_v1.m:1558-1564): band = N / 3.
int spectral_band(const double* re, const double* im, int h, int w);
// Column tiles [z0, z0 + nskip) left out of a column-pass launch.
struct TileSkip {
  int z0 = 0, nskip = 0;
};
// The fixed zero-band columns of an n x n window (BandCols in fft.cuh; lo = hi: none).
void band_columns(int n, int* lo, int* hi);
// Whether a request with propagator band ``band`` may skip band_columns(n) with the column-pass
// variant ``col_variant``: the columns lie in its zero band and the variant's tiles cover them
// whole.
bool band_skip_ok(int n, int band, int col_variant);
// The tiles of width n / nblk inside band_columns(n).
TileSkip band_tiles(int n, int nblk);
// Process-wide: skip the zero band where band_skip_ok (totem_set_band_skip; on by default).
bool band_skip_enabled();
// Measured FP32 FMA throughput of ``device`` in TFLOP/s (2 flops per FMA), scalar and packed.
Status measure_fma_rates(int device, double* ffma_tflops, double* ffma2_tflops);
// Host-side failure injection (totem_inject_failures): true when the next device allocation of
// the engine, or the next server preparation, is to fail (each call counts one event).
bool inject_alloc_failure();
bool inject_prepare_failure();

struct SliceLoopArgs {
  int n = 0;                       // window edge N (fused_window_ok)
  int items = 0;                   // items in this batch
  int item0 = 0;                   // first global item (w-major: item = w * depth + pos)
  ScanGeom geo{};
  int p_h = 0;
  float2* psi = nullptr;           // [items][N][N]
  const float2* probe = nullptr;   // [w_num][N][N]
  const float2* prop = nullptr;    // [N][N]
  const float2* tw = nullptr;      // N twiddles
  int aper_num = 0;
  const float* mask_mid = nullptr; // [A][N][N] (natural FFT order)
  const float* mask_exit = nullptr;
  double* part_mid = nullptr;      // [items][A][nblk]
  double* part_exit = nullptr;
  int col_variant = 0;             // column-pass variant (multislice.cu, col_pass)
  int t_bf16 = 0;                  // the transmission slices are bfloat16 pairs, not complex64
  int skip_band = 0;               // 1: the passes leave out band_columns(n) (band_skip_ok)
  int row_variant = 0;             // row-pass variant (multislice.cu, row_pass)
};
// Number of column tiles per item (detector partial sums per probe) of a column-pass variant.
int col_blocks(int n, int variant = 0);
// tslice: T[slice] as complex64, or bfloat16 pairs when a.t_bf16.
Status launch_row_pass(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st);
// flags: 1 = mid-slice detectors, 2 = exit detectors, 4 = final pass (no inverse transform),
// 8 = with 4, store the spectrum in psi
Status launch_col_pass(const SliceLoopArgs& a, int flags, cudaStream_t st);
// Continuous batching: one launch advances groups of items of several requests, each group at
// its own slice (slice = tick - start_tick).  Items of a launch are numbered group by group;
// item_begin[g] is the first launch item of group g (item_begin[ngroups] = items of the launch).
struct GroupDesc {
  float2* psi;                  // [items][N][N]
  const float2* t_stack;        // [slices][p_h][p_w]
  const float2* probe;          // [w_num][N][N]
  const float2* prop;           // [N][N]
  const float* mask_mid;        // [A][N][N]
  const float* mask_exit;       // [A][N][N]
  double* part;                 // [events][items][A][col_blocks(N)]
  const int* event_of_slice;    // [slices + 1]: 1-based slice -> mid-layer event or -1
  ScanGeom geo;
  int p_h;
  int item0;                    // first request item of the group (item = w * depth + pos)
  int items;
  int start_tick;
  int slices;
  int aper_num;
  int exit_event;
  int n;                        // window edge (the mixed-size kernels dispatch on it)
  int skip_band;                // 1: this group leaves out band_columns(n) in every pass
  TileSkip skip;                // its zero-band tiles (band_tiles), empty when skip_band is 0
};
Status launch_row_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, cudaStream_t st);
// Groups of 256^2, 512^2 and 1024^2 windows in one persistent launch (k_row_mixed / k_col_mixed):
// CTAs of kMixedThreads threads take work units from ``queue`` (an int the caller zeroes) until
// work_begin[ngroups] units are done; a group has mixed_units(n, row, skip) units per item.
constexpr int kMixedThreads = 256;
struct MixedTwiddles {
  const float2* n256;
  const float2* n512;
  const float2* n1024;
};
bool mixed_window_ok(int n);
int mixed_units(int n, bool row, TileSkip skip);
Status launch_mixed_groups(bool row, const GroupDesc* groups, const int* work_begin, int ngroups, long units,
                           int tick, const MixedTwiddles& tw, int* queue, cudaStream_t st);
// ``skip``: column tiles left out of the launch, wholly inside the zero band of every group in it
Status launch_col_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, TileSkip skip, cudaStream_t st);

// Square windows the fused passes take: powers of two 64..2048, and the mixed-radix edges of
// TOTEM_MR_WINDOWS in fft.cuh (2^a times 3, 5, 7, 9 or 25, 96..1600).
bool fused_window_ok(int n);
// The entry points of one mixed-radix window size (their default launch shapes), which the
// power-of-two dispatchers above fall through to; nullptr when n is not such a size.
struct WindowOps {
  int n;
  int col_tiles;         // column tiles (detector partial sums) per probe
  int band_lo, band_hi;  // BandCols<n>
  Status (*row_pass)(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st);
  Status (*col_pass)(const SliceLoopArgs& a, int flags, cudaStream_t st);
  Status (*row_groups)(const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                       const float2* tw, cudaStream_t st);
  Status (*col_groups)(const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                       const float2* tw, TileSkip skip, cudaStream_t st);
  std::vector<float2> (*twiddles)();
  // HRTEM imaging (launch_exit_wave / launch_tcc_image semantics: out_i == nullptr for the exit wave)
  Status (*image)(const float2* spec, const float2* tf, int planes, const double* w, float2* work, float2* out_c,
                  float* out_i, const float2* tw, cudaStream_t st);
  int row_tile_rows;     // RowCfg<n>::G
  int col_tile_cols;     // the transmission column pass's tile width (GridColCfg<n>::G)
  // the transmission's inverse FFT: rows of length n, then columns of length n with the sign and exp
  Status (*tx_rows_inv)(float2* data, long nrows, const float2* tw, cudaStream_t st);
  Status (*tx_cols_exp)(float2* data, int slices, int p_w, const float2* tw, float sig, cudaStream_t st);
};
const WindowOps* radix_window_ops(int n);

// HRTEM imaging from the exit-wave spectrum spec [N][N] (FFT order): the exit wave
// IFFT2(spec)/N^2 (complex64), and the image sum_k w_k |IFFT2(spec .* tf_k)/N^2|^2 (float32).
// work holds `planes` N x N complex64 planes.
Status launch_exit_wave(int n, const float2* spec, float2* work, float2* out, const float2* tw, cudaStream_t st);
Status launch_tcc_image(int n, const float2* spec, const float2* tf, int planes, const double* w, float2* work,
                        float* out, const float2* tw, cudaStream_t st);

// Sum the per-column-block partials in a fixed order: acc[(w*A + a)*depth + pos].  Tiles
// [skip.z0, skip.z0 + skip.nskip) are left out (zero-band tiles: zero or never written).
Status launch_det_reduce(const double* part, int nblk, int aper_num, int items, int item0, int depth,
                         double* acc, cudaStream_t st, TileSkip skip = TileSkip());
// out[i] = sum_w gfsf[w] * acc[w*AD + i], w in ascending order (accumulate_result).
Status launch_combine(const double* acc, const double* gfsf, int w_num, long ad, double* out, cudaStream_t st);

// ---------------------------------------------------------------------------------------------
// Plain path (cuFFT + element-wise kernels)
// ---------------------------------------------------------------------------------------------
Status launch_plain_init(float2* psi, const float2* probe, int h, int w, int items, int item0, int depth,
                         cudaStream_t st);
Status launch_plain_gather_mul(float2* psi, const float2* tslice, int h, int w, int items, int item0,
                               ScanGeom geo, cudaStream_t st);
Status launch_plain_mul(float2* psi, const float2* m, int vol, int items, cudaStream_t st);
Status launch_plain_scale(float2* psi, float s, long total, cudaStream_t st);
// HRTEM on cuFFT: work[k] = spec .* tf[k] for k < planes (vol elements each), and
// out[e] = sum_k w_k |work[k][e] * s|^2 in ascending k (the order of the fused image kernel).
Status launch_plain_tf_mul(float2* work, const float2* spec, const float2* tf, int vol, int planes, cudaStream_t st);
Status launch_plain_image(const float2* work, int planes, const double* w, float s, int vol, float* out,
                          cudaStream_t st);
// CBED: out[h][w] = sum_q gfsf[q] |fftshift(spec_q)|^2 over w_num kept spectra [w_num][h][w] (FP64).
Status launch_cbed_pattern(const float2* spec, const double* gfsf, int w_num, int h, int w, double* out,
                           cudaStream_t st);
Status launch_plain_detect(const float2* psi, const float* masks, int aper_num, int vol, int items,
                           double* part, int nblk, cudaStream_t st);

// Conversions used by the uploader.
Status launch_d2f2(const double* re, const double* im, float2* out, long n, cudaStream_t st);
Status launch_d2f(const double* in, float* out, long n, cudaStream_t st);
Status launch_shift_masks(const double* aper, float* out, int aper_num, int h, int w, int shift,
                          cudaStream_t st);
// complex64 -> bfloat16 pairs (round to nearest even), the storage of the BF16 transmission trial.
Status launch_to_bf16(const float2* in, void* out, long n, cudaStream_t st);

}  // namespace totem
