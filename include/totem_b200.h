/*
 * totem_b200 -- B200-native multislice STEM engine, C ABI.
 *
 * The engine replaces the GPU back end of ToTem's MEX entry points
 *   waveCudalobato_<v>, waveCudaPengAndCorr_<v>        (STEM: cuda_stem.m:83-106)
 *   waveCudalobatoP_<v>, waveCudaPengAndCorrP_<v>      (transmission only: cuda_stem_potential.m)
 * whose MEX shim (waveCuda.cpp:4-101) forwards 41 MATLAB arguments to the C++ function
 *   void myProjectfun(...)                             (waveCuda.h:10-21)
 * implemented by cuda_source_lobato.cu:1018-1562 / cuda_source_peng_and_corr.cu:1217-1786 and,
 * for the transmission-only variants, cuda_source_lobato_potential.cu:747-927 /
 * cuda_source_peng_and_corr_potential.cu:952-1149.
 *
 * Two ways in:
 *   1. ``myProjectfun`` with the reference's exact 44-parameter C++ signature, exported by the
 *      four small libraries libwaveCuda{Lobato,Peng,LobatoP,PengP}.so so that the unchanged
 *      waveCuda.cpp links against them (declared at the end of this header, C++ only).
 *   2. The C entry points below (plain pointers and sizes, status codes, no torch types).
 *
 * Array layouts are the ones ``myProjectfun`` receives: every matrix is row-major with the
 * MATLAB row index first (the MEX caller transposes, cuda_stem.m:22-58); stacks are
 * (count, rows, cols).  All arrays passed in are host memory; a session keeps its uploaded
 * inputs resident on the device between runs.
 */
#ifndef TOTEM_B200_H
#define TOTEM_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define TOTEM_API __attribute__((visibility("default")))
#else
#define TOTEM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define TOTEM_ABI_VERSION 4

/* Status codes.  The reference returns silently or aborts MATLAB (waveCuda.cpp:7-16,
 * cuda_source_lobato.cu:1253-1256); every entry point here returns one of these instead. */
enum {
  TOTEM_OK = 0,
  TOTEM_ERR_INVALID_ARG = 1,   /* a size, pointer or index is out of range            */
  TOTEM_ERR_UNSUPPORTED = 2,   /* valid input this build does not handle (e.g. sizes) */
  TOTEM_ERR_CUDA = 3,          /* a CUDA runtime call failed                          */
  TOTEM_ERR_CUFFT = 4,         /* a cuFFT call failed                                 */
  TOTEM_ERR_OOM = 5,           /* device allocation failed                            */
  TOTEM_ERR_NO_DEVICE = 6,     /* no CUDA device is visible                           */
  TOTEM_ERR_STATE = 7,         /* call sequence error (e.g. run before upload)        */
  TOTEM_ERR_TIMEOUT = 8        /* a wait ended before the request finished            */
};

/* Scattering-factor parameterisation: selects the coefficient-row layout, i.e. which MEX the
 * request targets (cuda_stem.m:83-94). */
enum { TOTEM_PARAM_PENG = 0,   /* rows of 13 (neutral) / 25 (ionic) columns */
       TOTEM_PARAM_LOBATO = 1  /* rows of 14 / 26 columns                     */ };

/* Slice-loop implementation.  TOTEM_PATH_FUSED runs the hand-written kernels where they apply
 * (square windows of 64..2048 for the slice loop: powers of two and the mixed-radix edges 96, 160,
 * 192, 288, 320, 384, 400, 448, 576, 640, 768, 800, 1152, 1280, 1536, 1600; potential grids of
 * 64..4096 whose edges are powers of two or those mixed-radix edges, in whole row and column tiles,
 * for the transmission FFT) and cuFFT elsewhere; TotemTiming reports what ran.
 * TOTEM_PATH_FUSED_ONLY fails with TOTEM_ERR_UNSUPPORTED instead of using cuFFT. */
enum { TOTEM_PATH_FUSED = 0,      /* shared-memory FFT passes fused with the multiplies and detectors */
       TOTEM_PATH_PLAIN = 1,      /* cuFFT plus separate element-wise kernels (comparator)           */
       TOTEM_PATH_FUSED_ONLY = 2  /* the fused kernels or an error, never cuFFT                     */ };

/*
 * The inputs of myProjectfun (waveCuda.h:10-21), one field per parameter, same meaning.
 */
typedef struct TotemStemArgs {
  int struct_size;                 /* sizeof(TotemStemArgs)                                    */
  int param;                       /* TOTEM_PARAM_*                                            */

  const double *probe_re, *probe_im; /* w_num x height x width (prhs[0..1])                    */
  const double *aper;              /* aper_num x height x width, centred masks (prhs[2])       */
  const double *atom_slice;        /* slices: neutral rows per slice (prhs[3], series_n)       */
  const double *absorp_n;          /* rows x 10 absorptive coefficients or NULL (prhs[4])      */
  const double *atom_slice_i;      /* slices: ionic rows per slice (prhs[5])                   */
  const double *absorp_n_i;        /* or NULL (prhs[6])                                        */
  const double *proj_coff_mat;     /* neutral rows x 13|14 (prhs[7])                           */
  const double *proj_coff_mat_i;   /* ionic rows x 25|26 (prhs[8])                             */
  const double *kx, *ky, *s_2;     /* p_height x p_width (prhs[9..11])                         */
  const double *prop_re, *prop_im; /* height x width Fresnel propagator, FFT order (prhs[12..13]) */
  const double *gfsf;              /* w_num weights (prhs[14])                                 */
  int height, width, depth;        /* window rows, cols; scan positions (prhs[15..17])         */
  int p_height, p_width, slices;   /* potential grid and slice count (prhs[18..20])            */
  int step;                        /* scan step in pixels (prhs[21])                           */
  int begin_row, begin_col;        /* 0-based window origin (prhs[22..23] minus one)           */
  int width_red;                   /* scan positions per scan row (prhs[24])                   */
  double sigma;                    /* interaction constant, 1/(kV*A) (prhs[25])               */
  int w_num, aper_num;             /* probes (defocus spread) and detectors (prhs[26..27])     */
  double parameter;                /* PARAMETER (prhs[28])                                     */
  const double *aper_true;         /* p_height x p_width multiplier of V(g) (prhs[29])         */
  const int *mid_layer;            /* 1-based slice indices (prhs[32])                         */
  int layer_len;                   /* (prhs[33])                                               */
  const double *aper2;             /* aper_num x height x width, ifftshift(aper) (prhs[34])    */
  const double *series_n_corr;     /* slices or NULL (prhs[35])                                */
  const double *series_n_i_corr;   /* slices or NULL (prhs[36])                                */
  const double *ele_n_corr;        /* rows x 5 (prhs[37])                                      */
  const double *ele_n_i_corr;      /* rows x 8 (prhs[38])                                      */
  const double *corr_info_matrix;  /* cim_len x p_height x p_width (prhs[39])                  */
  int cim_len;                     /* (prhs[40])                                               */
} TotemStemArgs;

/* Outputs (plhs[0..3] of waveCuda.cpp:85-92).  NULL pointers are skipped. */
typedef struct TotemStemOut {
  double *result;                  /* aper_num*depth, result[a*depth + pos]                    */
  double *mid_layer_mat;           /* depth*aper_num*layer_len, [(l*aper_num + a)*depth + pos]  */
  double *potential_re;            /* p_height*p_width*slices, transmission (the *P variants)  */
  double *potential_im;
} TotemStemOut;

/* Storage of the transmission stack read by the slice loop. */
enum {
  TOTEM_T_COMPLEX64 = 0,         /* FP32 re/im (the reference's layout)                          */
  TOTEM_T_BF16 = 1               /* bfloat16 re/im: half the bytes per slice, ~3 significant digits;
                                    a precision trial, outside the 1e-4 parity bound            */
};

/* Engine options of one run (defaults: all zero). */
typedef struct TotemRunOptions {
  int path;                        /* TOTEM_PATH_*                                              */
  int batch;                       /* probes in flight per batch, 0 = the tuned choice (else up to
                                      4 GiB of waves for the fused path, 1 GiB for cuFFT)         */
  int skip_transmission;           /* 1 = reuse the transmission built by an earlier run        */
  int profile;                     /* 1 = CUDA events around every slice-loop pass launch       */
  int col_variant;                 /* fused column pass: 0 = the tuned choice for this window and
                                      GPU (totem_load_tuning), else 1; 1 = built-in default
                                      (propagator read from L2, 16-column tiles up to N = 512,
                                      8 above), 2 = propagator prefetched to shared memory,
                                      3 = 80-register cap (more resident CTAs), 5 = 8-column tiles,
                                      6 = 32-column tiles (N <= 512)                             */
  int t_storage;                   /* TOTEM_T_* (fused path only)                                */
  int row_variant;                 /* fused row pass: 0 = the tuned choice, else 1; 1 = built-in
                                      default; 3, 4, 5 = registers sized for that many resident
                                      128-thread CTAs per SM (3: N >= 1024, 5: N <= 1024)         */
} TotemRunOptions;

/* Device times (CUDA events) of the last run, milliseconds. */
typedef struct TotemTiming {
  float transmission_ms;
  float slice_loop_ms;
  float total_ms;
  int kernel_launches;             /* kernels this engine launched in the run                  */
  int batch;                       /* batch size used                                          */
  /* profile = 1 only: summed device time and launch count of the fused passes */
  float row_pass_ms, col_pass_ms;
  int row_pass_launches, col_pass_launches;
  long long probe_slices;          /* probes x slices advanced by the run                      */
  long long h2d_bytes, d2h_bytes;  /* host<->device bytes of the last upload / download        */
  /* what ran (-1 = that stage did not run): */
  int slice_path;                  /* TOTEM_PATH_FUSED or TOTEM_PATH_PLAIN (cuFFT)               */
  int tx_fft_path;                 /* transmission inverse FFT: TOTEM_PATH_FUSED or _PLAIN (cuFFT) */
  int tx_builder;                  /* TOTEM_TX_DIRECT, TOTEM_TX_GRIDDING or TOTEM_TX_ROWS          */
  int row_variant, col_variant;    /* fused pass variants used (after the tuning table)          */
} TotemTiming;

typedef struct totem_session totem_session;

TOTEM_API int totem_abi_version(void);
/* Measured FP32 FMA throughput of GPU ``device`` in TFLOP/s (2 flops per FMA): chains of scalar
 * FFMA and of packed FFMA2 (two FMAs per instruction), 8 independent chains per thread at full
 * occupancy, the best of 3 CUDA-event-timed launches after a warm-up (a few ms each).  The
 * compute-side ceiling of the fused passes, reported beside the HBM roofline. */
TOTEM_API int totem_fp32_peak(int device, double *ffma_tflops, double *ffma2_tflops);
TOTEM_API const char *totem_status_string(int status);
/* Message describing the last failure on the calling thread ("" if none). */
TOTEM_API const char *totem_last_error(void);

/* A session owns device buffers on one GPU and keeps them between calls.  ``device`` = -1
 * selects the GPU with the most free memory, as the reference does
 * (cuda_source_lobato.cu:1071-1081).  ``stream`` is a cudaStream_t (NULL = the session makes one). */
TOTEM_API int totem_session_create(int device, void *stream, totem_session **out);
TOTEM_API int totem_session_destroy(totem_session *s);
/* Copy (or, for TOTEM_MEM_DEVICE, adopt) the request's inputs and validate them. */
TOTEM_API int totem_session_upload(totem_session *s, const TotemStemArgs *args);
/* Device work only: transmission build, slice loop, detector reduction.  Results stay on the
 * device.  ``what`` = 0: STEM; 1: transmission only.  Asynchronous on the session's stream. */
TOTEM_API int totem_session_run(totem_session *s, int what, const TotemRunOptions *opt);
/* Wait for the stream and copy results into ``out`` (host pointers). */
TOTEM_API int totem_session_download(totem_session *s, TotemStemOut *out);
TOTEM_API int totem_session_timing(totem_session *s, TotemTiming *t);
/* Device pointer of the transmission stack (complex64, slices x p_height x p_width). */
TOTEM_API int totem_session_transmission(totem_session *s, void **ptr);

/* One call with host buffers: the semantics of the STEM MEX (result, mid_layer_mat).
 * Replaces myProjectfun in cuda_source_lobato.cu:1018 / cuda_source_peng_and_corr.cu:1217. */
TOTEM_API int totem_stem_run(const TotemStemArgs *args, const TotemRunOptions *opt, TotemStemOut *out);
/* One call with host buffers: the semantics of the *P MEX (potential_re/im = Re/Im of the
 * transmission exp(i sigma V / 1000)).  Replaces cuda_source_lobato_potential.cu:747. */
TOTEM_API int totem_transmission_run(const TotemStemArgs *args, TotemStemOut *out);

/* How the neutral and ionic potential sums are formed on separable reciprocal grids (the
 * reference's meshgrid layout).  Process-wide; later transmission builds use it.  No
 * counterpart in the reference, whose cal_p sums every atom at every pixel.
 *   TOTEM_TX_AUTO      the cheaper of the two by a cost model (default)
 *   TOTEM_TX_DIRECT    per-species sums over atoms at every pixel: O(atoms x pixels)
 *   TOTEM_TX_GRIDDING  Gaussian gridding onto a twice-finer grid and FFTs (a non-uniform FFT):
 *                      O(atoms + pixels log pixels), relative error ~1e-7; used where the axes
 *                      are uniform and the grid is a power of two from 64 to 4096, otherwise
 *                      DIRECT is used.
 * ``scratch_bytes`` bounds the gridding work memory taken during a build (0 = 1 GiB); at least
 * one species plane set (64 bytes per potential pixel) is always taken. */
#define TOTEM_TX_AUTO 0
#define TOTEM_TX_DIRECT 1
#define TOTEM_TX_GRIDDING 2
/* Reported in TotemTiming.tx_builder only: one thread per pixel and atom row (reciprocal grids
 * that are not the separable meshgrid). */
#define TOTEM_TX_ROWS 3
TOTEM_API int totem_set_tx_builder(int mode, size_t scratch_bytes);
/* Repeated runs of a session's fused slice loop with the same shapes and buffers replay as one
 * CUDA graph (captured on the second such run): 1 = on (default), 0 = off.  Process-wide; no
 * counterpart in the reference.  Runs on the legacy default stream, or on a stream the caller is
 * capturing, are never graphed. */
TOTEM_API int totem_set_slice_graphs(int enable);
/* The fused slice loop skips the wave's columns on which the propagator is zero in every row
 * (beyond the 2/3-of-Nyquist cut of the reference's propagator, ToTEM_submit_v1.m:1558-1564, about
 * a third of them; half with the HRTEM 1/2 cut): after the column pass multiplies by the
 * propagator they are zero whatever the wave was, so they are neither read, transformed nor
 * written, and the detector sums leave out their (zero) contributions.  The band is found from
 * the propagator the caller passes; results equal those with every column computed.  1 = on
 * (default), 0 = off.  Process-wide; no counterpart in the reference. */
TOTEM_API int totem_set_band_skip(int enable);
/* Failure injection on the host, for tests of the error paths (no GPU fault is involved): after
 * ``alloc_after`` further device allocations of the engine the next one fails once with
 * TOTEM_ERR_OOM, as if the device were full (-1 = off); every ``prepare_every``-th request a server
 * prepares fails in its preparation with TOTEM_ERR_STATE before it touches the device (0 = off).
 * Process-wide; each call resets the counts.  No counterpart in the reference. */
TOTEM_API int totem_inject_failures(long long alloc_after, int prepare_every);
/* Launch shapes chosen by measurement (python -m totem_b200.tune writes the table): one JSON
 * object per line, {"device": "<cudaDeviceProp.name>", "n": <window edge>, "row_variant": r,
 * "col_variant": c, "batch_mib": b, ...}.  Runs whose TotemRunOptions leave row_variant,
 * col_variant or batch at 0 use the entry of their GPU and window, and the built-in defaults where
 * there is none.  The library loads totem_b200/data/tuning.jsonl beside its lib/ directory on first
 * use (or the file named by TOTEM_TUNING_FILE); this call replaces the table with ``path`` (NULL
 * or "" = no table: built-in defaults).  ``entries`` receives the number of entries read.
 * Process-wide; no counterpart in the reference, which sizes its batch from free memory
 * (cuda_source_lobato.cu:1250-1260). */
TOTEM_API int totem_load_tuning(const char *path, int *entries);
/* The launch shapes a fused run on ``device`` with an n x n window would use by default. */
TOTEM_API int totem_tuned_config(int device, int n, int *row_variant, int *col_variant, long long *batch_bytes);
/* The gridding builder's batch plan, without a device (tests): jobs are numbered in slice order,
 * slice s owning jobs [job_beg[s], job_beg[s+1]); at most jobs_per_batch jobs run per batch.
 * Writes up to max_batches rows (s_lo, s_hi, j_lo, j_hi) to ``out`` and the batch count to
 * ``count``: batch b runs jobs [j_lo, j_hi) and writes slices [s_lo, s_hi), adding to a slice
 * whose first job ran in an earlier batch. */
TOTEM_API int totem_grid_batches(const int *job_beg, int slices, int jobs_per_batch, int *out, int max_batches,
                                 int *count);

/*
 * Specimen preparation (host only, no device needed): the coefficient rows above from atom
 * tables, as ToTem's MATLAB prepares them.
 *
 * Tables, one row per atom (getpotentialpara_lotabo_peng.m:26-84):
 *   nuclear, 16 columns: Z x y z B occ a1 b1 .. a5 b5
 *   nuc_ion, 28 columns: Z x y z B occ f_ion a1 b1 .. a5 b5 (ion) f_atom a1 b1 .. a5 b5 (atom)
 *
 * totem_slice_rows: slice assignment with erf weights; replaces
 * CalAllEquilent20210223_lobato_peng.m:23-228.  Slice i spans slicethick[i] .. + eachthick; an
 * atom within multiceng slices of it adds the share of its projected potential that falls inside
 * (|erf(2 pi z2/sqrt(b))/2 - erf(2 pi z1/sqrt(b))/2| on every a_i).  Writes the rows
 * (13/14 or 25/26 columns, TOTEM_PARAM_* layout; Lobato rows end with B * dbmode) slice by slice
 * into ele_n / ele_n_i (capacity cap_n / cap_i rows; NULL to count only), the per-slice counts
 * into series_n / series_n_i (slices entries each, or NULL), and the row totals into rows_n /
 * rows_i.  Returns TOTEM_ERR_INVALID_ARG when a capacity is too small (the totals are still set).
 */
TOTEM_API int totem_slice_rows(int param, const double *nuclear, int n_nuclear, const double *nuc_ion, int n_ion,
                               double eachthick, const double *slicethick, int slices, int multiceng, int dbmode,
                               double *ele_n, long long cap_n, double *ele_n_i, long long cap_i, double *series_n,
                               double *series_n_i, long long *rows_n, long long *rows_i);
/* Debye-Waller B added to every Peng b_i, in place (CommonPart_forsimulation_lobato_peng.m:88-110);
 * Lobato tables are left as they are (the engine applies exp(-B s^2) from the row's last column). */
TOTEM_API int totem_fold_debye_waller(int param, double *nuclear, int n_nuclear, double *nuc_ion, int n_ion);
/* One frozen-phonon configuration (randshiftpos.m:1-44): x, y, z (columns 1-3) of every row of
 * an n x ncol table displaced by normal deviates of sigma = sqrt(B / 8 pi^2) (B in column 4),
 * whole positions re-drawn while z leaves [slicethick[0], slicethick[slices-1] + eachthick).
 * The deviates are a function of (seed, row, draw): a configuration is reproducible from its
 * seed (the reference uses rng('shuffle')).  An atom still outside after 100 000 draws is an
 * error. */
TOTEM_API int totem_frozen_phonon(const double *table, int n, int ncol, double eachthick, const double *slicethick,
                                  int slices, unsigned long long seed, double *out);

/* Size of the fixed device scratch array used by totem_stem_slices_noalloc (per GPU). */
#define TOTEM_NOALLOC_SCRATCH_BYTES (32ull << 20)

/*
 * Slice loop and exit detectors without any device allocation.  This entry point has no
 * counterpart in the reference; it exists for callers that cannot allocate device memory:
 * code whose GPU memory belongs to a host framework's pool (a MEX function under MATLAB's GPU
 * memory manager, an operator in a PyTorch pipeline that must not bypass its caching
 * allocator), latency-bound serving loops that cannot pay for cudaMalloc / cudaFree (both
 * synchronise the device and stall other streams), and deployments with a fixed memory budget.
 *
 * All pointers are device memory owned by the caller: transmission complex64
 * [slices][p_height][p_width]; probe complex64 [w_num][n][n]; propagator complex64 [n][n] in FFT
 * order; masks float32 [aper_num][n][n] in FFT order (ifftshift of the centred detector masks);
 * result float64 [aper_num][items] receives sum |Psi|^2 * mask for items item0 .. item0+items-1,
 * item = w * depth + pos, with the window of pos placed as in TotemStemArgs.  No gfsf weighting.
 *
 * Intermediate buffers live in one fixed device array of TOTEM_NOALLOC_SCRATCH_BYTES (32 MiB)
 * that the library holds on every GPU that loads it until the process exits; a request that
 * needs more (about 15 probes of 512^2 per call) fails with TOTEM_ERR_INVALID_ARG and a message
 * (totem_last_error) giving the largest batch that fits.  The first call on a device performs a
 * one-time set-up with that device current (the array's device address and a blocking copy of
 * FFT twiddle tables into it); make that first call before any stream capture.  The set-up
 * belongs to the device's current CUDA context and is repeated when another context becomes
 * current (after cudaDeviceReset, or under a caller's own driver-API context), so the first call
 * after such a change must also come before any capture.  Every call shares the array: calls that
 * overlap on the GPU race; calls ordered on one stream do not.  n must be a power of two in
 * [64, 1024] (a single 2048^2 probe would need the whole array) and slices >= 1.  Asynchronous on
 * ``stream``.
 */
TOTEM_API int totem_stem_slices_noalloc(const void *transmission, int p_height, int p_width, int slices,
                                        const void *probe, int w_num, const void *propagator, const float *masks,
                                        int aper_num, int n, int step, int begin_row, int begin_col, int width_red,
                                        int depth, int item0, int items, double *result, void *stream);

/* ---------------------------------------------------------------------------------------------
 * HRTEM: plane-wave multislice over the whole potential grid, exit wave and partially coherent
 * image.  The reference builds the transmission with the *P MEX and runs this part in MATLAB
 * (ToTEM_submit_v1.m:1259-1369):  psi = incident wave;  per slice  psi = ifft2(fft2(psi .* T_k)
 * .* psf_fft);  exit wave = psi;  image = sum_k gfsf_k |ifft2(fft2(psi) .* tf_k)|^2 with
 * tf_k = ifftshift(tcc_k .* aperture).  The grid must be square (the reference squares the
 * potential grid, ToTEM_submit_v1.m:1240-1242).  Edges the fused slice loop takes (TOTEM_PATH_FUSED)
 * run the fused passes, every other edge cuFFT; totem_session_timing's slice_path says which.  The
 * bfloat16 transmission trial (t_storage TOTEM_T_BF16) needs a power-of-two edge of 64..2048.
 * ------------------------------------------------------------------------------------------- */
typedef struct TotemHrtemArgs {
  int struct_size;               /* sizeof(TotemHrtemArgs)                                     */
  const double *wave_re;         /* incident wave [P_H][P_W]; both NULL = plane wave of 1      */
  const double *wave_im;
  const double *prop_re;         /* propagator psf_fft [P_H][P_W], FFT order (:1330-1334)      */
  const double *prop_im;
  int defoci;                    /* transfer functions of the image; 0 = exit wave only        */
  const double *tf_re;           /* [defoci][P_H][P_W], FFT order                              */
  const double *tf_im;
  const double *weights;         /* [defoci] (gfsf)                                            */
  int t_storage;                 /* TOTEM_T_*                                                  */
} TotemHrtemArgs;

typedef struct TotemHrtemOut {
  double *exit_re;               /* [P_H][P_W] exit wave, or NULL                              */
  double *exit_im;
  double *image;                 /* [P_H][P_W] image, or NULL                                  */
} TotemHrtemOut;

/* HRTEM on the specimen uploaded to ``s`` (totem_session_upload; its transmission is built if
 * the session has none).  Synchronous: the outputs are filled on return. */
TOTEM_API int totem_session_hrtem(totem_session *s, const TotemHrtemArgs *h, TotemHrtemOut *out);
/* One-shot HRTEM: the specimen fields of ``specimen`` (probe, window and detector fields unused). */
TOTEM_API int totem_hrtem_run(const TotemStemArgs *specimen, const TotemHrtemArgs *h, TotemHrtemOut *out);

/* ---------------------------------------------------------------------------------------------
 * CBED: the convergent-beam diffraction pattern of one probe position.  The reference builds the
 * transmission with the *P MEX and runs this part in MATLAB (ToTEM_submit_v1.m:1478-1492): per
 * defocus probe n, psi = probe_n; per slice psi = ifft2(fft2(psi .* T_k[window]) .* psf_fft);
 * pattern = sum_n gfsf_n |fftshift(fft2(psi))|^2.  The request is a STEM request with depth 1: the
 * probes (w_num), the propagator, gfsf and the window origin begin_row / begin_col (0-based) are
 * used; the detector fields are not (aper_num may be 0).  ``pattern`` receives height x width
 * doubles, row-major, zero frequency at the centre.  Windows of the fused slice loop run the fused
 * passes, other windows cuFFT; totem_session_timing's slice_path says which.
 * ------------------------------------------------------------------------------------------- */
TOTEM_API int totem_session_cbed(totem_session *s, double *pattern);
TOTEM_API int totem_cbed_run(const TotemStemArgs *request, double *pattern);

/* ---------------------------------------------------------------------------------------------
 * Probe / image transfer functions (WholeTCC2D_newTEM, ToTEM_submit_v1.m:2305-2406), evaluated on
 * the current device in FP64.  The reference computes them in MATLAB for every request.
 * ------------------------------------------------------------------------------------------- */
typedef struct TotemAberrations {  /* magnitudes in nm, angles in degrees as entered in ToTem */
  int struct_size;                 /* sizeof(TotemAberrations)                                 */
  double focus;                    /* C1 */
  double A1, phiA1, A2, phiA2, B2, phiB2;
  double Cs;                       /* C3 */
  double A3, phiA3, S3, phiS3, A4, phiA4, D4, phiD4, B4, phiB4, A5, phiA5;
  double C5;
  double S5, phiS5, D5, phiD5;
} TotemAberrations;

/* tcc[m][r][c] (centred grid, m = 0 .. steps-1) = E_s * E_f,m * exp(-i chi): chi from the
 * aberrations to 5th order, the spatial envelope E_s of semi-angle alpha with the aberration
 * gradient (with_gradient = 1, the reference's flag 2) or C1 alone, and focal-spread step m at
 * (m + 1 - (steps + 1)/2) * delta_nm (Gaussian_focal gives delta and the weights).  lambda_nm is
 * the electron wavelength; sampling_a the pixel size in Angstrom. */
TOTEM_API int totem_tcc_stack(const TotemAberrations *ab, double lambda_nm, int n, double sampling_a,
                              double alpha_mrad, int with_gradient, int steps, double delta_nm, double *tcc_re,
                              double *tcc_im);

/* ---------------------------------------------------------------------------------------------
 * Serving: a resident scheduler with continuous batching.  No counterpart in the reference,
 * whose entry point runs one blocking request at a time and allocates / frees everything per
 * call (waveCuda.cpp:4-101, cuda_source_lobato.cu:1018-1562).
 *
 * Requests are queued by totem_server_submit and run asynchronously:
 *   1. admission: a request waits until its resident footprint (transmission stack, probe,
 *      propagator, masks, coefficient rows, detector sums) fits in the budget;
 *   2. preparation (own stream, concurrent with running requests): upload and transmission build;
 *   3. slice loop: every tick advances all running probe groups by one slice, in one row-pass and
 *      one column-pass launch per window size.  Groups of probes from any number of requests, each
 *      at its own slice, share those launches, so a request's probes start as soon as wave memory
 *      is free and small requests run in the gaps of large ones;
 *   4. completion: detector sums are combined and copied into the caller's TotemStemOut buffers.
 * Results are bit-identical to totem_stem_run on the same request (same kernels, same fixed
 * summation order), whatever else runs at the same time.
 *
 * The caller keeps every buffer of ``args`` and ``out`` alive and unmodified until the request is
 * done (totem_server_wait returned or totem_server_info reports DONE / FAILED).  Only the fused
 * path is served: the window must be square, of an edge the fused slice loop takes (see
 * TOTEM_PATH_FUSED), and slices >= 1.
 * ------------------------------------------------------------------------------------------- */
typedef struct totem_server totem_server;

enum {
  TOTEM_SCHED_FIFO = 0,          /* wave memory goes to prepared requests in arrival (ticket)
                                    order; one still being prepared does not hold back a later
                                    one that is ready                                          */
  TOTEM_SCHED_SHORTEST = 1       /* ... to the request with the least remaining work first, and
                                    preparation takes the cheapest queued request first         */
};

typedef struct TotemServerOptions {
  int struct_size;               /* sizeof(TotemServerOptions)                                 */
  int device;                    /* CUDA device; -1 = the one with the most free memory        */
  unsigned long long hbm_budget; /* device bytes for all requests; 0 = 90 % of free memory     */
  unsigned long long wave_bytes; /* of which for probe waves in flight (psi and detector
                                    partial sums); 0 = min(1 GiB, hbm_budget / 4).  It bounds
                                    the duration of a tick, hence the slice-loop latency of a
                                    small request running beside large ones                   */
  unsigned long long chunk_bytes;/* wave bytes one request may claim per tick; 0 = wave_bytes/4 */
  int ticks_ahead;               /* slice steps queued ahead of the GPU; 0 = 4                 */
  int policy;                    /* TOTEM_SCHED_*                                              */
  int prep_threads;              /* host threads preparing requests (upload, transmission);
                                    0 = 2                                                      */
  int mixed_windows;             /* 1 = at a tick with groups of more than one of the window
                                    sizes 256^2, 512^2, 1024^2, all of them go through one
                                    persistent row-pass and one column-pass launch whose CTAs
                                    take tiles of any of these sizes from a queue; 0 = one launch
                                    pair per window size.  Results are the same either way      */
} TotemServerOptions;

enum {
  TOTEM_REQ_QUEUED = 0,          /* waiting for memory                                         */
  TOTEM_REQ_PREPARING = 1,       /* upload and transmission build                              */
  TOTEM_REQ_RUNNING = 2,         /* in the slice loop                                          */
  TOTEM_REQ_DONE = 3,            /* results are in the caller's buffers                        */
  TOTEM_REQ_FAILED = 4           /* see TotemRequestInfo.status and totem_server_info's message */
};

typedef struct TotemRequestInfo {
  int state;                     /* TOTEM_REQ_*                                                */
  int status;                    /* TOTEM_OK, or the error of a failed request                 */
  double queued_ms;              /* submit -> admission                                        */
  double prepare_ms;             /* admission -> transmission ready                            */
  double run_ms;                 /* transmission ready -> results in the caller's buffers      */
  double latency_ms;             /* submit -> results in the caller's buffers                  */
  long long probe_slices;        /* w_num * depth * slices                                     */
} TotemRequestInfo;

/* Scheduler counters since totem_server_create. */
typedef struct TotemServerStats {
  long long ticks;               /* slice steps issued                                          */
  long long probe_slices;        /* probe-slices advanced by them                                */
  long long launches;            /* kernels the tick loop launched                               */
  long long groups;              /* probe groups started                                         */
  long long requests_done;
  double issue_ms;               /* scheduler thread time spent issuing ticks                    */
  double throttle_ms;            /* ... waiting for the device (ticks_ahead ticks in flight)     */
  double idle_ms;                /* ... with nothing to run                                      */
} TotemServerStats;

TOTEM_API int totem_server_create(const TotemServerOptions *opt, totem_server **out);
/* Validates the request (same checks and codes as totem_stem_run) and queues it. */
TOTEM_API int totem_server_submit(totem_server *s, const TotemStemArgs *args, TotemStemOut *out,
                                  unsigned long long *ticket);
/* Blocks until the request is done or failed (returns its status) or timeout_ms passes
 * (TOTEM_ERR_TIMEOUT; timeout_ms < 0 waits without limit). */
TOTEM_API int totem_server_wait(totem_server *s, unsigned long long ticket, int timeout_ms);
TOTEM_API int totem_server_info(totem_server *s, unsigned long long ticket, TotemRequestInfo *info);
TOTEM_API int totem_server_stats(totem_server *s, TotemServerStats *stats);
/* Finishes every queued request, then releases the device state. */
TOTEM_API int totem_server_destroy(totem_server *s);

/* The scheduler's admission policy run without a device, for tests and capacity planning:
 * request i (window n[i], items[i] = w_num * depth probes, slices[i]) becomes ready at tick
 * arrive[i]; a probe takes n*n*8 bytes of wave memory.  Outputs the tick of each request's first
 * slice and of its last slice, and the largest wave memory in flight at any tick. */
TOTEM_API int totem_plan_simulate(int count, const int *n, const long long *items, const int *slices,
                                  const int *arrive, unsigned long long wave_bytes,
                                  unsigned long long chunk_bytes, int policy, int *first_tick, int *done_tick,
                                  unsigned long long *max_inflight);

#ifdef __cplusplus
} /* extern "C" */

/* The reference's own entry point, C++ linkage, exact signature of waveCuda.h:10-21.
 * Exported by libwaveCudaLobato.so / libwaveCudaPeng.so (STEM) and libwaveCudaLobatoP.so /
 * libwaveCudaPengP.so (transmission only). */
TOTEM_API void myProjectfun(double *my_real_w, double *my_imag_w, double *aper,
                  double *atom_slice, double *absorp_n, double *atom_slice_i,
                  double *absorp_n_i, double *proj_coff_mat, double *proj_coff_mat_i,
                  double *kx, double *ky, double *s_2, double *my_real_const,
                  double *my_img_const, double *gfsf, int Height, int Width, int Depth,
                  int P_Height, int P_Width, int Slices, int step, int beginRow, int beginCol,
                  int width_red, double sigma, int w_num, int aper_num, double parameter,
                  double *AperTrue, int *mid_ceng, int ceng_len, double *aper2,
                  double *series_n_corr, double *series_n_i_corr,
                  double *ele_n_corr, double *ele_n_i_corr,
                  double *corr_info_matrix, int cim_len,
                  double *return_result, double *mid_ceng_mat, double *potentialx, double *potentialy);
#endif

#endif /* TOTEM_B200_H */
