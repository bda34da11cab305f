// Sessions: the device-resident state of one request (inputs, transmission stack, work buffers
// and results) shared by the one-shot C ABI, the resident-session API and the serving scheduler.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

#include <functional>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace totem {

extern thread_local long long g_h2d_bytes;  // bytes copied host -> device by the current upload

// A growable device buffer.  With ``pool`` set, memory is taken from that pool in stream order on
// ``st`` (cudaMallocFromPoolAsync / cudaFreeAsync), so creating and retiring request state does
// not synchronise the device; otherwise plain cudaMalloc / cudaFree.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
  void release() {
    if (p) {
      if (pool) cudaFreeAsync(p, st);
      else cudaFree(p);
    }
    p = nullptr;
    cap = 0;
  }
  Status ensure(size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (bytes <= cap) return Status::Ok();
    if (inject_alloc_failure()) return Status::Err(TOTEM_ERR_OOM, "injected device allocation failure");
    release();
    if (pool) TOTEM_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool, st));
    else TOTEM_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
    return Status::Ok();
  }
};

template <class T>
Status upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  TOTEM_TRY(b.ensure(v.size() * sizeof(T)));
  if (!v.empty()) TOTEM_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  g_h2d_bytes += (long long)(v.size() * sizeof(T));
  return Status::Ok();
}

// Stage twiddle tables of the shared-memory FFT (a one-entry placeholder for sizes it does not
// handle; those sizes go through cuFFT).
std::vector<float2> twiddles(int n);

// Atom rows of one kind, split into FP64 positions and FP32 coefficients.
struct RowsHost {
  std::vector<double> pos;
  std::vector<float> coef;
  std::vector<float> absorp;
  std::vector<int> beg;
  int ncoef = 0;
  int count = 0;
};

struct RowsDev {
  DevBuf pos, coef, absorp, beg;
  AtomRowsDev view(bool present, bool has_absorp, int ncoef) const {
    AtomRowsDev d;
    if (!present) return d;
    d.pos = pos.as<double>();
    d.coef = coef.as<float>();
    d.absorp = has_absorp ? absorp.as<float>() : nullptr;
    d.beg = beg.as<int>();
    d.ncoef = ncoef;
    return d;
  }
  Status put(const RowsHost& h, cudaStream_t st) {
    TOTEM_TRY(upload(pos, h.pos, st));
    TOTEM_TRY(upload(coef, h.coef, st));
    TOTEM_TRY(upload(absorp, h.absorp, st));
    TOTEM_TRY(upload(beg, h.beg, st));
    return Status::Ok();
  }
};

// Atom rows of one kind grouped by species (identical coefficient and absorptive rows).
struct SpeciesHost {
  std::vector<double> pos;     // [n][2] ordered by (slice, species, row order)
  std::vector<float> coef;     // [species][ncoef]
  std::vector<float> absorp;   // [species][10] (rows with absorptive coefficients)
  std::vector<int> seg_beg;    // [slices + 1]
  std::vector<int> seg;        // [segments][3]: species, first atom, end atom
  int ncoef = 0;
};

struct SpeciesRowsDev {
  DevBuf pos, coef, absorp, seg_beg, seg;
  SpeciesDev view(bool present, bool has_absorp, int ncoef) const {
    SpeciesDev d;
    if (!present) return d;
    d.pos = pos.as<double>();
    d.coef = coef.as<float>();
    d.absorp = has_absorp ? absorp.as<float>() : nullptr;
    d.seg_beg = seg_beg.as<int>();
    d.seg = seg.as<int>();
    d.ncoef = ncoef;
    return d;
  }
  Status put(const SpeciesHost& h, cudaStream_t st) {
    TOTEM_TRY(upload(pos, h.pos, st));
    TOTEM_TRY(upload(coef, h.coef, st));
    TOTEM_TRY(upload(absorp, h.absorp, st));
    TOTEM_TRY(upload(seg_beg, h.seg_beg, st));
    TOTEM_TRY(upload(seg, h.seg, st));
    return Status::Ok();
  }
};

struct PlanKey {
  int h, w, batch;
  bool operator<(const PlanKey& o) const {
    return h != o.h ? h < o.h : (w != o.w ? w < o.w : batch < o.batch);
  }
};

// Detection events of a request: every distinct valid mid-layer slice (first occurrence wins, as
// find(midslice==k, 1) in cuda_STEM_CPU_Mcore_lobato_peng.m:66-67), then the exit wave.
struct DetectionEvents {
  std::vector<int> event_of_slice;  // [slices + 1], 1-based slice -> event or -1
  std::vector<int> layer_event;     // [layer_len], mid layer -> event or -1 (repeat / out of range)
  int n_events = 0;
  int exit_event = 0;
};

}  // namespace totem

struct totem_session {
  using Status = totem::Status;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::mutex mu;

  // request metadata
  bool uploaded = false;
  bool stem_ready = false;  // STEM inputs present (the transmission-only MEX passes none)
  int param = 0, h = 0, w = 0, depth = 0, p_h = 0, p_w = 0, slices = 0, step = 0, begin_row = 0, begin_col = 0,
      width_red = 0, w_num = 0, aper_num = 0;
  double sigma = 0, parameter = 0;
  std::vector<int> mid_layer;
  std::vector<double> gfsf;
  bool separable = false, aper_true_ones = true, has_abs_n = false, has_abs_i = false;
  int n_rows = 0, n_rows_i = 0, n_corr = 0, n_corr_i = 0, cim_len = 0, ncoef_n = 0, ncoef_i = 0;

  // device inputs
  totem::DevBuf probe, prop, mask_mid, mask_exit, tw_n, tw_pw, tw_ph, gfsf_d;
  totem::RowsDev rows_n, rows_i, rows_cn, rows_ci;
  totem::SpeciesRowsDev species_n, species_i;  // the neutral / ionic rows by species (separable grids)
  totem::SpeciesRowsDev species_cn, species_ci;  // the correction rows by species (separable grids)
  // correction rows by species (few distinct rows per slice), or by the per-atom kernel on top
  bool corr_by_species = true;
  // gridding builder (uniform separable axes): job table, deconvolution tables, work memory
  bool grid_ok = false;
  bool grid_scratch_zero = false;  // grid_scratch is as the last gridding build left it, for
  long long grid_scratch_layout = -1;  // that build's grid and jobs per batch
  double grid_dkx = 0, grid_dky = 0, grid_sx = 0, grid_sy = 0;
  long long grid_atoms = 0;
  std::vector<int> grid_job_beg_h;
  std::vector<int4> grid_jobs_h;
  totem::DevBuf grid_jobs, grid_job_beg, grid_ax, grid_ay, grid_scratch;
  totem::DevBuf kx_axis, ky_axis, kx, ky, s2, aper_true, cim;
  // work buffers and results
  totem::DevBuf T, psi, part, acc, out_result, out_mid;
  totem::DevBuf ev_slice;  // device copy of DetectionEvents::event_of_slice (serving scheduler)
  totem::DevBuf Tb;        // the transmission as bfloat16 pairs (TOTEM_T_BF16)
  bool tb_valid = false;
  // HRTEM inputs and outputs
  totem::DevBuf hr_wave, hr_prop, hr_tf, hr_w, hr_work, hr_exit, hr_img;
  totem::DevBuf cbed_out;  // the CBED pattern [H][W] (FP64)
  bool t_valid = false;
  bool has_result = false;
  int last_what = 0;
  std::map<totem::PlanKey, cufftHandle> plans;
  // the fused slice loop of the last run, as a CUDA graph (run_graphed)
  std::vector<long long> graph_key;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_launches = 0;

  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  TotemTiming timing{};
  long long h2d_bytes = 0, d2h_bytes = 0;
  // band of the uploaded propagator (totem::spectral_band; n / 2 and above: no zero band)
  int band = 1 << 30;
  // which implementations the last run used (TotemTiming.slice_path / tx_fft_path / tx_builder)
  int ran_slice_path = -1, ran_tx_fft = -1, ran_tx_builder = -1;
  int used_row_variant = 0, used_col_variant = 0;
  // per-launch profiling of the fused passes (TotemRunOptions.profile)
  bool profiling = false;
  std::vector<cudaEvent_t> pev;
  std::vector<int> pkind;  // 0 = row pass, 1 = column pass
  size_t pused = 0;

  ~totem_session() {
    // buffers first: pool-backed ones are freed in order on ``stream``, which must still exist
    for_each_buf([](totem::DevBuf& b) { b.release(); });
    for (auto& kv : plans) cufftDestroy(kv.second);
    drop_graph();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : pev) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  template <class F>
  void for_each_buf(F&& f) {
    for (totem::DevBuf* b : {&probe, &prop, &mask_mid, &mask_exit, &tw_n, &tw_pw, &tw_ph, &gfsf_d, &kx_axis, &ky_axis,
                             &kx, &ky, &s2, &aper_true, &cim, &T, &psi, &part, &acc, &out_result, &out_mid,
                             &ev_slice, &Tb, &hr_wave, &hr_prop, &hr_tf, &hr_w, &hr_work, &hr_exit, &hr_img, &grid_jobs,
                             &grid_job_beg, &grid_ax, &grid_ay, &grid_scratch})
      f(*b);
    for (totem::RowsDev* r : {&rows_n, &rows_i, &rows_cn, &rows_ci})
      for (totem::DevBuf* b : {&r->pos, &r->coef, &r->absorp, &r->beg}) f(*b);
    for (totem::SpeciesRowsDev* r : {&species_n, &species_i, &species_cn, &species_ci})
      for (totem::DevBuf* b : {&r->pos, &r->coef, &r->absorp, &r->seg_beg, &r->seg}) f(*b);
  }

  // Take every device buffer of this session from ``pool`` in stream order on the session's stream.
  void use_pool(cudaMemPool_t pool) {
    for_each_buf([&](totem::DevBuf& b) {
      b.pool = pool;
      b.st = stream;
    });
  }

  Status prof_begin() {
    if (!profiling) return Status::Ok();
    while (pev.size() < pused + 2) {
      cudaEvent_t e;
      TOTEM_CUDA(cudaEventCreate(&e));
      pev.push_back(e);
    }
    TOTEM_CUDA(cudaEventRecord(pev[pused], stream));
    return Status::Ok();
  }
  Status prof_end(int kind) {
    if (!profiling) return Status::Ok();
    TOTEM_CUDA(cudaEventRecord(pev[pused + 1], stream));
    pkind.push_back(kind);
    pused += 2;
    return Status::Ok();
  }

  Status plan(int ph, int pw, int batch, cufftHandle* out) {
    totem::PlanKey k{ph, pw, batch};
    auto it = plans.find(k);
    if (it != plans.end()) {
      *out = it->second;
      return Status::Ok();
    }
    cufftHandle p;
    int n[2] = {ph, pw};
    TOTEM_CUFFT(cufftPlanMany(&p, 2, n, nullptr, 1, ph * pw, nullptr, 1, ph * pw, CUFFT_C2C, batch));
    TOTEM_CUFFT(cufftSetStream(p, stream));
    plans[k] = p;
    *out = p;
    return Status::Ok();
  }

  // Validation of a request without touching the device (the checks of upload_args).
  static Status validate(const TotemStemArgs* a, bool stem);
  Status upload_args(const TotemStemArgs* a, bool stem);
  Status build_transmission(int path, int* launches);
  Status plan_gridding(const TotemStemArgs* a, const totem::SpeciesHost* const (&kinds)[4]);
  bool gridding_cheaper() const;
  totem::DetectionEvents detection_events() const;
  // Per-event detector sums acc[event][w][A][depth] -> out_result (exit) and out_mid (layers),
  // weighted by gfsf over w (accumulate_result, cuda_source_lobato.cu:981-1015).
  Status combine_results(const totem::DetectionEvents& de, int* launches);
  Status slice_loop(int path, int batch, int col_variant, int t_storage, int* launches, int* batch_used,
                    int row_variant = 0);
  // The transmission slices as the slice loop reads them (complex64, or bfloat16 pairs).
  Status transmission_for(int t_storage, const void** t, size_t* slice_bytes, int* launches);
  Status run_graphed(const std::vector<long long>& key, const std::function<Status()>& enqueue, int* launches);
  void drop_graph();
  Status hrtem(const TotemHrtemArgs* h, TotemHrtemOut* out);
  Status hrtem_plain(const TotemHrtemArgs* hr, TotemHrtemOut* out, const float2* Tp);
  Status cbed(double* pattern);
  Status run(int what, const TotemRunOptions* opt);
  Status collect_timing();
  Status download(TotemStemOut* out);
  bool timing_pending = false;
};

namespace totem {
// Device choice: ``*dev`` >= 0 is checked, -1 picks the device with the most free memory (as
// cuda_source_lobato.cu:1071-1081).
Status pick_device(int* dev);
// A session on ``device`` (-1: pick) using ``stream``, or a new non-blocking stream if null.
Status create_session(int device, void* stream, totem_session** out);
}  // namespace totem
