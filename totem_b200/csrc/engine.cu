// Engine runtime: sessions, request validation and upload, orchestration of the transmission
// builder and the slice loop, and the C ABI declared in include/totem_b200.h.
//
// Reference orchestrator: myProjectfun (cuda_source_lobato.cu:1018-1562,
// cuda_source_peng_and_corr.cu:1217-1786).  Differences by design:
//  * device buffers live in a session and are reused across calls (the reference allocates and
//    frees everything per call, several buffers per slice);
//  * no host synchronisation inside the loop, cuFFT plans are created once and cached;
//  * probes run in batches sized for the L2 cache instead of for half the free memory
//    (cuda_source_lobato.cu:1250);
//  * every CUDA / cuFFT status is checked and returned as a TOTEM_ERR_* code.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <fstream>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "session.h"

using totem::Status;
using totem::DevBuf;
using totem::RowsHost;
using totem::PlanKey;
using totem::twiddles;
using totem::upload;
using totem::g_h2d_bytes;

namespace {

thread_local std::string g_last_error;
std::atomic<int> g_tx_mode{TOTEM_TX_AUTO};
std::atomic<int> g_slice_graphs{1};
std::atomic<int> g_band_skip{1};
std::atomic<long long> g_fail_alloc_after{-1};  // allocations to let through before one fails; -1 off
std::atomic<long long> g_fail_prepare_every{0};  // every k-th server preparation fails; 0 off
std::atomic<long long> g_prepares{0};
std::atomic<size_t> g_tx_scratch{0};

int fail(const Status& s) {
  g_last_error = s.msg;
  return s.code;
}

// ---------------------------------------------------------------------------------------------
// Tuning table: launch shapes per (GPU name, window edge), measured by python -m totem_b200.tune
// ---------------------------------------------------------------------------------------------
struct TuneEntry {
  std::string device;
  int n = 0;
  int row_variant = 0, col_variant = 0;
  long long batch_bytes = 0;
};
std::mutex g_tune_mu;
bool g_tune_loaded = false;
std::vector<TuneEntry> g_tune;

// The value of "key" in one line of the table (a flat JSON object of numbers and strings).
bool json_field(const std::string& line, const char* key, std::string* out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = line.find(k);
  if (p == std::string::npos) return false;
  p = line.find(':', p + k.size());
  if (p == std::string::npos) return false;
  ++p;
  while (p < line.size() && std::isspace((unsigned char)line[p])) ++p;
  if (p < line.size() && line[p] == '"') {
    const size_t e = line.find('"', p + 1);
    if (e == std::string::npos) return false;
    *out = line.substr(p + 1, e - p - 1);
    return true;
  }
  size_t e = p;
  while (e < line.size() && line[e] != ',' && line[e] != '}' && !std::isspace((unsigned char)line[e])) ++e;
  *out = line.substr(p, e - p);
  return !out->empty();
}

Status read_tuning(const std::string& path, std::vector<TuneEntry>* out) {
  std::ifstream f(path);
  if (!f) return Status::Err(TOTEM_ERR_INVALID_ARG, "cannot open the tuning table " + path);
  std::string line, v;
  int lineno = 0;
  while (std::getline(f, line)) {
    ++lineno;
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    TuneEntry e;
    if (!json_field(line, "device", &e.device) || !json_field(line, "n", &v))
      return Status::Err(TOTEM_ERR_INVALID_ARG, path + ":" + std::to_string(lineno) + ": no \"device\" or \"n\"");
    e.n = std::atoi(v.c_str());
    if (json_field(line, "row_variant", &v)) e.row_variant = std::atoi(v.c_str());
    if (json_field(line, "col_variant", &v)) e.col_variant = std::atoi(v.c_str());
    if (json_field(line, "batch_mib", &v)) e.batch_bytes = (long long)(std::atof(v.c_str()) * 1048576.0);
    if (e.n <= 0 || e.row_variant < 0 || e.col_variant < 0 || e.batch_bytes < 0)
      return Status::Err(TOTEM_ERR_INVALID_ARG, path + ":" + std::to_string(lineno) + ": invalid entry");
    out->push_back(e);
  }
  return Status::Ok();
}

// TOTEM_TUNING_FILE, else data/tuning.jsonl beside the directory this library was loaded from.
std::string default_tuning_path() {
  if (const char* e = std::getenv("TOTEM_TUNING_FILE")) return e;
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&default_tuning_path), &info) && info.dli_fname) {
    std::string lib(info.dli_fname);
    const size_t slash = lib.rfind('/');
    return (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/../data/tuning.jsonl";
  }
  return "";
}

// Entry for (device, n); the default table is read on first use (missing or unreadable: none).
bool tuned_entry(int device, int n, TuneEntry* out) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (!g_tune_loaded) {
    g_tune_loaded = true;
    std::vector<TuneEntry> t;
    const std::string path = default_tuning_path();
    if (!path.empty() && read_tuning(path, &t).ok()) g_tune = std::move(t);
  }
  if (g_tune.empty()) return false;
  static std::map<int, std::string> names;  // device -> cudaDeviceProp::name (under g_tune_mu)
  auto it = names.find(device);
  if (it == names.end()) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return false;
    it = names.emplace(device, std::string(prop.name)).first;
  }
  for (const TuneEntry& e : g_tune)
    if (e.n == n && e.device == it->second) {
      *out = e;
      return true;
    }
  return false;
}

// Per-slice counts -> prefix offsets; validates that the counts are whole, non-negative numbers.
Status offsets(const double* counts, int slices, std::vector<int>& beg, int& total, const char* what) {
  beg.assign(slices + 1, 0);
  total = 0;
  for (int s = 0; s < slices; ++s) {
    const double c = counts ? counts[s] : 0.0;
    if (!(c >= 0.0) || c != std::floor(c) || c > 1e9)
      return Status::Err(TOTEM_ERR_INVALID_ARG, std::string(what) + ": per-slice count is not a whole number >= 0");
    total += (int)c;
    beg[s + 1] = total;
  }
  return Status::Ok();
}

RowsHost split_rows(const double* rows, int count, int ncol, const double* absorp, const std::vector<int>& beg) {
  RowsHost h;
  h.count = count;
  h.ncoef = ncol - 2;
  h.beg = beg;
  h.pos.resize((size_t)count * 2);
  h.coef.resize((size_t)count * h.ncoef);
  for (int a = 0; a < count; ++a) {
    h.pos[2 * a] = rows[(size_t)a * ncol];
    h.pos[2 * a + 1] = rows[(size_t)a * ncol + 1];
    for (int k = 0; k < h.ncoef; ++k) h.coef[(size_t)a * h.ncoef + k] = (float)rows[(size_t)a * ncol + 2 + k];
  }
  if (absorp) {
    h.absorp.resize((size_t)count * 10);
    for (size_t i = 0; i < h.absorp.size(); ++i) h.absorp[i] = (float)absorp[i];
  }
  return h;
}

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Rows grouped by species: within every slice, atoms whose coefficient row (and absorptive row)
// are identical share one form factor.  Species keep their order of first appearance in the
// slice and atoms their row order within a species.
totem::SpeciesHost group_species(const RowsHost& h, int slices) {
  totem::SpeciesHost sp;
  sp.ncoef = h.ncoef;
  sp.seg_beg.assign(slices + 1, 0);
  sp.pos.reserve(h.pos.size());
  const bool ab = !h.absorp.empty();
  // key: the bytes of the coefficient row (and absorptive row); rows of one species usually come
  // in runs, so the previous row's id is tried first
  std::unordered_map<std::string, int> ids;
  std::string key, prev_key;
  int prev_id = -1;
  const size_t cbytes = (size_t)h.ncoef * sizeof(float);
  for (int s = 0; s < slices && h.count > 0; ++s) {
    std::vector<int> order;              // species in order of appearance in this slice
    std::map<int, std::vector<int>> atoms;
    for (int a = h.beg[s]; a < h.beg[s + 1]; ++a) {
      key.assign(reinterpret_cast<const char*>(h.coef.data() + (size_t)a * h.ncoef), cbytes);
      if (ab) key.append(reinterpret_cast<const char*>(h.absorp.data() + (size_t)a * 10), 10 * sizeof(float));
      int id = prev_id;
      if (prev_id < 0 || key != prev_key) {
        auto it = ids.find(key);
        if (it == ids.end()) {
          it = ids.emplace(key, (int)ids.size()).first;
          const float* f = reinterpret_cast<const float*>(key.data());
          sp.coef.insert(sp.coef.end(), f, f + h.ncoef);
          if (ab) sp.absorp.insert(sp.absorp.end(), f + h.ncoef, f + h.ncoef + 10);
        }
        id = it->second;
        prev_key = key;
        prev_id = id;
      }
      auto& v = atoms[id];
      if (v.empty()) order.push_back(id);
      v.push_back(a);
    }
    for (int id : order) {
      const int first = (int)(sp.pos.size() / 2);
      for (int a : atoms[id]) {
        sp.pos.push_back(h.pos[2 * (size_t)a]);
        sp.pos.push_back(h.pos[2 * (size_t)a + 1]);
      }
      sp.seg.insert(sp.seg.end(), {id, first, (int)(sp.pos.size() / 2)});
    }
    sp.seg_beg[s + 1] = (int)(sp.seg.size() / 3);
  }
  return sp;
}


}  // namespace

void totem::set_last_error(const std::string& msg) { g_last_error = msg; }

int totem::tx_builder_mode() { return g_tx_mode.load(); }
bool totem::slice_graphs_enabled() { return g_slice_graphs.load() != 0; }
bool totem::band_skip_enabled() { return g_band_skip.load() != 0; }

bool totem::inject_alloc_failure() {
  long long left = g_fail_alloc_after.load();
  while (left >= 0) {  // armed: count down, fail once at zero, then disarm
    if (g_fail_alloc_after.compare_exchange_weak(left, left - 1)) return left == 0;
  }
  return false;
}

bool totem::inject_prepare_failure() {
  const long long k = g_fail_prepare_every.load();
  if (k <= 0) return false;
  return (g_prepares.fetch_add(1) + 1) % k == 0;
}
size_t totem::tx_gridding_scratch() {
  const size_t b = g_tx_scratch.load();
  return b ? b : (1ull << 30);
}

thread_local long long totem::g_h2d_bytes = 0;

std::vector<float2> totem::twiddles(int n) {
  std::vector<float2> t = totem::stage_twiddles(n);
  if (t.empty()) t.assign(1, make_float2(1.f, 0.f));
  return t;
}

// ---------------------------------------------------------------------------------------------
// Upload
// ---------------------------------------------------------------------------------------------
Status totem_session::validate(const TotemStemArgs* a, bool stem) {
  if (a == nullptr) return Status::Err(TOTEM_ERR_INVALID_ARG, "args is NULL");
  if (a->struct_size != (int)sizeof(TotemStemArgs))
    return Status::Err(TOTEM_ERR_INVALID_ARG, "TotemStemArgs.struct_size does not match this library");
  if (a->param != TOTEM_PARAM_PENG && a->param != TOTEM_PARAM_LOBATO)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "param must be TOTEM_PARAM_PENG or TOTEM_PARAM_LOBATO");
  if (a->p_height <= 0 || a->p_width <= 0 || a->slices < 0)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "negative or zero potential-grid size");
  if ((a->p_height | a->p_width) & 1)
    return Status::Err(TOTEM_ERR_UNSUPPORTED, "odd grid sizes are not supported (the ifftshift is a quadrant swap)");
  if (a->layer_len < 0 || a->cim_len < 0) return Status::Err(TOTEM_ERR_INVALID_ARG, "negative count");
  // The transmission-only MEX receives empty probe / aperture inputs (cuda_stem_potential.m,
  // HRTEMsimulation sets probe = [] at ToTEM_submit_v1.m:1259); STEM fields are checked only
  // when a STEM request is present.
  const bool want_stem = stem && a->depth > 0;
  if (want_stem) {
    if (a->height <= 0 || a->width <= 0 || a->w_num <= 0 || a->aper_num < 0)
      return Status::Err(TOTEM_ERR_INVALID_ARG, "negative or zero window size");
    if ((a->height | a->width) & 1)
      return Status::Err(TOTEM_ERR_UNSUPPORTED, "odd window sizes are not supported (the ifftshift is a quadrant swap)");
    if (a->width_red <= 0 || a->step < 0)
      return Status::Err(TOTEM_ERR_INVALID_ARG, "width_red must be positive and step non-negative");
    const long last = a->depth - 1;
    const long rmax = a->begin_row + (last / a->width_red) * (long)a->step;
    const long cmax = a->begin_col + (long)std::min<long>(last, a->width_red - 1) * a->step;
    if (a->begin_row < 0 || a->begin_col < 0 || rmax + a->height > a->p_height || cmax + a->width > a->p_width)
      return Status::Err(TOTEM_ERR_INVALID_ARG, "probe windows leave the potential grid");
    if (!a->probe_re || !a->probe_im || !a->prop_re || !a->prop_im || !a->gfsf || (a->aper_num > 0 && !a->aper))
      return Status::Err(TOTEM_ERR_INVALID_ARG, "probe, propagator, gfsf and aper are required for STEM");
    if (a->layer_len > 0 && (!a->mid_layer || (a->aper_num > 0 && !a->aper2)))
      return Status::Err(TOTEM_ERR_INVALID_ARG, "mid_layer and aper2 are required when layer_len > 0");
    if ((long long)a->w_num * a->depth > (1LL << 30)) return Status::Err(TOTEM_ERR_INVALID_ARG, "too many probes");
  }
  if (!a->kx || !a->ky || !a->s_2 || !a->aper_true)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "kx, ky, s_2 and aper_true are required");
  std::vector<int> beg;
  int count = 0;
  TOTEM_TRY(offsets(a->atom_slice, a->slices, beg, count, "atom_slice"));
  if (count > 0 && !a->proj_coff_mat) return Status::Err(TOTEM_ERR_INVALID_ARG, "proj_coff_mat is NULL");
  TOTEM_TRY(offsets(a->atom_slice_i, a->slices, beg, count, "atom_slice_i"));
  if (count > 0 && !a->proj_coff_mat_i) return Status::Err(TOTEM_ERR_INVALID_ARG, "proj_coff_mat_i is NULL");
  return Status::Ok();
}

Status totem_session::upload_args(const TotemStemArgs* a, bool stem) {
  g_h2d_bytes = 0;
  stem_ready = false;
  TOTEM_TRY(validate(a, stem));
  const bool want_stem = stem && a->depth > 0;
  param = a->param;
  p_h = a->p_height; p_w = a->p_width; slices = a->slices;
  sigma = a->sigma; parameter = a->parameter;
  if (want_stem) {
    h = a->height; w = a->width; depth = a->depth;
    step = a->step; begin_row = a->begin_row; begin_col = a->begin_col; width_red = a->width_red;
    w_num = a->w_num; aper_num = a->aper_num;
    mid_layer.assign(a->mid_layer, a->mid_layer + a->layer_len);
    gfsf.assign(a->gfsf, a->gfsf + a->w_num);
  } else {
    h = w = depth = step = begin_row = begin_col = width_red = aper_num = 0;
    w_num = 1;
    mid_layer.clear();
    gfsf.assign(1, 1.0);
  }
  cudaStream_t st = stream;
  uploaded = false;
  t_valid = false;
  tb_valid = false;
  has_result = false;

  // coefficient rows
  const int nc_n = (param == TOTEM_PARAM_LOBATO) ? 14 : 13;
  const int nc_i = (param == TOTEM_PARAM_LOBATO) ? 26 : 25;
  std::vector<int> beg_n, beg_i, beg_cn, beg_ci;
  TOTEM_TRY(offsets(a->atom_slice, slices, beg_n, n_rows, "atom_slice"));
  TOTEM_TRY(offsets(a->atom_slice_i, slices, beg_i, n_rows_i, "atom_slice_i"));
  if (n_rows > 0 && !a->proj_coff_mat) return Status::Err(TOTEM_ERR_INVALID_ARG, "proj_coff_mat is NULL");
  if (n_rows_i > 0 && !a->proj_coff_mat_i) return Status::Err(TOTEM_ERR_INVALID_ARG, "proj_coff_mat_i is NULL");
  has_abs_n = a->absorp_n != nullptr && n_rows > 0;
  has_abs_i = a->absorp_n_i != nullptr && n_rows_i > 0;
  ncoef_n = nc_n - 2;
  ncoef_i = nc_i - 2;
  const RowsHost host_n = split_rows(a->proj_coff_mat, n_rows, nc_n, has_abs_n ? a->absorp_n : nullptr, beg_n);
  const RowsHost host_i = split_rows(a->proj_coff_mat_i, n_rows_i, nc_i, has_abs_i ? a->absorp_n_i : nullptr, beg_i);
  cim_len = a->cim_len;
  n_corr = n_corr_i = 0;
  RowsHost host_cn, host_ci;
  if (cim_len > 0) {
    if (!a->corr_info_matrix) return Status::Err(TOTEM_ERR_INVALID_ARG, "corr_info_matrix is NULL");
    TOTEM_TRY(offsets(a->series_n_corr, slices, beg_cn, n_corr, "series_n_corr"));
    TOTEM_TRY(offsets(a->series_n_i_corr, slices, beg_ci, n_corr_i, "series_n_i_corr"));
    if ((n_corr > 0 && !a->ele_n_corr) || (n_corr_i > 0 && !a->ele_n_i_corr))
      return Status::Err(TOTEM_ERR_INVALID_ARG, "correction rows are NULL");
    host_cn = split_rows(a->ele_n_corr, n_corr, 5, nullptr, beg_cn);
    host_ci = split_rows(a->ele_n_i_corr, n_corr_i, 8, nullptr, beg_ci);
    const size_t plane = (size_t)p_h * p_w;
    std::vector<float> c(plane * cim_len);
    for (size_t i = 0; i < c.size(); ++i) c[i] = (float)a->corr_info_matrix[i];
    TOTEM_TRY(upload(cim, c, st));
  }

  // reciprocal grids: detect the reference's separable meshgrid layout
  const size_t plane = (size_t)p_h * p_w;
  separable = true;
  for (int r = 0; r < p_h && separable; ++r)
    for (int c = 0; c < p_w; ++c)
      if (a->kx[(size_t)r * p_w + c] != a->kx[c] || a->ky[(size_t)r * p_w + c] != a->ky[(size_t)r * p_w]) {
        separable = false;
        break;
      }
  // neutral, ionic and correction rows: by species on separable grids (k_tx_species or
  // gridding), row by row otherwise
  grid_ok = false;
  if (separable) {
    const totem::SpeciesHost spn = group_species(host_n, slices), spi = group_species(host_i, slices);
    const totem::SpeciesHost spcn = group_species(host_cn, slices), spci = group_species(host_ci, slices);
    TOTEM_TRY(species_n.put(spn, st));
    TOTEM_TRY(species_i.put(spi, st));
    // Correction rows share a form factor when they share B, amplitude and plane, i.e. per element
    // (CalAllEquilent20210305_peng_corr.m); rows that are nearly all distinct are cheaper per atom
    const size_t corr_rows = (size_t)n_corr + n_corr_i, corr_species = (spcn.seg.size() + spci.seg.size()) / 3;
    corr_by_species = corr_rows == 0 || corr_species * 4 <= corr_rows;
    const totem::SpeciesHost none;
    if (corr_by_species) {
      TOTEM_TRY(species_cn.put(spcn, st));
      TOTEM_TRY(species_ci.put(spci, st));
    } else {
      TOTEM_TRY(rows_cn.put(host_cn, st));
      TOTEM_TRY(rows_ci.put(host_ci, st));
    }
    const totem::SpeciesHost* const kinds[4] = {&spn, &spi, corr_by_species ? &spcn : &none,
                                                corr_by_species ? &spci : &none};
    TOTEM_TRY(plan_gridding(a, kinds));
  } else {
    TOTEM_TRY(rows_n.put(host_n, st));
    TOTEM_TRY(rows_i.put(host_i, st));
    TOTEM_TRY(rows_cn.put(host_cn, st));
    TOTEM_TRY(rows_ci.put(host_ci, st));
  }
  std::vector<float> s2f(plane);
  for (size_t i = 0; i < plane; ++i) s2f[i] = (float)a->s_2[i];
  TOTEM_TRY(upload(s2, s2f, st));
  if (separable) {
    std::vector<double> kxa(a->kx, a->kx + p_w), kya(p_h);
    for (int r = 0; r < p_h; ++r) kya[r] = a->ky[(size_t)r * p_w];
    TOTEM_TRY(upload(kx_axis, kxa, st));
    TOTEM_TRY(upload(ky_axis, kya, st));
  } else {
    TOTEM_TRY(upload(kx, std::vector<double>(a->kx, a->kx + plane), st));
    TOTEM_TRY(upload(ky, std::vector<double>(a->ky, a->ky + plane), st));
  }
  aper_true_ones = true;
  for (size_t i = 0; i < plane; ++i)
    if (a->aper_true[i] != 1.0) {
      aper_true_ones = false;
      break;
    }
  if (!aper_true_ones) {
    std::vector<float> at(plane);
    for (size_t i = 0; i < plane; ++i) at[i] = (float)a->aper_true[i];
    TOTEM_TRY(upload(aper_true, at, st));
  }
  TOTEM_TRY(upload(tw_pw, twiddles(p_w), st));
  TOTEM_TRY(upload(tw_ph, twiddles(p_h), st));

  // probe, propagator, masks
  if (want_stem) {
    const size_t vol = (size_t)h * w;
    std::vector<float2> pr(vol * w_num), hp(vol);
    for (size_t i = 0; i < pr.size(); ++i) pr[i] = make_float2((float)a->probe_re[i], (float)a->probe_im[i]);
    for (size_t i = 0; i < vol; ++i) hp[i] = make_float2((float)a->prop_re[i], (float)a->prop_im[i]);
    TOTEM_TRY(upload(probe, pr, st));
    TOTEM_TRY(upload(prop, hp, st));
    band = (h == w) ? totem::spectral_band(a->prop_re, a->prop_im, h, w) : (1 << 30);
    // exit detector: ifftshift(aper) (the reference shifts the wave instead, cuda_source_lobato.cu:1415)
    std::vector<float> me(vol * std::max(aper_num, 1)), mm;
    for (int q = 0; q < aper_num; ++q)
      for (int r = 0; r < h; ++r)
        for (int c = 0; c < w; ++c)
          me[(size_t)q * vol + (size_t)r * w + c] =
              (float)a->aper[(size_t)q * vol + (size_t)((r + h / 2) % h) * w + (c + w / 2) % w];
    TOTEM_TRY(upload(mask_exit, me, st));
    if (a->layer_len > 0 && aper_num > 0) {
      mm.resize(vol * aper_num);
      for (size_t i = 0; i < mm.size(); ++i) mm[i] = (float)a->aper2[i];
      TOTEM_TRY(upload(mask_mid, mm, st));
    }
    if (h == w) TOTEM_TRY(upload(tw_n, twiddles(h), st));
    TOTEM_TRY(upload(gfsf_d, gfsf, st));
  }
  TOTEM_CUDA(cudaStreamSynchronize(st));  // host staging vectors die at return
  uploaded = true;
  stem_ready = want_stem;
  h2d_bytes = g_h2d_bytes;
  return Status::Ok();
}

// ---------------------------------------------------------------------------------------------
// Transmission
// ---------------------------------------------------------------------------------------------
Status totem_session::build_transmission(int path, int* launches) {
  const size_t plane = (size_t)p_h * p_w;
  const bool fft_fused = totem::tx_fft_shape_ok(p_h, p_w, std::max(slices, 1));
  if (path == TOTEM_PATH_FUSED_ONLY && !fft_fused && slices > 0)
    return Status::Err(TOTEM_ERR_UNSUPPORTED,
                       "TOTEM_PATH_FUSED_ONLY: the transmission FFT needs potential grid edges of 64..4096 "
                       "that are powers of two or mixed-radix edges, in whole tiles");
  TOTEM_TRY(T.ensure(plane * std::max(slices, 1) * sizeof(float2)));
  if (slices == 0) return Status::Ok();
  totem::TxGrid g;
  g.p_h = p_h; g.p_w = p_w; g.slices = slices;
  g.separable = separable;
  g.kx_axis = kx_axis.as<double>(); g.ky_axis = ky_axis.as<double>();
  g.kx = kx.as<double>(); g.ky = ky.as<double>();
  g.s2 = s2.as<float>();
  g.aper_true = aper_true_ones ? nullptr : aper_true.as<float>();
  g.parameter = (float)parameter;
  g.lobato = (param == TOTEM_PARAM_LOBATO);
  g.cim = cim_len > 0 ? cim.as<float>() : nullptr;
  g.cim_len = cim_len;
  const auto vcn = rows_cn.view(cim_len > 0 && n_corr > 0, false, 3);
  const auto vci = rows_ci.view(cim_len > 0 && n_corr_i > 0, false, 6);
  if (separable) {
    totem::SpeciesSet set;
    set.k[0] = species_n.view(n_rows > 0, has_abs_n, ncoef_n);
    set.k[1] = species_i.view(n_rows_i > 0, has_abs_i, ncoef_i);
    if (corr_by_species) {
      set.k[2] = species_cn.view(cim_len > 0 && n_corr > 0, false, 3);
      set.k[3] = species_ci.view(cim_len > 0 && n_corr_i > 0, false, 6);
    }
    const int mode = totem::tx_builder_mode();
    if (grid_ok && (mode == TOTEM_TX_GRIDDING || (mode == TOTEM_TX_AUTO && gridding_cheaper()))) {
      // jobs per batch from the budget for their planes (64 bytes per pixel); the row flags on top
      const size_t jobs = std::max<size_t>(grid_jobs_h.size(), 1);
      const size_t per = std::min(totem::tx_gridding_scratch() / ((size_t)p_h * p_w * 64), jobs);
      const size_t bytes = std::max<size_t>(1, per) * totem::grid_job_bytes(p_h, p_w);
      // the state the kernels leave the scratch in depends on the row layout and the batch size
      const long long layout = ((long long)p_h << 40) | ((long long)p_w << 20) | (long long)std::max<size_t>(1, per);
      if (bytes > grid_scratch.cap || layout != grid_scratch_layout) grid_scratch_zero = false;
      TOTEM_TRY(grid_scratch.ensure(bytes));
      grid_scratch_layout = layout;
      totem::GridPlanDev gp;
      gp.dkx = grid_dkx; gp.dky = grid_dky; gp.sx = grid_sx; gp.sy = grid_sy;
      gp.ax = grid_ax.as<float2>(); gp.ay = grid_ay.as<float2>();
      gp.jobs = grid_jobs.as<int4>(); gp.job_beg = grid_job_beg.as<int>();
      const bool was_zero = grid_scratch_zero;
      grid_scratch_zero = false;  // until every batch has been enqueued
      ran_tx_builder = TOTEM_TX_GRIDDING;
      TOTEM_TRY(totem::launch_tx_gridding(g, set, gp, grid_job_beg_h, grid_jobs_h, tw_pw.as<float2>(),
                                          tw_ph.as<float2>(), grid_scratch.p, bytes, was_zero, T.as<float2>(), stream,
                                          launches));
      grid_scratch_zero = true;  // left as the next build expects it (in stream order)
      // work memory of the build only: returned at once to a server's pool (stream-ordered and
      // cheap); a plain session keeps it, cleared, for its next build (cudaFree would synchronise)
      if (grid_scratch.pool) {
        grid_scratch.release();
        grid_scratch_zero = false;
      }
    } else {
      ran_tx_builder = TOTEM_TX_DIRECT;
      TOTEM_TRY(totem::launch_tx_species(g, set, T.as<float2>(), stream));
      ++*launches;
    }
    if (!corr_by_species && (vcn.beg || vci.beg)) {  // nearly distinct correction rows: per atom, added
      TOTEM_TRY(totem::launch_tx_structure(g, totem::AtomRowsDev{}, totem::AtomRowsDev{}, vcn, vci, T.as<float2>(),
                                           stream, true));
      ++*launches;
    }
  } else {
    const auto vn = rows_n.view(n_rows > 0, has_abs_n, ncoef_n);
    const auto vi = rows_i.view(n_rows_i > 0, has_abs_i, ncoef_i);
    ran_tx_builder = TOTEM_TX_ROWS;
    TOTEM_TRY(totem::launch_tx_structure(g, vn, vi, vcn, vci, T.as<float2>(), stream));
    ++*launches;
  }
  const float sig = (float)(sigma / 1000.0);
  if (path != TOTEM_PATH_PLAIN && fft_fused) {
    ran_tx_fft = TOTEM_PATH_FUSED;
    TOTEM_TRY(totem::launch_tx_fft_exp(T.as<float2>(), slices, p_h, p_w, sig, tw_pw.as<float2>(),
                                       tw_ph.as<float2>(), stream));
    *launches += 2;
  } else {
    ran_tx_fft = TOTEM_PATH_PLAIN;
    cufftHandle p;
    TOTEM_TRY(plan(p_h, p_w, slices, &p));
    TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)T.p, (cufftComplex*)T.p, CUFFT_INVERSE));
    TOTEM_TRY(totem::launch_sign_exp(T.as<float2>(), (long)plane * slices, p_h, p_w, sig, stream));
    *launches += 2;
  }
  t_valid = true;
  tb_valid = false;
  return Status::Ok();
}

// Uniform separable axes, kx(c) = kx0 + c dkx and ky(r) = ky0 + r dky (the reference's
// meshgrid of (-P/2 : P/2-1) / (P dx), ToTEM_submit_v1.m:1534-1538), on power-of-two grids admit
// the gridding builder.  Its job table holds one job per species segment of every slice
// (neutral, ionic, then the correction kinds), in slice order.
Status totem_session::plan_gridding(const TotemStemArgs* a, const totem::SpeciesHost* const (&kinds)[4]) {
  grid_ok = false;
  grid_job_beg_h.clear();
  grid_jobs_h.clear();
  grid_atoms = 0;
  if (!totem::gridding_size_ok(p_h) || !totem::gridding_size_ok(p_w) || slices <= 0) return Status::Ok();
  auto uniform = [](const double* v, int n, long stride, double* d) {
    *d = (v[(long)(n - 1) * stride] - v[0]) / (n - 1);
    if (!std::isfinite(*d) || *d == 0.0) return false;
    for (int i = 0; i < n; ++i)
      if (!(std::fabs(v[(long)i * stride] - (v[0] + i * *d)) <= 1e-9 * std::fabs(*d))) return false;
    return true;
  };
  double dkx = 0, dky = 0;
  if (!uniform(a->kx, p_w, 1, &dkx) || !uniform(a->ky, p_h, p_w, &dky)) return Status::Ok();
  grid_dkx = dkx;
  grid_dky = dky;
  grid_sx = a->kx[0] + dkx * (p_w / 2);
  grid_sy = a->ky[0] + dky * (p_h / 2);
  grid_job_beg_h.assign(slices + 1, 0);
  for (int s = 0; s < slices; ++s) {
    for (int kind = 0; kind < 4; ++kind) {
      const totem::SpeciesHost& sp = *kinds[kind];
      if ((int)sp.seg_beg.size() != slices + 1) continue;
      for (int q = sp.seg_beg[s]; q < sp.seg_beg[s + 1]; ++q) {
        grid_jobs_h.push_back(make_int4(kind, sp.seg[3 * q], sp.seg[3 * q + 1], sp.seg[3 * q + 2]));
        grid_atoms += sp.seg[3 * q + 2] - sp.seg[3 * q + 1];
      }
    }
    grid_job_beg_h[s + 1] = (int)grid_jobs_h.size();
  }
  cudaStream_t st = stream;
  TOTEM_TRY(upload(grid_jobs, grid_jobs_h, st));
  TOTEM_TRY(upload(grid_job_beg, grid_job_beg_h, st));
  TOTEM_TRY(upload(grid_ax, totem::grid_deconvolution(p_w), st));
  TOTEM_TRY(upload(grid_ay, totem::grid_deconvolution(p_h), st));
  grid_ok = true;
  return Status::Ok();
}

// Cost model of the two separable builders, measured on B200 (SrTiO3 supercells filling the
// grid, 20 slices): the direct sums take ~0.29 ps per atom and pixel; gridding takes per job
// (species and slice) and pixel 29 ps at 1024^2, 35 ps at 2048^2 and 44 ps at 4096^2 (the
// long column transforms run below bandwidth), plus ~20 us of launches per batch.
bool totem_session::gridding_cheaper() const {
  const double plane = (double)p_h * p_w;
  const double jobs = (double)grid_jobs_h.size();
  const int edge = std::max(p_h, p_w);
  const double per_px = edge <= 1024 ? 2.9e-11 : (edge <= 2048 ? 3.5e-11 : 4.4e-11);
  const double per_batch = std::max(1.0, std::floor((double)totem::tx_gridding_scratch() / (plane * 64.0)));
  const double direct = 2.9e-13 * (double)grid_atoms * plane;
  const double gridding = per_px * jobs * plane + 2e-5 * (std::ceil(jobs / per_batch) + 1);
  return gridding < direct;
}

// ---------------------------------------------------------------------------------------------
// Slice loop
// ---------------------------------------------------------------------------------------------
Status totem_session::transmission_for(int t_storage, const void** t, size_t* slice_bytes, int* launches) {
  const size_t plane = (size_t)p_h * p_w;
  if (t_storage == TOTEM_T_BF16) {
    if (!tb_valid) {
      TOTEM_TRY(Tb.ensure(plane * std::max(slices, 1) * 4));
      TOTEM_TRY(totem::launch_to_bf16(T.as<float2>(), Tb.p, (long)(plane * slices), stream));
      ++*launches;
      tb_valid = true;
    }
    *t = Tb.p;
    *slice_bytes = plane * 4;
  } else {
    *t = T.p;
    *slice_bytes = plane * sizeof(float2);
  }
  return Status::Ok();
}

Status totem_session::slice_loop(int path, int batch, int col_variant, int t_storage, int* launches,
                                 int* batch_used, int row_variant) {
  const long items_total = (long)w_num * depth;
  const long ad = (long)aper_num * depth;
  const int L = (int)mid_layer.size();
  TOTEM_TRY(out_result.ensure(std::max<long>(ad, 1) * sizeof(double)));
  TOTEM_TRY(out_mid.ensure(std::max<long>(ad * L, 1) * sizeof(double)));
  if (items_total == 0 || aper_num == 0) {
    has_result = true;
    return Status::Ok();
  }
  const totem::DetectionEvents de = detection_events();
  const std::vector<int>& event_of_slice = de.event_of_slice;
  const int n_events = de.n_events, exit_event = de.exit_event;

  const bool fused = (path != TOTEM_PATH_PLAIN) && h == w && totem::fused_window_ok(h) && slices > 0;
  if (path == TOTEM_PATH_FUSED_ONLY && !fused && slices > 0)
    return Status::Err(TOTEM_ERR_UNSUPPORTED,
                       "TOTEM_PATH_FUSED_ONLY: the fused slice loop needs a square window of 64..2048, a power of "
                       "two or a mixed-radix edge (96, 160, 192, 288, 320, 384, 400, 448, 576, 640, 768, 800, "
                       "1152, 1280, 1536, 1600)");
  ran_slice_path = fused ? TOTEM_PATH_FUSED : TOTEM_PATH_PLAIN;
  const size_t vol = (size_t)h * w;
  int B = batch;
  if (B <= 0) {
    // Large batches win on B200: keeping a batch L2-resident between passes (<= ~64 MB) was
    // measured slower than streaming a large batch through HBM, because wave tails dominate the
    // short launches (SrTiO3 512^2: 24 probes 948 ms, 4096 probes 879 ms per request).
    const size_t target = fused ? (4ull << 30) : (1ull << 30);
    B = (int)std::max<size_t>(1, target / (vol * sizeof(float2)));
  }
  B = (int)std::min<long>(B, items_total);
  {  // spread the items evenly over the batches
    const long nb = (items_total + B - 1) / B;
    B = (int)((items_total + nb - 1) / nb);
  }
  *batch_used = B;
  const int nblk = fused ? totem::col_blocks(h, col_variant) : 64;
  // the zero band of the propagator: columns the fused passes leave out, tiles the detector sums
  // leave out (the bfloat16 trial computes every column)
  const bool skip_band = fused && totem::band_skip_enabled() && t_storage == TOTEM_T_COMPLEX64 &&
                         totem::band_skip_ok(h, band, col_variant);
  const totem::TileSkip skip = skip_band ? totem::band_tiles(h, nblk) : totem::TileSkip();
  TOTEM_TRY(psi.ensure((size_t)B * vol * sizeof(float2)));
  TOTEM_TRY(part.ensure((size_t)n_events * B * aper_num * nblk * sizeof(double)));
  TOTEM_TRY(acc.ensure((size_t)n_events * w_num * ad * sizeof(double)));
  double* part_e = part.as<double>();
  const size_t part_stride = (size_t)B * aper_num * nblk;
  totem::ScanGeom geo{begin_row, begin_col, step, width_red, depth, p_w};
  const float2* Tp = T.as<float2>();
  const size_t plane = (size_t)p_h * p_w;
  const void* Tslices = Tp;
  size_t tslice_bytes = plane * sizeof(float2);
  if (t_storage != TOTEM_T_COMPLEX64) {
    if (!fused) return Status::Err(TOTEM_ERR_UNSUPPORTED, "bfloat16 transmission storage needs the fused path");
    TOTEM_TRY(transmission_for(t_storage, &Tslices, &tslice_bytes, launches));
  }
  auto tslice = [&](int k) { return static_cast<const char*>(Tslices) + (size_t)k * tslice_bytes; };

  // Everything below is stream work only (no allocation, no host synchronisation), so a repeated
  // fused run can replay it as one CUDA graph (see run_graphed).
  auto enqueue = [&]() -> Status {
    TOTEM_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)n_events * w_num * ad * sizeof(double), stream));
    for (long item0 = 0; item0 < items_total; item0 += B) {
      const int items = (int)std::min<long>(B, items_total - item0);
      if (fused) {
        totem::SliceLoopArgs s;
        s.n = h; s.items = items; s.item0 = (int)item0; s.geo = geo; s.p_h = p_h;
        s.psi = psi.as<float2>(); s.probe = probe.as<float2>(); s.prop = prop.as<float2>();
        s.tw = tw_n.as<float2>(); s.aper_num = aper_num;
        s.mask_mid = mask_mid.as<float>(); s.mask_exit = mask_exit.as<float>();
        s.col_variant = col_variant;
        s.t_bf16 = (t_storage == TOTEM_T_BF16);
        s.skip_band = skip_band ? 1 : 0;
        s.row_variant = row_variant;
        TOTEM_TRY(prof_begin());
        TOTEM_TRY(totem::launch_row_pass(s, tslice(0), true, stream));
        TOTEM_TRY(prof_end(0));
        ++*launches;
        for (int k = 0; k < slices; ++k) {
          const int ev_mid = event_of_slice[k + 1];
          int flags = 0;
          if (ev_mid >= 0) {
            flags |= 1;
            s.part_mid = part_e + ev_mid * part_stride;
          }
          if (k == slices - 1) {
            flags |= 2 | 4;
            s.part_exit = part_e + exit_event * part_stride;
          }
          TOTEM_TRY(prof_begin());
          TOTEM_TRY(totem::launch_col_pass(s, flags, stream));
          TOTEM_TRY(prof_end(1));
          ++*launches;
          if (k < slices - 1) {
            TOTEM_TRY(prof_begin());
            TOTEM_TRY(totem::launch_row_pass(s, tslice(k + 1), false, stream));
            TOTEM_TRY(prof_end(0));
            ++*launches;
          }
        }
      } else {
        cufftHandle p;
        TOTEM_TRY(plan(h, w, items, &p));
        float2* ps = psi.as<float2>();
        TOTEM_TRY(totem::launch_plain_init(ps, probe.as<float2>(), h, w, items, (int)item0, depth, stream));
        ++*launches;
        for (int k = 0; k < slices; ++k) {
          TOTEM_TRY(totem::launch_plain_gather_mul(ps, Tp + (size_t)k * plane, h, w, items, (int)item0, geo, stream));
          TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_FORWARD));
          TOTEM_TRY(totem::launch_plain_mul(ps, prop.as<float2>(), (int)vol, items, stream));
          *launches += 3;
          const int ev_mid = event_of_slice[k + 1];
          if (ev_mid >= 0) {
            TOTEM_TRY(totem::launch_plain_detect(ps, mask_mid.as<float>(), aper_num, (int)vol, items,
                                                 part_e + ev_mid * part_stride, nblk, stream));
            ++*launches;
          }
          TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_INVERSE));
          TOTEM_TRY(totem::launch_plain_scale(ps, 1.f / (float)vol, (long)items * vol, stream));
          *launches += 2;
        }
        TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_FORWARD));
        TOTEM_TRY(totem::launch_plain_detect(ps, mask_exit.as<float>(), aper_num, (int)vol, items,
                                             part_e + exit_event * part_stride, nblk, stream));
        *launches += 2;
      }
      for (int e = 0; e < n_events; ++e) {
        TOTEM_TRY(totem::launch_det_reduce(part_e + e * part_stride, nblk, aper_num, items, (int)item0, depth,
                                           acc.as<double>() + (size_t)e * w_num * ad, stream, skip));
        ++*launches;
      }
    }
    return combine_results(de, launches);
  };

  if (!fused || profiling || !totem::slice_graphs_enabled()) {
    TOTEM_TRY(enqueue());
  } else {
    // what the launches embed: sizes, buffer addresses and the detection events
    std::vector<long long> key = {h, items_total, B, slices, col_variant, t_storage, n_events, exit_event, aper_num,
                                  w_num, depth, nblk, L, p_h, p_w, begin_row, begin_col, step, width_red,
                                  (long long)tslice_bytes, skip_band ? 1 : 0, row_variant};
    for (const void* q : {(const void*)psi.p, (const void*)part.p, (const void*)acc.p, (const void*)probe.p,
                          (const void*)prop.p, (const void*)tw_n.p, (const void*)mask_mid.p, (const void*)mask_exit.p,
                          Tslices, (const void*)gfsf_d.p, (const void*)out_result.p, (const void*)out_mid.p})
      key.push_back((long long)(uintptr_t)q);
    key.insert(key.end(), event_of_slice.begin(), event_of_slice.end());
    key.insert(key.end(), de.layer_event.begin(), de.layer_event.end());
    TOTEM_TRY(run_graphed(key, enqueue, launches));
  }
  has_result = true;
  return Status::Ok();
}

// A run whose launches repeat an earlier run's exactly (same key) is captured into a CUDA graph
// the second time and replayed from then on: one launch call instead of two per slice and
// batch, and no host launch gaps between the short kernels of small requests.  The first run
// with a new key executes directly (it also sets every kernel's shared-memory limit, which is
// not done during capture).  Streams that cannot be captured (the legacy default stream, or one
// the caller is capturing already) run directly.
Status totem_session::run_graphed(const std::vector<long long>& key, const std::function<Status()>& enqueue,
                                  int* launches) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturable = stream != nullptr && stream != cudaStreamLegacy && stream != cudaStreamPerThread &&
                          cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
  if (!capturable) return enqueue();
  if (graph_exec != nullptr && key == graph_key) {
    TOTEM_CUDA(cudaGraphLaunch(graph_exec, stream));
    *launches += graph_launches;
    return Status::Ok();
  }
  if (key != graph_key) {  // first run of this shape
    drop_graph();
    graph_key = key;
    return enqueue();
  }
  const int before = *launches;
  TOTEM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  const Status st = enqueue();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(stream, &g);
  if (!st.ok() || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    graph_key.clear();
    return st.ok() ? totem::cuda_status(e, "cudaStreamEndCapture") : st;
  }
  cudaGraphExec_t x = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    graph_key.clear();
    return totem::cuda_status(ei, "cudaGraphInstantiate");
  }
  graph_exec = x;
  graph_launches = *launches - before;
  TOTEM_CUDA(cudaGraphLaunch(graph_exec, stream));
  return Status::Ok();
}

void totem_session::drop_graph() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  graph_launches = 0;
}

totem::DetectionEvents totem_session::detection_events() const {
  totem::DetectionEvents de;
  const int L = (int)mid_layer.size();
  de.event_of_slice.assign(slices + 1, -1);
  de.layer_event.assign(L, -1);
  for (int l = 0; l < L; ++l) {
    const int k = mid_layer[l];
    if (k < 1 || k > slices) continue;
    if (de.event_of_slice[k] < 0) {
      de.event_of_slice[k] = de.n_events++;
      de.layer_event[l] = de.event_of_slice[k];
    }
  }
  de.exit_event = de.n_events++;
  return de;
}

Status totem_session::combine_results(const totem::DetectionEvents& de, int* launches) {
  const long ad = (long)aper_num * depth;
  const int L = (int)mid_layer.size();
  TOTEM_TRY(totem::launch_combine(acc.as<double>() + (size_t)de.exit_event * w_num * ad, gfsf_d.as<double>(), w_num,
                                  ad, out_result.as<double>(), stream));
  ++*launches;
  if (L > 0) TOTEM_CUDA(cudaMemsetAsync(out_mid.p, 0, (size_t)ad * L * sizeof(double), stream));
  for (int l = 0; l < L; ++l) {
    if (de.layer_event[l] < 0) continue;
    TOTEM_TRY(totem::launch_combine(acc.as<double>() + (size_t)de.layer_event[l] * w_num * ad, gfsf_d.as<double>(),
                                    w_num, ad, out_mid.as<double>() + (size_t)l * ad, stream));
    ++*launches;
  }
  return Status::Ok();
}

// ---------------------------------------------------------------------------------------------
// HRTEM
// ---------------------------------------------------------------------------------------------
Status totem_session::hrtem(const TotemHrtemArgs* hr, TotemHrtemOut* out) {
  if (!uploaded) return Status::Err(TOTEM_ERR_STATE, "HRTEM before a successful upload");
  if (hr == nullptr || hr->struct_size != (int)sizeof(TotemHrtemArgs))
    return Status::Err(TOTEM_ERR_INVALID_ARG, "TotemHrtemArgs missing or of another size");
  if (!hr->prop_re || !hr->prop_im) return Status::Err(TOTEM_ERR_INVALID_ARG, "the propagator is required");
  if ((hr->wave_re == nullptr) != (hr->wave_im == nullptr))
    return Status::Err(TOTEM_ERR_INVALID_ARG, "wave_re and wave_im must both be given or both be NULL");
  if (hr->defoci < 0 || (hr->defoci > 0 && (!hr->tf_re || !hr->tf_im || !hr->weights)))
    return Status::Err(TOTEM_ERR_INVALID_ARG, "defoci > 0 needs tf_re, tf_im and weights");
  if (hr->t_storage != TOTEM_T_COMPLEX64 && hr->t_storage != TOTEM_T_BF16)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "unknown transmission storage");
  // the reference squares the potential grid (ToTEM_submit_v1.m:1240-1242); the fused passes take
  // the edges of fused_window_ok, cuFFT every other edge
  if (p_h != p_w || p_h < 2 || slices < 1)
    return Status::Err(TOTEM_ERR_UNSUPPORTED, "HRTEM needs a square grid and a slice");
  const int n = p_h;
  const bool fused = totem::fused_window_ok(n);
  if (!fused && hr->t_storage != TOTEM_T_COMPLEX64)
    return Status::Err(TOTEM_ERR_UNSUPPORTED, "the bfloat16 transmission trial needs a grid of the fused passes");
  TOTEM_CUDA(cudaSetDevice(device));
  const size_t vol = (size_t)n * n;
  int launches = 0;
  if (!t_valid) TOTEM_TRY(build_transmission(TOTEM_PATH_FUSED, &launches));
  const void* Tslices = nullptr;
  size_t tslice_bytes = 0;
  TOTEM_TRY(transmission_for(hr->t_storage, &Tslices, &tslice_bytes, &launches));

  std::vector<float2> wave(vol), prop(vol);
  for (size_t i = 0; i < vol; ++i) {
    wave[i] = hr->wave_re ? make_float2((float)hr->wave_re[i], (float)hr->wave_im[i]) : make_float2(1.f, 0.f);
    prop[i] = make_float2((float)hr->prop_re[i], (float)hr->prop_im[i]);
  }
  TOTEM_TRY(upload(hr_wave, wave, stream));
  TOTEM_TRY(upload(hr_prop, prop, stream));
  TOTEM_TRY(psi.ensure(vol * sizeof(float2)));
  timing.slice_path = fused ? TOTEM_PATH_FUSED : TOTEM_PATH_PLAIN;
  timing.tx_fft_path = ran_tx_fft;
  timing.tx_builder = ran_tx_builder;
  if (!fused) return hrtem_plain(hr, out, static_cast<const float2*>(Tslices));

  totem::SliceLoopArgs s;
  s.n = n; s.items = 1; s.item0 = 0;
  s.geo = totem::ScanGeom{0, 0, 0, 1, 1, n};
  s.p_h = n;
  s.psi = psi.as<float2>(); s.probe = hr_wave.as<float2>(); s.prop = hr_prop.as<float2>();
  s.tw = tw_pw.as<float2>();
  s.aper_num = 0;
  s.t_bf16 = (hr->t_storage == TOTEM_T_BF16);
  // every pass leaves out the propagator's zero band (the last column pass writes zeros there
  // into the kept spectrum); the bfloat16 trial computes every column
  s.skip_band = (totem::band_skip_enabled() && hr->t_storage == TOTEM_T_COMPLEX64 &&
                 totem::band_skip_ok(n, totem::spectral_band(hr->prop_re, hr->prop_im, n, n), 0))
                    ? 1
                    : 0;
  auto tslice = [&](int k) { return static_cast<const char*>(Tslices) + (size_t)k * tslice_bytes; };
  // psi = wave .* T_0, then per slice FFT2 .* psf_fft IFFT2 .* T_{k+1}; the last column pass keeps
  // the spectrum FFT2(psi_{S-1} .* T) .* psf_fft, whose IFFT2 is the exit wave
  TOTEM_TRY(totem::launch_row_pass(s, tslice(0), true, stream));
  for (int k = 0; k < slices; ++k) {
    TOTEM_TRY(totem::launch_col_pass(s, k == slices - 1 ? 4 | 8 : 0, stream));
    if (k < slices - 1) TOTEM_TRY(totem::launch_row_pass(s, tslice(k + 1), false, stream));
  }
  const float2* spec = psi.as<float2>();
  const bool want_exit = out && (out->exit_re || out->exit_im);
  const bool want_img = out && out->image && hr->defoci > 0;
  std::vector<float2> exit_h;
  std::vector<float> img_h;
  if (want_exit) {
    TOTEM_TRY(hr_work.ensure(vol * sizeof(float2)));
    TOTEM_TRY(hr_exit.ensure(vol * sizeof(float2)));
    TOTEM_TRY(totem::launch_exit_wave(n, spec, hr_work.as<float2>(), hr_exit.as<float2>(), tw_pw.as<float2>(), stream));
    exit_h.resize(vol);
    TOTEM_CUDA(cudaMemcpyAsync(exit_h.data(), hr_exit.p, vol * sizeof(float2), cudaMemcpyDeviceToHost, stream));
  }
  if (want_img) {
    const int K = hr->defoci;
    std::vector<float2> tf((size_t)K * vol);
    for (size_t i = 0; i < tf.size(); ++i) tf[i] = make_float2((float)hr->tf_re[i], (float)hr->tf_im[i]);
    TOTEM_TRY(upload(hr_tf, tf, stream));
    TOTEM_TRY(upload(hr_w, std::vector<double>(hr->weights, hr->weights + K), stream));
    TOTEM_TRY(hr_work.ensure((size_t)K * vol * sizeof(float2)));
    TOTEM_TRY(hr_img.ensure(vol * sizeof(float)));
    TOTEM_TRY(totem::launch_tcc_image(n, spec, hr_tf.as<float2>(), K, hr_w.as<double>(), hr_work.as<float2>(),
                                      hr_img.as<float>(), tw_pw.as<float2>(), stream));
    img_h.resize(vol);
    TOTEM_CUDA(cudaMemcpyAsync(img_h.data(), hr_img.p, vol * sizeof(float), cudaMemcpyDeviceToHost, stream));
  }
  TOTEM_CUDA(cudaStreamSynchronize(stream));
  for (size_t i = 0; i < exit_h.size(); ++i) {
    if (out->exit_re) out->exit_re[i] = exit_h[i].x;
    if (out->exit_im) out->exit_im[i] = exit_h[i].y;
  }
  for (size_t i = 0; i < img_h.size(); ++i) out->image[i] = img_h[i];
  return Status::Ok();
}

// HRTEM on cuFFT for grid edges the fused passes do not take: the same steps as the fused route
// (psi = wave .* T_0; per slice FFT2, .* propagator, and except after the last slice IFFT2 / N^2 and
// .* T_{k+1}), the spectrum of the last slice kept; the exit wave is its IFFT2 / N^2 and the image
// sum_k w_k |IFFT2(spectrum .* tf_k) / N^2|^2.
Status totem_session::hrtem_plain(const TotemHrtemArgs* hr, TotemHrtemOut* out, const float2* Tp) {
  const int n = p_h;
  const size_t vol = (size_t)n * n;
  const totem::ScanGeom geo{0, 0, 0, 1, 1, n};
  cufftHandle one;
  TOTEM_TRY(plan(n, n, 1, &one));
  float2* ps = psi.as<float2>();
  TOTEM_CUDA(cudaMemcpyAsync(ps, hr_wave.p, vol * sizeof(float2), cudaMemcpyDeviceToDevice, stream));
  for (int k = 0; k < slices; ++k) {
    TOTEM_TRY(totem::launch_plain_gather_mul(ps, Tp + (size_t)k * vol, n, n, 1, 0, geo, stream));
    TOTEM_CUFFT(cufftExecC2C(one, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_FORWARD));
    TOTEM_TRY(totem::launch_plain_mul(ps, hr_prop.as<float2>(), (int)vol, 1, stream));
    if (k < slices - 1) {
      TOTEM_CUFFT(cufftExecC2C(one, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_INVERSE));
      TOTEM_TRY(totem::launch_plain_scale(ps, 1.f / (float)vol, (long)vol, stream));
    }
  }
  const float scale = 1.f / ((float)n * (float)n);
  const bool want_exit = out && (out->exit_re || out->exit_im);
  const bool want_img = out && out->image && hr->defoci > 0;
  std::vector<float2> exit_h;
  std::vector<float> img_h;
  if (want_exit) {
    TOTEM_TRY(hr_exit.ensure(vol * sizeof(float2)));
    TOTEM_CUDA(cudaMemcpyAsync(hr_exit.p, ps, vol * sizeof(float2), cudaMemcpyDeviceToDevice, stream));
    TOTEM_CUFFT(cufftExecC2C(one, (cufftComplex*)hr_exit.p, (cufftComplex*)hr_exit.p, CUFFT_INVERSE));
    TOTEM_TRY(totem::launch_plain_scale(hr_exit.as<float2>(), scale, (long)vol, stream));
    exit_h.resize(vol);
    TOTEM_CUDA(cudaMemcpyAsync(exit_h.data(), hr_exit.p, vol * sizeof(float2), cudaMemcpyDeviceToHost, stream));
  }
  if (want_img) {
    const int K = hr->defoci;
    std::vector<float2> tf((size_t)K * vol);
    for (size_t i = 0; i < tf.size(); ++i) tf[i] = make_float2((float)hr->tf_re[i], (float)hr->tf_im[i]);
    TOTEM_TRY(upload(hr_tf, tf, stream));
    TOTEM_TRY(upload(hr_w, std::vector<double>(hr->weights, hr->weights + K), stream));
    TOTEM_TRY(hr_work.ensure((size_t)K * vol * sizeof(float2)));
    TOTEM_TRY(hr_img.ensure(vol * sizeof(float)));
    TOTEM_TRY(totem::launch_plain_tf_mul(hr_work.as<float2>(), ps, hr_tf.as<float2>(), (int)vol, K, stream));
    cufftHandle planes;
    TOTEM_TRY(plan(n, n, K, &planes));
    TOTEM_CUFFT(cufftExecC2C(planes, (cufftComplex*)hr_work.p, (cufftComplex*)hr_work.p, CUFFT_INVERSE));
    TOTEM_TRY(totem::launch_plain_image(hr_work.as<float2>(), K, hr_w.as<double>(), scale, (int)vol,
                                        hr_img.as<float>(), stream));
    img_h.resize(vol);
    TOTEM_CUDA(cudaMemcpyAsync(img_h.data(), hr_img.p, vol * sizeof(float), cudaMemcpyDeviceToHost, stream));
  }
  TOTEM_CUDA(cudaStreamSynchronize(stream));
  for (size_t i = 0; i < exit_h.size(); ++i) {
    if (out->exit_re) out->exit_re[i] = exit_h[i].x;
    if (out->exit_im) out->exit_im[i] = exit_h[i].y;
  }
  for (size_t i = 0; i < img_h.size(); ++i) out->image[i] = img_h[i];
  return Status::Ok();
}

// CBED (ToTEM_submit_v1.m:1478-1492): the uploaded probes (w_num defocus probes, one scan
// position) through every slice, and sum_w gfsf_w |fftshift(FFT2(psi_w))|^2.  The final FFT2 of
// the reference follows an IFFT2 of the last slice's spectrum .* psf, so it is that spectrum: the
// fused route keeps it from the last column pass (flag 8), the cuFFT route stops after its
// multiply.
Status totem_session::cbed(double* pattern) {
  if (!uploaded || !stem_ready) return Status::Err(TOTEM_ERR_STATE, "CBED before the upload of a probe request");
  if (pattern == nullptr) return Status::Err(TOTEM_ERR_INVALID_ARG, "pattern is NULL");
  if (depth != 1) return Status::Err(TOTEM_ERR_INVALID_ARG, "CBED takes one probe position (depth 1)");
  if (slices < 1) return Status::Err(TOTEM_ERR_INVALID_ARG, "CBED needs a slice");
  TOTEM_CUDA(cudaSetDevice(device));
  int launches = 0;
  if (!t_valid) TOTEM_TRY(build_transmission(TOTEM_PATH_FUSED, &launches));
  const size_t vol = (size_t)h * w;
  const bool fused = h == w && totem::fused_window_ok(h);
  TOTEM_TRY(psi.ensure((size_t)w_num * vol * sizeof(float2)));
  const totem::ScanGeom geo{begin_row, begin_col, step, width_red, depth, p_w};
  const float2* Tp = T.as<float2>();
  const size_t plane = (size_t)p_h * p_w;
  float2* ps = psi.as<float2>();
  if (fused) {
    totem::SliceLoopArgs s;
    s.n = h; s.items = w_num; s.item0 = 0; s.geo = geo; s.p_h = p_h;
    s.psi = ps; s.probe = probe.as<float2>(); s.prop = prop.as<float2>();
    s.tw = tw_n.as<float2>(); s.aper_num = 0;
    s.skip_band = (totem::band_skip_enabled() && totem::band_skip_ok(h, band, 0)) ? 1 : 0;
    TOTEM_TRY(totem::launch_row_pass(s, Tp, true, stream));
    for (int k = 0; k < slices; ++k) {
      TOTEM_TRY(totem::launch_col_pass(s, k == slices - 1 ? 4 | 8 : 0, stream));
      if (k < slices - 1) TOTEM_TRY(totem::launch_row_pass(s, Tp + (k + 1) * plane, false, stream));
    }
  } else {
    cufftHandle p;
    TOTEM_TRY(plan(h, w, w_num, &p));
    TOTEM_TRY(totem::launch_plain_init(ps, probe.as<float2>(), h, w, w_num, 0, depth, stream));
    for (int k = 0; k < slices; ++k) {
      TOTEM_TRY(totem::launch_plain_gather_mul(ps, Tp + (size_t)k * plane, h, w, w_num, 0, geo, stream));
      TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_FORWARD));
      TOTEM_TRY(totem::launch_plain_mul(ps, prop.as<float2>(), (int)vol, w_num, stream));
      if (k < slices - 1) {
        TOTEM_CUFFT(cufftExecC2C(p, (cufftComplex*)ps, (cufftComplex*)ps, CUFFT_INVERSE));
        TOTEM_TRY(totem::launch_plain_scale(ps, 1.f / (float)vol, (long)w_num * vol, stream));
      }
    }
  }
  TOTEM_TRY(cbed_out.ensure(vol * sizeof(double)));
  TOTEM_TRY(totem::launch_cbed_pattern(ps, gfsf_d.as<double>(), w_num, h, w, cbed_out.as<double>(), stream));
  TOTEM_CUDA(cudaMemcpyAsync(pattern, cbed_out.p, vol * sizeof(double), cudaMemcpyDeviceToHost, stream));
  TOTEM_CUDA(cudaStreamSynchronize(stream));
  timing.slice_path = fused ? TOTEM_PATH_FUSED : TOTEM_PATH_PLAIN;
  timing.tx_fft_path = ran_tx_fft;
  timing.tx_builder = ran_tx_builder;
  return Status::Ok();
}

Status totem_session::run(int what, const TotemRunOptions* opt) {
  if (!uploaded) return Status::Err(TOTEM_ERR_STATE, "run before a successful upload");
  TotemRunOptions o{};
  if (opt) o = *opt;
  if (o.path != TOTEM_PATH_FUSED && o.path != TOTEM_PATH_PLAIN && o.path != TOTEM_PATH_FUSED_ONLY)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "unknown path");
  TOTEM_CUDA(cudaSetDevice(device));
  for (auto& e : ev)
    if (!e) TOTEM_CUDA(cudaEventCreate(&e));
  int launches = 0, batch_used = 0;
  has_result = false;
  last_what = what;
  ran_slice_path = ran_tx_fft = ran_tx_builder = -1;
  profiling = o.profile != 0;
  pkind.clear();
  pused = 0;
  TOTEM_CUDA(cudaEventRecord(ev[0], stream));
  if (!(o.skip_transmission && t_valid)) TOTEM_TRY(build_transmission(o.path, &launches));
  TOTEM_CUDA(cudaEventRecord(ev[1], stream));
  if (what == 0) {
    if (!stem_ready && depth > 0) return Status::Err(TOTEM_ERR_STATE, "no STEM inputs uploaded");
    if (o.t_storage != TOTEM_T_COMPLEX64 && o.t_storage != TOTEM_T_BF16)
      return Status::Err(TOTEM_ERR_INVALID_ARG, "unknown transmission storage");
    // launch shapes left at 0: the tuning table's entry for this GPU and window, else built-in
    int rv = o.row_variant, cv = o.col_variant, batch = o.batch;
    if (o.path != TOTEM_PATH_PLAIN && h == w && (rv == 0 || cv == 0 || batch == 0)) {
      TuneEntry e;
      if (tuned_entry(device, h, &e)) {
        if (rv == 0) rv = e.row_variant;
        if (cv == 0) cv = e.col_variant;
        if (batch == 0 && e.batch_bytes > 0)
          batch = (int)std::max<long long>(1, e.batch_bytes / ((long long)h * w * (long long)sizeof(float2)));
      }
    }
    if (h == w && totem::radix_window_ops(h)) rv = cv = 0;  // mixed-radix windows: default shapes only
    used_row_variant = rv ? rv : 1;
    used_col_variant = cv ? cv : 1;
    TOTEM_TRY(slice_loop(o.path, batch, cv, o.t_storage, &launches, &batch_used, rv));
  }
  else has_result = true;
  TOTEM_CUDA(cudaEventRecord(ev[2], stream));
  profiling = false;
  timing = TotemTiming{};
  timing.kernel_launches = launches;
  timing.batch = batch_used;
  timing.probe_slices = (what == 0) ? (long long)w_num * depth * slices : 0;
  timing.h2d_bytes = h2d_bytes;
  timing.slice_path = ran_slice_path;
  timing.tx_fft_path = ran_tx_fft;
  timing.tx_builder = ran_tx_builder;
  timing.row_variant = (what == 0 && ran_slice_path == TOTEM_PATH_FUSED) ? used_row_variant : 0;
  timing.col_variant = (what == 0 && ran_slice_path == TOTEM_PATH_FUSED) ? used_col_variant : 0;
  timing_pending = true;
  return Status::Ok();
}

Status totem_session::collect_timing() {
  if (!timing_pending) return Status::Ok();
  TOTEM_CUDA(cudaStreamSynchronize(stream));
  TOTEM_CUDA(cudaEventElapsedTime(&timing.transmission_ms, ev[0], ev[1]));
  TOTEM_CUDA(cudaEventElapsedTime(&timing.slice_loop_ms, ev[1], ev[2]));
  TOTEM_CUDA(cudaEventElapsedTime(&timing.total_ms, ev[0], ev[2]));
  for (size_t i = 0; i < pkind.size(); ++i) {
    float ms = 0.f;
    TOTEM_CUDA(cudaEventElapsedTime(&ms, pev[2 * i], pev[2 * i + 1]));
    if (pkind[i] == 0) {
      timing.row_pass_ms += ms;
      ++timing.row_pass_launches;
    } else {
      timing.col_pass_ms += ms;
      ++timing.col_pass_launches;
    }
  }
  timing_pending = false;
  return Status::Ok();
}

Status totem_session::download(TotemStemOut* out) {
  if (!has_result) return Status::Err(TOTEM_ERR_STATE, "no result to download");
  TOTEM_CUDA(cudaSetDevice(device));
  TOTEM_TRY(collect_timing());
  if (out == nullptr) return Status::Ok();
  const size_t ad = (size_t)aper_num * depth;
  long long d2h = 0;
  if (last_what == 0) {
    if (out->result && ad) {
      TOTEM_CUDA(cudaMemcpy(out->result, out_result.p, ad * sizeof(double), cudaMemcpyDeviceToHost));
      d2h += (long long)(ad * sizeof(double));
    }
    if (out->mid_layer_mat && ad * mid_layer.size()) {
      TOTEM_CUDA(cudaMemcpy(out->mid_layer_mat, out_mid.p, ad * mid_layer.size() * sizeof(double),
                            cudaMemcpyDeviceToHost));
      d2h += (long long)(ad * mid_layer.size() * sizeof(double));
    }
  }
  if ((out->potential_re || out->potential_im) && t_valid && slices > 0) {
    const size_t n = (size_t)p_h * p_w * slices;
    std::vector<float2> t(n);
    TOTEM_CUDA(cudaMemcpy(t.data(), T.p, n * sizeof(float2), cudaMemcpyDeviceToHost));
    d2h += (long long)(n * sizeof(float2));
    for (size_t i = 0; i < n; ++i) {
      if (out->potential_re) out->potential_re[i] = t[i].x;
      if (out->potential_im) out->potential_im[i] = t[i].y;
    }
  }
  d2h_bytes = d2h;
  timing.d2h_bytes = d2h;
  return Status::Ok();
}

// ---------------------------------------------------------------------------------------------
// Device choice and the cached default sessions used by the one-shot entry points
// ---------------------------------------------------------------------------------------------
Status totem::pick_device(int* dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return Status::Err(TOTEM_ERR_NO_DEVICE, "no CUDA device visible");
  if (*dev >= 0) {
    if (*dev >= n) return Status::Err(TOTEM_ERR_INVALID_ARG, "device index out of range");
    return Status::Ok();
  }
  size_t best = 0;
  int bi = 0;
  for (int i = 0; i < n; ++i) {  // most free memory, as cuda_source_lobato.cu:1071-1081
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(i) == cudaSuccess && cudaMemGetInfo(&fr, &tot) == cudaSuccess && fr > best) {
      best = fr;
      bi = i;
    }
  }
  *dev = bi;
  return Status::Ok();
}

Status totem::create_session(int device, void* stream, totem_session** out) {
  TOTEM_TRY(pick_device(&device));
  TOTEM_CUDA(cudaSetDevice(device));
  std::unique_ptr<totem_session> s(new totem_session());
  s->device = device;
  if (stream) {
    s->stream = (cudaStream_t)stream;
  } else {
    TOTEM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  *out = s.release();
  return Status::Ok();
}

namespace {

using totem::create_session;
using totem::pick_device;

std::mutex g_default_mu;
std::map<int, totem_session*> g_default;  // device -> session kept for the one-shot calls

Status default_session(totem_session** out) {
  int dev = -1;
  if (const char* e = std::getenv("TOTEM_DEVICE")) dev = std::atoi(e);
  TOTEM_TRY(pick_device(&dev));
  std::lock_guard<std::mutex> lk(g_default_mu);
  auto it = g_default.find(dev);
  if (it != g_default.end()) {
    *out = it->second;
    return Status::Ok();
  }
  totem_session* s = nullptr;
  TOTEM_TRY(create_session(dev, nullptr, &s));
  g_default[dev] = s;
  *out = s;
  return Status::Ok();
}

template <class F>
int guarded(F&& f) {
  try {
    Status s = f();
    if (!s.ok()) return fail(s);
    g_last_error.clear();
    return TOTEM_OK;
  } catch (const std::bad_alloc&) {
    return fail(Status::Err(TOTEM_ERR_OOM, "host allocation failed"));
  } catch (const std::exception& e) {
    return fail(Status::Err(TOTEM_ERR_CUDA, e.what()));
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
extern "C" {

int totem_abi_version(void) { return TOTEM_ABI_VERSION; }

int totem_fp32_peak(int device, double* ffma_tflops, double* ffma2_tflops) {
  if (!ffma_tflops || !ffma2_tflops) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "output pointer is NULL"));
  return guarded([&]() -> Status {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return Status::Err(TOTEM_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= count) return Status::Err(TOTEM_ERR_INVALID_ARG, "device index out of range");
    return totem::measure_fma_rates(device, ffma_tflops, ffma2_tflops);
  });
}

const char* totem_status_string(int status) {
  switch (status) {
    case TOTEM_OK: return "ok";
    case TOTEM_ERR_INVALID_ARG: return "invalid argument";
    case TOTEM_ERR_UNSUPPORTED: return "unsupported";
    case TOTEM_ERR_CUDA: return "CUDA error";
    case TOTEM_ERR_CUFFT: return "cuFFT error";
    case TOTEM_ERR_OOM: return "out of memory";
    case TOTEM_ERR_NO_DEVICE: return "no CUDA device";
    case TOTEM_ERR_STATE: return "invalid call sequence";
    case TOTEM_ERR_TIMEOUT: return "timed out";
  }
  return "unknown status";
}

const char* totem_last_error(void) { return g_last_error.c_str(); }

int totem_session_create(int device, void* stream, totem_session** out) {
  if (!out) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "out is NULL"));
  return guarded([&] { return create_session(device, stream, out); });
}

int totem_session_destroy(totem_session* s) {
  if (!s) return TOTEM_OK;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  delete s;
  return TOTEM_OK;
}

int totem_session_upload(totem_session* s, const TotemStemArgs* args) {
  if (!s) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "session is NULL"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&]() -> Status {
    TOTEM_CUDA(cudaSetDevice(s->device));
    return s->upload_args(args, true);
  });
}

int totem_session_run(totem_session* s, int what, const TotemRunOptions* opt) {
  if (!s) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "session is NULL"));
  if (what != 0 && what != 1) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "what must be 0 or 1"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&] { return s->run(what, opt); });
}

int totem_session_download(totem_session* s, TotemStemOut* out) {
  if (!s) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "session is NULL"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&] { return s->download(out); });
}

int totem_session_timing(totem_session* s, TotemTiming* t) {
  if (!s || !t) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&]() -> Status {
    TOTEM_CUDA(cudaSetDevice(s->device));
    TOTEM_TRY(s->collect_timing());
    *t = s->timing;
    return Status::Ok();
  });
}

int totem_session_transmission(totem_session* s, void** ptr) {
  if (!s || !ptr) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  if (!s->t_valid) return fail(Status::Err(TOTEM_ERR_STATE, "no transmission built"));
  *ptr = s->T.p;
  return TOTEM_OK;
}

int totem_session_hrtem(totem_session* s, const TotemHrtemArgs* h, TotemHrtemOut* out) {
  if (!s) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "session is NULL"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&] { return s->hrtem(h, out); });
}

int totem_hrtem_run(const TotemStemArgs* specimen, const TotemHrtemArgs* h, TotemHrtemOut* out) {
  return guarded([&]() -> Status {
    totem_session* s = nullptr;
    TOTEM_TRY(default_session(&s));
    std::lock_guard<std::mutex> lk(s->mu);
    TOTEM_CUDA(cudaSetDevice(s->device));
    TOTEM_TRY(s->upload_args(specimen, false));
    return s->hrtem(h, out);
  });
}

int totem_session_cbed(totem_session* s, double* pattern) {
  if (!s) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "session is NULL"));
  std::lock_guard<std::mutex> lk(s->mu);
  return guarded([&] { return s->cbed(pattern); });
}

int totem_cbed_run(const TotemStemArgs* args, double* pattern) {
  return guarded([&]() -> Status {
    totem_session* s = nullptr;
    TOTEM_TRY(default_session(&s));
    std::lock_guard<std::mutex> lk(s->mu);
    TOTEM_CUDA(cudaSetDevice(s->device));
    TOTEM_TRY(s->upload_args(args, true));
    return s->cbed(pattern);
  });
}

int totem_stem_run(const TotemStemArgs* args, const TotemRunOptions* opt, TotemStemOut* out) {
  return guarded([&]() -> Status {
    totem_session* s = nullptr;
    TOTEM_TRY(default_session(&s));
    std::lock_guard<std::mutex> lk(s->mu);
    TOTEM_CUDA(cudaSetDevice(s->device));
    TOTEM_TRY(s->upload_args(args, true));
    TOTEM_TRY(s->run(0, opt));
    return s->download(out);
  });
}

int totem_set_tx_builder(int mode, size_t scratch_bytes) {
  if (mode != TOTEM_TX_AUTO && mode != TOTEM_TX_DIRECT && mode != TOTEM_TX_GRIDDING)
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "unknown transmission builder mode"));
  g_tx_mode.store(mode);
  g_tx_scratch.store(scratch_bytes);
  g_last_error.clear();
  return TOTEM_OK;
}

int totem_set_slice_graphs(int enable) {
  if (enable != 0 && enable != 1) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "enable must be 0 or 1"));
  g_slice_graphs.store(enable);
  g_last_error.clear();
  return TOTEM_OK;
}

int totem_load_tuning(const char* path, int* entries) {
  return guarded([&]() -> Status {
    std::vector<TuneEntry> t;
    if (path && *path) TOTEM_TRY(read_tuning(path, &t));
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune = std::move(t);
    g_tune_loaded = true;
    if (entries) *entries = (int)g_tune.size();
    return Status::Ok();
  });
}

int totem_tuned_config(int device, int n, int* row_variant, int* col_variant, long long* batch_bytes) {
  if (!row_variant || !col_variant || !batch_bytes || n <= 0)
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "invalid tuned-config arguments"));
  return guarded([&]() -> Status {
    TOTEM_TRY(totem::pick_device(&device));
    *row_variant = 1;
    *col_variant = 1;
    *batch_bytes = 4ll << 30;
    TuneEntry e;
    if (tuned_entry(device, n, &e)) {
      if (e.row_variant) *row_variant = e.row_variant;
      if (e.col_variant) *col_variant = e.col_variant;
      if (e.batch_bytes) *batch_bytes = e.batch_bytes;
    }
    return Status::Ok();
  });
}

int totem_inject_failures(long long alloc_after, int prepare_every) {
  if (alloc_after < -1 || prepare_every < 0)
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "alloc_after must be >= -1 and prepare_every >= 0"));
  g_fail_alloc_after.store(alloc_after);
  g_fail_prepare_every.store(prepare_every);
  g_prepares.store(0);
  g_last_error.clear();
  return TOTEM_OK;
}

int totem_set_band_skip(int enable) {
  if (enable != 0 && enable != 1) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "enable must be 0 or 1"));
  g_band_skip.store(enable);
  g_last_error.clear();
  return TOTEM_OK;
}

int totem_grid_batches(const int* job_beg, int slices, int jobs_per_batch, int* out, int max_batches, int* count) {
  if (!job_beg || !out || !count || slices < 0 || jobs_per_batch < 1 || max_batches < 0)
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "invalid batch-plan arguments"));
  for (int s = 0; s < slices; ++s)
    if (job_beg[s + 1] < job_beg[s] || job_beg[0] != 0)
      return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "job_beg is not a prefix sum from 0"));
  const auto b = totem::grid_batches(std::vector<int>(job_beg, job_beg + slices + 1), jobs_per_batch);
  *count = (int)b.size();
  for (int i = 0; i < (int)b.size() && i < max_batches; ++i) {
    out[4 * i] = b[i].s_lo;
    out[4 * i + 1] = b[i].s_hi;
    out[4 * i + 2] = b[i].j_lo;
    out[4 * i + 3] = b[i].j_hi;
  }
  g_last_error.clear();
  return TOTEM_OK;
}

int totem_transmission_run(const TotemStemArgs* args, TotemStemOut* out) {
  return guarded([&]() -> Status {
    totem_session* s = nullptr;
    TOTEM_TRY(default_session(&s));
    std::lock_guard<std::mutex> lk(s->mu);
    TOTEM_CUDA(cudaSetDevice(s->device));
    TOTEM_TRY(s->upload_args(args, false));
    TOTEM_TRY(s->run(1, nullptr));
    return s->download(out);
  });
}

}  // extern "C"
