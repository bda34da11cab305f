// Allocation-free variant of the fused slice loop (totem_stem_slices_noalloc).
//
// Some callers cannot allocate device memory themselves: code that runs inside a host framework
// whose GPU memory is owned by that framework's pool (a MEX function under MATLAB's GPU memory
// manager, an operator inside a PyTorch pipeline that must not bypass the caching allocator),
// serving loops that cannot afford cudaMalloc / cudaFree because they synchronise the whole
// device and stall the other streams, and embedded deployments with a fixed, pre-planned memory
// budget.  For them this entry point takes device-resident inputs and outputs and keeps every
// intermediate buffer in one file-scope device array of fixed size, so the library never calls
// cudaMalloc, cudaFree or an allocating library routine on this path.
//
// Properties callers must know:
//  * the array is NOALLOC_SCRATCH_BYTES (32 MiB) and exists on every GPU that loads this
//    library, for the life of the process;
//  * the first call on a device does a one-time set-up with that device current: it looks up
//    the array's device address (cudaGetSymbolAddress) and copies the FFT twiddle tables into it
//    with a blocking copy.  Make that first call before any stream capture.  The set-up belongs
//    to the device's current CUDA context: it is done again when another context becomes
//    current on that device (after cudaDeviceReset, or a caller's own driver-API context);
//  * windows of 64^2 .. 1024^2: one 2048^2 probe alone (32 MiB) would fill the whole array;
//  * every call uses the same array and leaves its contents behind; two calls that overlap on
//    the GPU (different streams, or different host threads without ordering) race on it.
//    Everything a call reads from the array it has written itself first in stream order, so
//    back-to-back calls on one stream are independent.
#include <cuda.h>  // driver-API types of the two context queries looked up through the runtime

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 32ull << 20;  // 32 MiB per GPU
constexpr size_t NOALLOC_TW_BYTES = 64u << 10;         // twiddle tables of N = 64 .. 1024
constexpr int NOALLOC_MAX_N = 1024;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct DeviceScratch {
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch on that device
  size_t tw_offset[12] = {};      // byte offset of the twiddle table of N = 2^k
  unsigned long long context = 0; // id of the context the address and the tables belong to
};

std::mutex g_setup_mu;
DeviceScratch g_dev[NOALLOC_MAX_DEVICES];
bool g_ready[NOALLOC_MAX_DEVICES] = {};

// Id of the calling thread's current CUDA context, unique for the life of the process
// (cuCtxGetId), or 0 when no context is current.  The two driver functions are looked up through
// the runtime once, so the library keeps no link-time dependency on the driver library.
unsigned long long current_context_id() {
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    void* f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c != nullptr && get_id(c, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

int log2i(int n) {
  int k = 0;
  while ((1 << k) < n) ++k;
  return k;
}

// Set-up on the current device, once per device and context: device address of the array,
// twiddle tables.
totem::Status setup(int dev, DeviceScratch** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return totem::Status::Err(TOTEM_ERR_UNSUPPORTED, "device index too large");
  const unsigned long long ctx = current_context_id();
  if (!g_ready[dev] || ctx == 0 || ctx != g_dev[dev].context) {
    g_ready[dev] = false;
    DeviceScratch d;
    void* p = nullptr;
    TOTEM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // makes the device's context current
    d.base = static_cast<unsigned char*>(p);
    d.context = current_context_id();
    size_t off = 0;
    for (int n = 64; n <= NOALLOC_MAX_N; n *= 2) {
      const std::vector<float2> tw = totem::stage_twiddles(n);
      const size_t bytes = tw.size() * sizeof(float2);
      if (off + bytes > NOALLOC_TW_BYTES) return totem::Status::Err(TOTEM_ERR_UNSUPPORTED, "twiddle region too small");
      TOTEM_CUDA(cudaMemcpy(d.base + off, tw.data(), bytes, cudaMemcpyHostToDevice));
      d.tw_offset[log2i(n)] = off;
      off += (bytes + 255) & ~size_t(255);
    }
    g_dev[dev] = d;
    g_ready[dev] = true;
  }
  *out = &g_dev[dev];
  return totem::Status::Ok();
}

totem::Status run(const void* transmission, int p_height, int p_width, int slices, const void* probe, int w_num,
                  const void* propagator, const float* masks, int aper_num, int n, int step, int begin_row,
                  int begin_col, int width_red, int depth, int item0, int items, double* result, void* stream) {
  using totem::Status;
  if (!transmission || !probe || !propagator || !masks || !result)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "NULL device pointer");
  if (n < 64 || n > NOALLOC_MAX_N || (n & (n - 1)))
    return Status::Err(TOTEM_ERR_UNSUPPORTED,
                       "window edge must be a power of two in [64, 1024] (one 2048^2 probe needs more than the "
                       "fixed scratch array)");
  if (slices < 1) return Status::Err(TOTEM_ERR_INVALID_ARG, "slices must be >= 1");
  if (aper_num < 1 || aper_num > 32) return Status::Err(TOTEM_ERR_INVALID_ARG, "aper_num must be in [1, 32]");
  if (w_num < 1 || depth < 1 || width_red < 1 || step < 0 || items < 1 || item0 < 0 ||
      (long long)item0 + items > (long long)w_num * depth)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "item range, depth, width_red or step out of range");
  const long last = depth - 1;
  const long rmax = begin_row + (last / width_red) * (long)step;
  const long cmax = begin_col + (long)std::min<long>(last, width_red - 1) * step;
  if (begin_row < 0 || begin_col < 0 || rmax + n > p_height || cmax + n > p_width)
    return Status::Err(TOTEM_ERR_INVALID_ARG, "probe windows leave the potential grid");
  const int nblk = totem::col_blocks(n);
  const size_t psi_bytes = (size_t)items * n * n * sizeof(float2);
  const size_t part_bytes = (size_t)items * aper_num * nblk * sizeof(double);
  const size_t need = NOALLOC_TW_BYTES + ((psi_bytes + 255) & ~size_t(255)) + part_bytes;
  if (need > NOALLOC_SCRATCH_BYTES) {
    const size_t per_item = (size_t)n * n * sizeof(float2) + (size_t)aper_num * nblk * sizeof(double);
    const size_t max_items = (NOALLOC_SCRATCH_BYTES - NOALLOC_TW_BYTES - 256) / per_item;
    return Status::Err(TOTEM_ERR_INVALID_ARG,
                       "request needs " + std::to_string(need) + " bytes of scratch, more than the fixed " +
                           std::to_string(NOALLOC_SCRATCH_BYTES) + "; at most " + std::to_string(max_items) +
                           " probes per call for this window and detector count");
  }
  int dev = 0;
  TOTEM_CUDA(cudaGetDevice(&dev));
  DeviceScratch* d = nullptr;
  TOTEM_TRY(setup(dev, &d));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* psi = d->base + NOALLOC_TW_BYTES;
  double* part = reinterpret_cast<double*>(psi + ((psi_bytes + 255) & ~size_t(255)));

  totem::SliceLoopArgs s;
  s.n = n;
  s.items = items;
  s.item0 = item0;
  s.geo = totem::ScanGeom{begin_row, begin_col, step, width_red, depth, p_width};
  s.p_h = p_height;
  s.psi = reinterpret_cast<float2*>(psi);
  s.probe = static_cast<const float2*>(probe);
  s.prop = static_cast<const float2*>(propagator);
  s.tw = reinterpret_cast<const float2*>(d->base + d->tw_offset[log2i(n)]);
  s.aper_num = aper_num;
  s.mask_exit = masks;
  s.part_exit = part;
  const float2* T = static_cast<const float2*>(transmission);
  const size_t plane = (size_t)p_height * p_width;
  TOTEM_TRY(totem::launch_row_pass(s, T, true, st));
  for (int k = 0; k < slices; ++k) {
    const int flags = (k == slices - 1) ? (2 | 4) : 0;
    TOTEM_TRY(totem::launch_col_pass(s, flags, st));
    if (k < slices - 1) TOTEM_TRY(totem::launch_row_pass(s, T + (size_t)(k + 1) * plane, false, st));
  }
  // per-item sums in a fixed order: result[a * items + i]
  return totem::launch_det_reduce(part, nblk, aper_num, items, 0, items, result, st);
}

}  // namespace

static_assert(NOALLOC_SCRATCH_BYTES == TOTEM_NOALLOC_SCRATCH_BYTES, "header and library disagree on the scratch size");

extern "C" int totem_stem_slices_noalloc(const void* transmission, int p_height, int p_width, int slices,
                                         const void* probe, int w_num, const void* propagator, const float* masks,
                                         int aper_num, int n, int step, int begin_row, int begin_col, int width_red,
                                         int depth, int item0, int items, double* result, void* stream) {
  totem::Status s;
  try {
    s = run(transmission, p_height, p_width, slices, probe, w_num, propagator, masks, aper_num, n, step, begin_row,
            begin_col, width_red, depth, item0, items, result, stream);
  } catch (const std::exception& e) {
    s = totem::Status::Err(TOTEM_ERR_CUDA, e.what());
  }
  totem::set_last_error(s.msg);  // readable through totem_last_error()
  return s.code;
}
