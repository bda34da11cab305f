// Status helpers and the small conversion kernels used while uploading a request.
#include <cuda_bf16.h>

#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace totem {

Status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return Status::Ok();
  const int code = (e == cudaErrorMemoryAllocation) ? TOTEM_ERR_OOM
                   : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? TOTEM_ERR_NO_DEVICE
                                                                                   : TOTEM_ERR_CUDA;
  return Status::Err(code, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

Status cufft_status(cufftResult r, const char* what) {
  if (r == CUFFT_SUCCESS) return Status::Ok();
  const int code = (r == CUFFT_ALLOC_FAILED) ? TOTEM_ERR_OOM : TOTEM_ERR_CUFFT;
  return Status::Err(code, std::string(what) + ": cufftResult " + std::to_string((int)r));
}

Status ensure_smem(const void* func, size_t bytes) {
  if (bytes <= 48 * 1024) return Status::Ok();
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;  // one entry per (kernel, device)
  int dev = 0;
  TOTEM_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_pair(func, dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return Status::Ok();
  TOTEM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done[key] = bytes;
  return Status::Ok();
}

namespace {

__global__ void k_d2f2(const double* __restrict__ re, const double* __restrict__ im, float2* __restrict__ out,
                       long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = make_float2((float)re[i], im ? (float)im[i] : 0.f);
}

__global__ void k_d2f(const double* __restrict__ in, float* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

// out[a][r][c] = aper[a][(r + shift) % h][(c + shift') % w]; shift = 1 gives ifftshift for even
// sizes (the quadrant swap the reference applies to the exit wave, cuda_source_lobato.cu:210-253).
__global__ void k_shift_masks(const double* __restrict__ aper, float* __restrict__ out, int aper_num, int h, int w,
                              int shift) {
  const long total = (long)aper_num * h * w;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int a = (int)(i / ((long)h * w));
    const int e = (int)(i % ((long)h * w)), r = e / w, c = e % w;
    const int rs = shift ? (r + h / 2) % h : r, cs = shift ? (c + w / 2) % w : c;
    out[i] = (float)aper[(long)a * h * w + (long)rs * w + cs];
  }
}

__global__ void k_to_bf16(const float2* __restrict__ in, __nv_bfloat162* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = __float22bfloat162_rn(in[i]);
}

inline int grid_for(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 16); }

}  // namespace

Status launch_d2f2(const double* re, const double* im, float2* out, long n, cudaStream_t st) {
  if (n == 0) return Status::Ok();
  k_d2f2<<<grid_for(n), 256, 0, st>>>(re, im, out, n);
  return cuda_status(cudaGetLastError(), "k_d2f2");
}

Status launch_d2f(const double* in, float* out, long n, cudaStream_t st) {
  if (n == 0) return Status::Ok();
  k_d2f<<<grid_for(n), 256, 0, st>>>(in, out, n);
  return cuda_status(cudaGetLastError(), "k_d2f");
}

Status launch_shift_masks(const double* aper, float* out, int aper_num, int h, int w, int shift, cudaStream_t st) {
  const long n = (long)aper_num * h * w;
  if (n == 0) return Status::Ok();
  k_shift_masks<<<grid_for(n), 256, 0, st>>>(aper, out, aper_num, h, w, shift);
  return cuda_status(cudaGetLastError(), "k_shift_masks");
}

Status launch_to_bf16(const float2* in, void* out, long n, cudaStream_t st) {
  if (n == 0) return Status::Ok();
  k_to_bf16<<<grid_for(n), 256, 0, st>>>(in, static_cast<__nv_bfloat162*>(out), n);
  return cuda_status(cudaGetLastError(), "k_to_bf16");
}

namespace {

// FP32 FMA throughput: every thread runs kFmaChains independent chains a = a * m + c, scalar (FFMA)
// or on packed pairs (FFMA2, __ffma2_rn, two FMAs per instruction); with m = 0.999, c = 0.001 the
// values stay near 1.  The sum is stored so that nothing is dead code.
constexpr int kFmaChains = 8;

__global__ void k_fma_rate(float* __restrict__ out, int iters) {
  float a[kFmaChains];
#pragma unroll
  for (int i = 0; i < kFmaChains; ++i) a[i] = 1.f + 1e-3f * i + 1e-7f * threadIdx.x;
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int i = 0; i < kFmaChains; ++i) a[i] = fmaf(a[i], 0.999f, 0.001f);
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < kFmaChains; ++i) s += a[i];
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_fma2_rate(float* __restrict__ out, int iters) {
  float2 a[kFmaChains];
#pragma unroll
  for (int i = 0; i < kFmaChains; ++i) a[i] = make_float2(1.f + 1e-3f * i, 1.f - 1e-3f * i + 1e-7f * threadIdx.x);
  const float2 m = make_float2(0.999f, 0.999f), c = make_float2(0.001f, 0.001f);
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int i = 0; i < kFmaChains; ++i) a[i] = __ffma2_rn(a[i], m, c);
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < kFmaChains; ++i) s += a[i].x + a[i].y;
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

Status measure_fma_rates(int device, double* ffma_tflops, double* ffma2_tflops) {
  int previous = 0;
  TOTEM_CUDA(cudaGetDevice(&previous));
  struct Restore {  // the caller's current device is left as it was, on every return
    int dev;
    ~Restore() { cudaSetDevice(dev); }
  } restore{previous};
  TOTEM_CUDA(cudaSetDevice(device));
  int sms = 0;
  TOTEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  constexpr int threads = 256, per_sm = 8, iters = 1 << 16;
  const int blocks = sms * per_sm;
  float* out = nullptr;
  TOTEM_CUDA(cudaMalloc(&out, sizeof(float) * blocks * threads));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto rate = [&](bool packed, double* tflops) -> Status {
    float best = 0.f;
    for (int rep = 0; rep < 4; ++rep) {  // the first launch is the warm-up
      TOTEM_CUDA(cudaEventRecord(e0));
      if (packed) k_fma2_rate<<<blocks, threads>>>(out, iters);
      else k_fma_rate<<<blocks, threads>>>(out, iters);
      TOTEM_CUDA(cudaGetLastError());
      TOTEM_CUDA(cudaEventRecord(e1));
      TOTEM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      TOTEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    const double fmas = (double)blocks * threads * iters * kFmaChains * (packed ? 2 : 1);
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
    return Status::Ok();
  };
  Status st = rate(false, ffma_tflops);
  if (st.ok()) st = rate(true, ffma2_tflops);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return st;
}

}  // namespace totem
