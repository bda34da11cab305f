// Plain slice loop: cuFFT batched transforms plus one element-wise kernel per step.
//
// This is the comparator the fused path is timed against; its steps mirror the reference's
// sequence (cuda_source_lobato.cu:1304-1458): initKernel_W, w_p_pointMul, FFT, w_constM_pointMul,
// [mid detectors], IFFT, scaler, ..., final FFT, detectors.  Plans are cached by the engine and
// nothing synchronises between launches.  The same kernels (plus the transfer-function multiply
// and the image sum below) carry HRTEM on grids the fused passes do not take.
#include "common.cuh"

namespace totem {

namespace {

__global__ void k_plain_init(float2* __restrict__ psi, const float2* __restrict__ probe, int vol, int items,
                             int item0, int depth) {
  const long total = (long)items * vol;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int item = (int)(i / vol), e = (int)(i % vol);
    const int w = (item0 + item) / depth;
    psi[i] = probe[(long)w * vol + e];
  }
}

__global__ void k_plain_gather_mul(float2* __restrict__ psi, const float2* __restrict__ tslice, int h, int w,
                                   int items, int item0, ScanGeom geo) {
  const long vol = (long)h * w, total = items * vol;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int item = (int)(i / vol);
    const int e = (int)(i % vol), r = e / w, c = e % w;
    const int pos = (item0 + item) % geo.depth;
    const int x0 = geo.begin_row + (pos / geo.width_red) * geo.step;
    const int y0 = geo.begin_col + (pos % geo.width_red) * geo.step;
    const float2 t = tslice[(long)(x0 + r) * geo.p_width + y0 + c];
    const float2 v = psi[i];
    psi[i] = make_float2(v.x * t.x - v.y * t.y, v.x * t.y + v.y * t.x);
  }
}

__global__ void k_plain_mul(float2* __restrict__ psi, const float2* __restrict__ m, int vol, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const float2 t = m[i % vol];
    const float2 v = psi[i];
    psi[i] = make_float2(v.x * t.x - v.y * t.y, v.x * t.y + v.y * t.x);
  }
}

__global__ void k_plain_scale(float2* __restrict__ psi, float s, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const float2 v = psi[i];
    psi[i] = make_float2(v.x * s, v.y * s);
  }
}

// grid (nblk, items): block b of item sums its contiguous chunk for every detector.
__global__ void k_plain_detect(const float2* __restrict__ psi, const float* __restrict__ masks, int aper_num,
                               int vol, double* __restrict__ part, int nblk) {
  __shared__ double red[32];
  const int item = blockIdx.y, b = blockIdx.x;
  const int chunk = (vol + nblk - 1) / nblk;
  const int e0 = b * chunk, e1 = min(vol, e0 + chunk);
  const float2* p = psi + (long)item * vol;
  for (int a = 0; a < aper_num; ++a) {
    double acc = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      const float2 v = p[e];
      acc += (double)fmaf(v.x, v.x, v.y * v.y) * (double)masks[(long)a * vol + e];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
      part[((long)item * aper_num + a) * nblk + b] = s;
    }
  }
}

__global__ void k_plain_tf_mul(float2* __restrict__ work, const float2* __restrict__ spec,
                               const float2* __restrict__ tf, int vol, long total) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const float2 v = spec[i % vol], t = tf[i];
    work[i] = make_float2(v.x * t.x - v.y * t.y, v.x * t.y + v.y * t.x);
  }
}

__global__ void k_plain_image(const float2* __restrict__ work, int planes, const double* __restrict__ w, float s,
                              int vol, float* __restrict__ out) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < vol; e += (long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int k = 0; k < planes; ++k) {
      const float2 v = work[(long)k * vol + e];
      const float ux = v.x * s, uy = v.y * s;
      acc = fmaf((float)w[k], fmaf(ux, ux, uy * uy), acc);
    }
    out[e] = acc;
  }
}

// CBED pattern: out[r][c] = sum_w gfsf[w] |spec_w[(r + h/2) % h][(c + w/2) % w]|^2 (fftshift of the
// kept spectra, FP64, probes in ascending order).
__global__ void k_cbed_pattern(const float2* __restrict__ spec, const double* __restrict__ gfsf, int w_num, int h,
                               int w, double* __restrict__ out) {
  const long vol = (long)h * w;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < vol; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / w), c = (int)(i % w);
    const long src = (long)((r + h / 2) % h) * w + (c + w / 2) % w;
    double acc = 0.0;
    for (int q = 0; q < w_num; ++q) {
      const float2 v = spec[(long)q * vol + src];
      acc += gfsf[q] * ((double)v.x * v.x + (double)v.y * v.y);
    }
    out[i] = acc;
  }
}

inline int grid_for(long total) { return (int)std::min<long>((total + 255) / 256, 148L * 32); }

}  // namespace

Status launch_plain_init(float2* psi, const float2* probe, int h, int w, int items, int item0, int depth,
                         cudaStream_t st) {
  const long total = (long)items * h * w;
  k_plain_init<<<grid_for(total), 256, 0, st>>>(psi, probe, h * w, items, item0, depth);
  return cuda_status(cudaGetLastError(), "k_plain_init");
}

Status launch_plain_gather_mul(float2* psi, const float2* tslice, int h, int w, int items, int item0, ScanGeom geo,
                               cudaStream_t st) {
  const long total = (long)items * h * w;
  k_plain_gather_mul<<<grid_for(total), 256, 0, st>>>(psi, tslice, h, w, items, item0, geo);
  return cuda_status(cudaGetLastError(), "k_plain_gather_mul");
}

Status launch_plain_mul(float2* psi, const float2* m, int vol, int items, cudaStream_t st) {
  const long total = (long)items * vol;
  k_plain_mul<<<grid_for(total), 256, 0, st>>>(psi, m, vol, total);
  return cuda_status(cudaGetLastError(), "k_plain_mul");
}

Status launch_plain_scale(float2* psi, float s, long total, cudaStream_t st) {
  k_plain_scale<<<grid_for(total), 256, 0, st>>>(psi, s, total);
  return cuda_status(cudaGetLastError(), "k_plain_scale");
}

Status launch_plain_detect(const float2* psi, const float* masks, int aper_num, int vol, int items, double* part,
                           int nblk, cudaStream_t st) {
  if (items == 0 || aper_num == 0) return Status::Ok();
  dim3 grid(nblk, items);
  k_plain_detect<<<grid, 256, 0, st>>>(psi, masks, aper_num, vol, part, nblk);
  return cuda_status(cudaGetLastError(), "k_plain_detect");
}

Status launch_plain_tf_mul(float2* work, const float2* spec, const float2* tf, int vol, int planes, cudaStream_t st) {
  const long total = (long)planes * vol;
  if (total == 0) return Status::Ok();
  k_plain_tf_mul<<<grid_for(total), 256, 0, st>>>(work, spec, tf, vol, total);
  return cuda_status(cudaGetLastError(), "k_plain_tf_mul");
}

Status launch_plain_image(const float2* work, int planes, const double* w, float s, int vol, float* out,
                          cudaStream_t st) {
  if (vol == 0) return Status::Ok();
  k_plain_image<<<grid_for(vol), 256, 0, st>>>(work, planes, w, s, vol, out);
  return cuda_status(cudaGetLastError(), "k_plain_image");
}

Status launch_cbed_pattern(const float2* spec, const double* gfsf, int w_num, int h, int w, double* out,
                           cudaStream_t st) {
  const long vol = (long)h * w;
  if (vol == 0) return Status::Ok();
  k_cbed_pattern<<<grid_for(vol), 256, 0, st>>>(spec, gfsf, w_num, h, w, out);
  return cuda_status(cudaGetLastError(), "k_cbed_pattern");
}

}  // namespace totem
