// Transfer functions of the probe / image (WholeTCC2D_newTEM, ToTEM_submit_v1.m:2305-2406) on the
// device, in FP64.  The reference evaluates them in MATLAB for every request; at 1024^2 the
// aberration gradient alone is seconds of host time, here it is one elementwise kernel.
//
// Per pixel of the centred grid (u, v) = (ax[c], ax[r]), ax[i] = (i - half + 1) / (dx n),
// half = round((n + 1) / 2):
//   W   = Re((A1x + i A1y) w~^2) / 2 + C1 |w|^2 / 2 + W_residual   (w = lambda (u + i v))
//   es  = exp(-alpha^2 pi^2 / lambda^2 (gu^2 + gv^2)),  (gu, gv) = grad W without C1 + C1 lambda (u, v)
//   tcc_m = es * exp(-i pi (m - (M+1)/2) delta (u^2 + v^2) lambda) * exp(-2 pi i W / lambda)
// The residual and the gradient follow WholeTCC_residual_newTEM (:2263-2299) and the flag == 2
// branch (:2336-2369) term by term, including the reference's asymmetric terms.
#include <math_constants.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace totem {

namespace {

struct Cd {
  double x, y;
};
__device__ __forceinline__ Cd cmk(double x, double y) { return Cd{x, y}; }
__device__ __forceinline__ Cd operator*(Cd a, Cd b) { return Cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ Cd cpow(Cd a, int k) {
  Cd r{1.0, 0.0};
  for (int i = 0; i < k; ++i) r = r * a;
  return r;
}
__device__ __forceinline__ double re_mul(Cd a, Cd b) { return a.x * b.x - a.y * b.y; }

// Aberration coefficients as (x, y) pairs (magnitude in nm, angle negated as the reference does).
struct AbXY {
  double C1, A1x, A1y, A2x, A2y, B2x, B2y, C3, A3x, A3y, S3x, S3y, A4x, A4y, D4x, D4y, B4x, B4y, A5x, A5y, C5, S5x,
      S5y, D5x, D5y;
};

__device__ double residual_w(const AbXY& a, double u, double v, double L) {
  const Cd om = cmk(u * L, v * L), omc = cmk(u * L, -v * L);
  double W = 0.0;
  W += re_mul(cmk(a.A2x / 3, a.A2y / 3), cpow(omc, 3));
  W += re_mul(cmk(a.B2x, a.B2y), cpow(om, 2) * omc);
  W += re_mul(cmk(a.A3x / 4, a.A3y / 4), cpow(omc, 4));
  W += re_mul(omc * cpow(om, 3), cmk(a.S3x, a.S3y));
  W += a.C3 * (cpow(om, 2) * cpow(omc, 2)).x / 4;
  W += re_mul(cmk(a.A4x / 5, a.A4y / 5), cpow(omc, 5));
  W += re_mul(cmk(a.D4x, a.D4y), cpow(om, 4) * omc);
  W += re_mul(cmk(a.B4x, a.B4y), cpow(om, 3) * cpow(omc, 2));
  W += re_mul(cmk(a.A5x / 6, a.A5y / 6), cpow(omc, 6));
  W += re_mul(cpow(om, 4) * cpow(omc, 2), cmk(a.S5x, a.S5y));
  W += a.C5 * (cpow(om, 3) * cpow(omc, 3)).x / 6;
  W += re_mul(cmk(a.D5x, a.D5y), cpow(om, 5) * omc);
  return W;
}

__device__ void gradient_w(const AbXY& a, double u, double v, double L, double& gu, double& gv) {
  const double u2 = u * u, v2 = v * v, u3 = u2 * u, v3 = v2 * v, u4 = u2 * u2, v4 = v2 * v2;
  const double r2 = u2 + v2, L2 = L * L, L3 = L2 * L, L4 = L3 * L, L5 = L4 * L;
  gu = L * (a.A1x * u + a.A1y * v)
     + a.A2x * L2 / 3 * (3 * u2 - 3 * v2) + a.A2y * L2 / 3 * 6 * u * v
     + a.B2x * (3 * u2 + v2) * L2 - a.B2y * L2 * 2 * u * v
     + 0.25 * L3 * (a.A3x * (4 * u3 - 12 * u * v2) + a.A3y * (12 * u2 * v - 4 * v3))
     + L3 * (2 * u * (a.S3x * (u2 - v2) - a.S3y * 2 * u * v) + r2 * (2 * a.S3x * u - 2 * a.S3y * v))
     + a.C3 * L3 * r2 * u
     + 0.2 * L4 * (a.A4x * (5 * u4 + 5 * v4 - 30 * u2 * v2) + a.A4y * (20 * u3 * v - 20 * u * v3))
     + L4 * ((2 * u) * (a.D4x * (u3 - 3 * u * v2) - a.D4y * (3 * u2 * v - v3))
             + r2 * (a.D4x * (3 * u2 - 3 * v2) - a.D4y * 6 * u * v))
     + L4 * (2 * r2 * 2 * u * (a.B4x * u - a.B4y * v) + r2 * r2 * a.B4x)
     + L5 / 6 * (a.A5x * (4 * u3 - 14 * v) * (u2 - v2) + a.A5x * (u4 + v4 - 14 * u * v) * 2 * u
                 - a.A5y * 2 * v * (3 * u4 + 3 * v4 - 10 * u2 * v2)
                 - a.A5y * 2 * v * u * (12 * u3 - 20 * u * v2))
     + L5 * (2 * r2 * 2 * u * (a.S5x * (u2 - v2) - 2 * u * v * a.S5y) + r2 * r2 * (2 * a.S5x * u - 2 * v * a.S5y))
     + L5 / 6 * a.C5 * 3 * r2 * r2 * 2 * u
     + L5 * (2 * u * (a.D5x * (u4 + v4 - 6 * u2 * v2) - a.D5y * 4 * u * v * (u2 - v2))
             + r2 * (a.D5x * (4 * u3 - 12 * u * v2) - a.D5y * (12 * u2 * v - 4 * v3)));
  gv = L * (a.A1y * u - a.A1x * v)
     - a.A3x * L2 / 3 * 6 * u * v + a.A3y * L2 / 3 * (-3 * v2 + 3 * u2)
     + a.B2x * L2 * 2 * u * v - a.B2y * L2 * (u2 + 3 * v2)
     + 0.25 * L3 * (a.A3x * (4 * v3 - 12 * u2 * v) + a.A3y * (4 * u3 - 12 * u * v2))
     + L3 * (2 * v * (a.S3x * (u2 - v2) - a.S3y * 2 * u * v) + r2 * (-2 * a.S3x * v - 2 * a.S3y * u))
     + a.C3 * L3 * r2 * v
     + 0.2 * L4 * (a.A4x * (20 * u * v3 - 20 * u3 * v) + a.A4y * (5 * v4 + 5 * u4 - 30 * u2 * v2))
     + L4 * ((2 * v) * (a.D4x * (u3 - 3 * u * v2) - a.D4y * (3 * u2 * v - v3))
             + r2 * (-a.D4x * 6 * u * v - a.D4y * (3 * u2 - 3 * v2)))
     + L4 * (2 * r2 * 2 * v * (a.B4x * u - a.B4y * v) - r2 * r2 * a.B4y)
     + L5 / 6 * (a.A5x * (4 * v3 - 14 * u) * (u2 - v2) + a.A5x * (u4 + v4 - 14 * u * v) * (-2 * v)
                 - a.A5y * 2 * u * (3 * u4 + 3 * v4 - 10 * u2 * v2)
                 - a.A5y * 2 * v * u * (12 * v3 - 20 * u2 * v))
     + L5 * (2 * r2 * 2 * v * (a.S5x * (u2 - v2) - 2 * u * v * a.S5y) + r2 * r2 * (-2 * a.S5x * v - 2 * u * a.S5y))
     + L5 / 6 * a.C5 * 3 * r2 * r2 * 2 * v
     + L5 * (2 * v * (a.D5x * (u4 + v4 - 6 * u2 * v2) - a.D5y * 4 * u * v * (u2 - v2))
             + r2 * (a.D5x * (4 * v3 - 12 * u2 * v) - a.D5y * (4 * u3 - 12 * u * v2)));
}

__global__ void k_tcc(AbXY a, int n, int half, double dk, double lam, double alpha, int with_gradient, int steps,
                      double delta, double* __restrict__ out_re, double* __restrict__ out_im) {
  const long plane = (long)n * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < plane; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i - (long)r * n);
    const double u = (c - half + 1) * dk, v = (r - half + 1) * dk;
    const double wu = u * lam, wv = v * lam;
    // Re((A1x + i A1y) (wu - i wv)^2) / 2 + C1 (wu^2 + wv^2) / 2 + residual
    const double W = (a.A1x * (wu * wu - wv * wv) + a.A1y * 2 * wu * wv) / 2 + a.C1 * (wu * wu + wv * wv) / 2 +
                     residual_w(a, u, v, lam);
    double gu = 0.0, gv = 0.0;
    if (with_gradient) gradient_w(a, u, v, lam, gu, gv);
    gu += a.C1 * lam * u;
    gv += a.C1 * lam * v;
    const double es = exp(-alpha * alpha * CUDART_PI * CUDART_PI / lam / lam * (gu * gu + gv * gv));
    const double chi = 2 * CUDART_PI * W / lam;
    for (int m = 1; m <= steps; ++m) {
      const double ph = -CUDART_PI * (m - (steps + 1) / 2.0) * delta * (u * u + v * v) * lam - chi;
      double s, co;
      sincos(ph, &s, &co);
      out_re[(m - 1) * plane + i] = es * co;
      out_im[(m - 1) * plane + i] = es * s;
    }
  }
}

}  // namespace

}  // namespace totem

extern "C" int totem_tcc_stack(const TotemAberrations* ab, double lambda_nm, int n, double sampling_a,
                               double alpha_mrad, int with_gradient, int steps, double delta_nm, double* tcc_re,
                               double* tcc_im) {
  using totem::Status;
  auto fail = [](const Status& s) {
    totem::set_last_error(s.msg);
    return s.code;
  };
  if (!ab || !tcc_re || !tcc_im) return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "NULL argument"));
  if (ab->struct_size != (int)sizeof(TotemAberrations))
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "TotemAberrations.struct_size does not match this library"));
  if (n <= 0 || n > 16384 || steps <= 0 || !(sampling_a > 0) || !(lambda_nm > 0))
    return fail(Status::Err(TOTEM_ERR_INVALID_ARG, "sizes or optics out of range"));
  int devs = 0;
  if (cudaGetDeviceCount(&devs) != cudaSuccess || devs == 0)
    return fail(Status::Err(TOTEM_ERR_NO_DEVICE, "no CUDA device visible"));
  const double lam = lambda_nm;
  auto xy = [](double mag, double ang_deg, double& x, double& y) {
    const double a = -ang_deg / 180.0 * CUDART_PI;
    x = mag * cos(a);
    y = mag * sin(a);
  };
  totem::AbXY a{};
  a.C1 = ab->focus;
  xy(ab->A1, ab->phiA1, a.A1x, a.A1y);
  xy(ab->A2, ab->phiA2, a.A2x, a.A2y);
  xy(ab->B2, ab->phiB2, a.B2x, a.B2y);
  a.C3 = ab->Cs;
  xy(ab->A3, ab->phiA3, a.A3x, a.A3y);
  xy(ab->S3, ab->phiS3, a.S3x, a.S3y);
  xy(ab->A4, ab->phiA4, a.A4x, a.A4y);
  xy(ab->D4, ab->phiD4, a.D4x, a.D4y);
  xy(ab->B4, ab->phiB4, a.B4x, a.B4y);
  xy(ab->A5, ab->phiA5, a.A5x, a.A5y);
  a.C5 = ab->C5;
  xy(ab->S5, ab->phiS5, a.S5x, a.S5y);
  xy(ab->D5, ab->phiD5, a.D5x, a.D5y);
  const int half = (int)floor((n + 1) / 2.0 + 0.5);  // MATLAB round((n+1)/2)
  const double dk = 1.0 / (sampling_a * 0.1 * n);
  const size_t bytes = (size_t)steps * n * n * sizeof(double);
  double *dre = nullptr, *dim = nullptr;
  cudaStream_t st = nullptr;
  Status s = totem::cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  if (s.ok()) s = totem::cuda_status(cudaMallocAsync((void**)&dre, bytes, st), "cudaMallocAsync");
  if (s.ok()) s = totem::cuda_status(cudaMallocAsync((void**)&dim, bytes, st), "cudaMallocAsync");
  if (s.ok()) {
    const long plane = (long)n * n;
    const int grid = (int)std::min<long>((plane + 255) / 256, 148L * 8);
    totem::k_tcc<<<grid, 256, 0, st>>>(a, n, half, dk, lam, alpha_mrad * 1e-3, with_gradient, steps, delta_nm, dre,
                                        dim);
    s = totem::cuda_status(cudaGetLastError(), "k_tcc");
  }
  if (s.ok()) s = totem::cuda_status(cudaMemcpyAsync(tcc_re, dre, bytes, cudaMemcpyDeviceToHost, st), "D2H");
  if (s.ok()) s = totem::cuda_status(cudaMemcpyAsync(tcc_im, dim, bytes, cudaMemcpyDeviceToHost, st), "D2H");
  if (dre) cudaFreeAsync(dre, st);
  if (dim) cudaFreeAsync(dim, st);
  if (st) {
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (s.ok()) s = totem::cuda_status(e2, "cudaStreamSynchronize");
    cudaStreamDestroy(st);
  }
  if (!s.ok()) return fail(s);
  return TOTEM_OK;
}
