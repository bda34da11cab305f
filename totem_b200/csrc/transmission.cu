// Transmission builder: per-slice projected potential in Fourier space, inverse 2-D FFT, and
// T = exp(i * sigma/1000 * V).
//
// Reference: cal_p / initKernel_P (cuda_source_lobato.cu:585-956, cuda_source_peng_and_corr.cu
// :785-1156) and the correction potential p_corr (cuda_source_peng_and_corr.cu:587-779); the CPU
// statement of the same sums is GetPotential4AllSlice_multicore_lotabo_peng(_corr).m.
//
// Differences by design:
//  * one thread owns each pixel's accumulator for all atoms of a slice (the reference launches
//    one thread per (atom, pixel) and adds into the same pixel without atomics,
//    cuda_source_lobato.cu:82-83);
//  * the phase exp(-2 pi i (kx x + ky y)) is reduced modulo one in FP64 before the FP32
//    sincospi (the reference forms the angle in FP32 with pi = 3.14159265, :80-81); on the
//    reference's separable grids the two factors are tabulated per atom and tile;
//  * the ifftshift before the inverse FFT is folded into a (-1)^(r+c) factor after it, and
//    APERTURE is applied while the sum is written.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "fft.cuh"
#include "tx_fft.cuh"

namespace totem {

namespace {

constexpr int TX_TC = 32;      // tile columns (one per lane)
constexpr int TX_PR = 4;       // rows per thread
constexpr int TX_TR = 32;      // tile rows (8 warps x 4)
constexpr int TX_CH = 32;      // atoms staged per chunk
constexpr int TX_MAXC = 24;    // widest coefficient block (ionic Lobato row without x, y)

__device__ __forceinline__ float peng5(const float* c, float s2) {
  float f = 0.f;
#pragma unroll
  for (int i = 0; i < 5; ++i) f = fmaf(c[2 * i], __expf(-c[2 * i + 1] * s2), f);
  return f;
}

__device__ __forceinline__ float lobato5(const float* c, float g2) {
  float f = 0.f;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const float b = c[2 * i + 1];
    const float d = fmaf(b, g2, 1.f);
    f = fmaf(c[2 * i], __fdividef(fmaf(b, g2, 2.f), d * d), f);
  }
  return f;
}

// Form factor of one neutral (kind 0) or ionic (kind 1) coefficient row at s^2: real part fr
// (Peng: occ * sum a_i exp(-b_i s^2); Lobato: occ * sum a_i (2 + b_i g^2) / (1 + b_i g^2)^2 *
// exp(-B s^2), g^2 = 4 s^2; ionic rows mix the ion and atom sums by their fractions) and the
// absorptive imaginary part fi (occ * Peng sum of the absorptive row, or 0).
__device__ __forceinline__ void row_form(int kind, int lobato, const float* cf, const float* absorp, float s2,
                                         float& fr, float& fi) {
  if (kind == 0) {
    if (lobato) fr = cf[0] * lobato5(cf + 1, 4.f * s2) * __expf(-cf[11] * s2);
    else fr = cf[0] * peng5(cf + 1, s2);
  } else {
    if (lobato)
      fr = cf[0] * (cf[1] * lobato5(cf + 2, 4.f * s2) + cf[12] * lobato5(cf + 13, 4.f * s2)) * __expf(-cf[23] * s2);
    else fr = cf[0] * (cf[1] * peng5(cf + 2, s2) + cf[12] * peng5(cf + 13, s2));
  }
  fi = absorp != nullptr ? cf[0] * peng5(absorp, s2) : 0.f;
}

// Form factor of species ``sp`` of kind ``kind`` (SpeciesSet) at pixel ``pix`` (s^2 = s2):
// kinds 0 / 1 as row_form; the Peng-extended correction kinds 2 / 3
// (cuda_source_peng_and_corr.cu:587-779, GetPotential4AllSlice_multicore_lotabo_peng_corr.m:13-60)
// amplitude * exp(-B s^2) * the correction plane(s) at the pixel (planes numbered from 1).
__device__ __forceinline__ void species_form(int kind, const TxGrid& g, const SpeciesDev& d, int sp, float s2,
                                             long pix, float& fr, float& fi) {
  const float* cf = d.coef + (long)sp * d.ncoef;
  if (kind <= 1) {
    row_form(kind, g.lobato, cf, d.absorp != nullptr ? d.absorp + (long)sp * 10 : nullptr, s2, fr, fi);
    return;
  }
  const long plane = (long)g.p_h * g.p_w;
  float m = 0.f;
  if (kind == 2) {
    const int idx = (int)cf[2] - 1;
    if (idx >= 0 && idx < g.cim_len) m = g.cim[idx * plane + pix];
  } else {
    const int i1 = (int)cf[3] - 1, i2 = (int)cf[5] - 1;
    if (i1 >= 0 && i1 < g.cim_len) m = fmaf(cf[2], g.cim[i1 * plane + pix], m);
    if (i2 >= 0 && i2 < g.cim_len) m = fmaf(cf[4], g.cim[i2 * plane + pix], m);
  }
  fr = cf[1] * m * __expf(-cf[0] * s2);
  fi = 0.f;
}

// exp(-2 pi i t) for t given in FP64, reduced to [0, 1) before the FP32 evaluation.
__device__ __forceinline__ float2 phase_of(double t) {
  const double fr = t - floor(t);
  float s, c;
  sincospif(2.f * (float)fr, &s, &c);
  return make_float2(c, -s);
}

struct TxSmem {
  double pos[TX_CH][2];
  float coef[TX_CH][TX_MAXC];
  float absorp[TX_CH][10];
  float2 ex[TX_CH][TX_TC];
  float2 ey[TX_CH][TX_TR];
};

// kind: 0 neutral, 1 ionic, 2 correction (neutral), 3 correction (ionic)
template <bool SEP>
__device__ void accumulate_rows(const TxGrid& g, const AtomRowsDev& rows, int kind, int slice, TxSmem& sm,
                                int tx, int ty, int c, int r0, int c_tile, int r_tile, const float* s2v,
                                const double* kxv, const double* kyv, const int* pix, float2* acc) {
  if (rows.beg == nullptr) return;
  const int a_begin = rows.beg[slice], a_end = rows.beg[slice + 1];
  const long plane = (long)g.p_h * g.p_w;
  for (int a0 = a_begin; a0 < a_end; a0 += TX_CH) {
    const int na = min(TX_CH, a_end - a0);
    __syncthreads();
    for (int e = threadIdx.x; e < na * 2; e += blockDim.x) sm.pos[e >> 1][e & 1] = rows.pos[(long)(a0 + (e >> 1)) * 2 + (e & 1)];
    for (int e = threadIdx.x; e < na * rows.ncoef; e += blockDim.x) {
      const int a = e / rows.ncoef, k = e - a * rows.ncoef;
      sm.coef[a][k] = rows.coef[(long)(a0 + a) * rows.ncoef + k];
    }
    if (rows.absorp != nullptr)
      for (int e = threadIdx.x; e < na * 10; e += blockDim.x) sm.absorp[e / 10][e % 10] = rows.absorp[(long)a0 * 10 + e];
    __syncthreads();
    if (SEP) {
      for (int e = threadIdx.x; e < na * (TX_TC + TX_TR); e += blockDim.x) {
        const int a = e / (TX_TC + TX_TR), k = e - a * (TX_TC + TX_TR);
        if (k < TX_TC) {
          const int cc = min(c_tile + k, g.p_w - 1);
          sm.ex[a][k] = phase_of(g.kx_axis[cc] * sm.pos[a][0]);
        } else {
          const int rr = min(r_tile + k - TX_TC, g.p_h - 1);
          sm.ey[a][k - TX_TC] = phase_of(g.ky_axis[rr] * sm.pos[a][1]);
        }
      }
      __syncthreads();
    }
    for (int a = 0; a < na; ++a) {
      const float* cf = sm.coef[a];
      float2 ex = make_float2(1.f, 0.f);
      if (SEP) ex = sm.ex[a][tx];
#pragma unroll
      for (int i = 0; i < TX_PR; ++i) {
        const float s2 = s2v[i];
        float2 ph;
        if (SEP) ph = cmul(ex, sm.ey[a][ty * TX_PR + i]);
        else ph = phase_of(kxv[i] * sm.pos[a][0] + kyv[i] * sm.pos[a][1]);
        float fr, fi = 0.f;
        if (kind <= 1) {
          row_form(kind, g.lobato, cf, rows.absorp != nullptr ? sm.absorp[a] : nullptr, s2, fr, fi);
        } else if (kind == 2) {
          const int idx = (int)cf[2] - 1;
          const float m = (idx >= 0 && idx < g.cim_len && pix[i] >= 0) ? g.cim[idx * plane + pix[i]] : 0.f;
          fr = cf[1] * m * __expf(-cf[0] * s2);
        } else {
          const int i1 = (int)cf[3] - 1, i2 = (int)cf[5] - 1;
          float m = 0.f;
          if (pix[i] >= 0) {
            if (i1 >= 0 && i1 < g.cim_len) m = fmaf(cf[2], g.cim[i1 * plane + pix[i]], m);
            if (i2 >= 0 && i2 < g.cim_len) m = fmaf(cf[4], g.cim[i2 * plane + pix[i]], m);
          }
          fr = cf[1] * m * __expf(-cf[0] * s2);
        }
        acc[i].x = fmaf(fr, ph.x, fmaf(-fi, ph.y, acc[i].x));
        acc[i].y = fmaf(fr, ph.y, fmaf(fi, ph.x, acc[i].y));
      }
    }
  }
}

template <bool SEP>
__global__ void __launch_bounds__(256) k_tx_structure(TxGrid g, AtomRowsDev nr, AtomRowsDev ir, AtomRowsDev cn,
                                                      AtomRowsDev ci, float2* __restrict__ out, int accumulate) {
  __shared__ TxSmem sm;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int slice = blockIdx.z;
  const int c_tile = blockIdx.x * TX_TC, r_tile = blockIdx.y * TX_TR;
  const int c = c_tile + tx, r0 = r_tile + ty * TX_PR;
  float s2v[TX_PR];
  double kxv[TX_PR], kyv[TX_PR];
  int pix[TX_PR];
  float2 acc[TX_PR];
#pragma unroll
  for (int i = 0; i < TX_PR; ++i) {
    const int r = r0 + i;
    const bool in = (r < g.p_h) && (c < g.p_w);
    pix[i] = in ? r * g.p_w + c : -1;
    s2v[i] = in ? g.s2[pix[i]] : 0.f;
    kxv[i] = (!SEP && in) ? g.kx[pix[i]] : 0.0;
    kyv[i] = (!SEP && in) ? g.ky[pix[i]] : 0.0;
    acc[i] = make_float2(0.f, 0.f);
  }
  accumulate_rows<SEP>(g, nr, 0, slice, sm, tx, ty, c, r0, c_tile, r_tile, s2v, kxv, kyv, pix, acc);
  accumulate_rows<SEP>(g, ir, 1, slice, sm, tx, ty, c, r0, c_tile, r_tile, s2v, kxv, kyv, pix, acc);
  accumulate_rows<SEP>(g, cn, 2, slice, sm, tx, ty, c, r0, c_tile, r_tile, s2v, kxv, kyv, pix, acc);
  accumulate_rows<SEP>(g, ci, 3, slice, sm, tx, ty, c, r0, c_tile, r_tile, s2v, kxv, kyv, pix, acc);
  float2* dst = out + (long)slice * g.p_h * g.p_w;
#pragma unroll
  for (int i = 0; i < TX_PR; ++i) {
    if (pix[i] < 0) continue;
    const float ap = (g.aper_true != nullptr) ? g.aper_true[pix[i]] : 1.f;
    float2 v = cscale(acc[i], g.parameter * ap);
    if (accumulate) v = cadd(dst[pix[i]], v);
    dst[pix[i]] = v;
  }
}

// ---------------------------------------------------------------------------------------------
// By species.  A 256-thread block owns a 64 x 64 pixel tile of one slice; thread (tx, ty) owns the
// 16 pixels (r_tile + ty + 16 i, c_tile + tx + 16 j).  Per species the block accumulates
//   S(r, c) = sum_atoms ey_a(r) * ex_a(c),  ex_a(c) = exp(-2 pi i kx(c) x_a), ey_a(r) likewise,
// a complex rank-K update from per-atom tables staged in shared memory (16 atoms at a time),
// then adds f_species(s^2) * S.  Table entries are stored so that one complex multiply-add is two
// packed FMAs: ex as (re, im, -im, re), ey as (re, re, im, im).
// ---------------------------------------------------------------------------------------------
constexpr int SP_T = 64;
constexpr int SP_CH = 16;

struct SpSmem {
  double pos[SP_CH][2];
  float4 ex[SP_CH][SP_T];
  float4 ey[SP_CH][SP_T];
};

__global__ void __launch_bounds__(256, 2) k_tx_species(TxGrid g, SpeciesSet spset, float2* __restrict__ out) {
  __shared__ SpSmem sm;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int slice = blockIdx.z;
  const int c_tile = blockIdx.x * SP_T, r_tile = blockIdx.y * SP_T;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int kind = 0; kind < 4; ++kind) {
    const SpeciesDev& d = spset.k[kind];
    if (d.seg_beg == nullptr) continue;
    const int s_end = d.seg_beg[slice + 1];
    for (int sidx = d.seg_beg[slice]; sidx < s_end; ++sidx) {
      const int sp = d.seg[3 * sidx], a_begin = d.seg[3 * sidx + 1], a_end = d.seg[3 * sidx + 2];
      float2 S[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) S[i][j] = make_float2(0.f, 0.f);
      for (int a0 = a_begin; a0 < a_end; a0 += SP_CH) {
        const int na = min(SP_CH, a_end - a0);
        __syncthreads();  // previous chunk's tables fully read
        if (threadIdx.x < 2 * na) sm.pos[threadIdx.x >> 1][threadIdx.x & 1] = d.pos[(long)a0 * 2 + threadIdx.x];
        __syncthreads();
        for (int e = threadIdx.x; e < na * 2 * SP_T; e += blockDim.x) {
          const int a = e / (2 * SP_T), k = e - a * (2 * SP_T);
          if (k < SP_T) {
            const int cc = min(c_tile + k, g.p_w - 1);
            const float2 p = phase_of(g.kx_axis[cc] * sm.pos[a][0]);
            sm.ex[a][k] = make_float4(p.x, p.y, -p.y, p.x);
          } else {
            const int rr = min(r_tile + k - SP_T, g.p_h - 1);
            const float2 p = phase_of(g.ky_axis[rr] * sm.pos[a][1]);
            sm.ey[a][k - SP_T] = make_float4(p.x, p.x, p.y, p.y);
          }
        }
        __syncthreads();
#pragma unroll 2
        for (int a = 0; a < na; ++a) {
          float4 exv[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) exv[j] = sm.ex[a][tx + 16 * j];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float4 ey = sm.ey[a][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              S[i][j] = __ffma2_rn(make_float2(ey.x, ey.y), make_float2(exv[j].x, exv[j].y), S[i][j]);
              S[i][j] = __ffma2_rn(make_float2(ey.z, ey.w), make_float2(exv[j].z, exv[j].w), S[i][j]);
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int r = min(r_tile + ty + 16 * i, g.p_h - 1), c = min(c_tile + tx + 16 * j, g.p_w - 1);
          const long pix = (long)r * g.p_w + c;
          float fr, fi;
          species_form(kind, g, d, sp, __ldg(g.s2 + pix), pix, fr, fi);
          acc[i][j].x = fmaf(fr, S[i][j].x, fmaf(-fi, S[i][j].y, acc[i][j].x));
          acc[i][j].y = fmaf(fr, S[i][j].y, fmaf(fi, S[i][j].x, acc[i][j].y));
        }
    }
  }
  float2* dst = out + (long)slice * g.p_h * g.p_w;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r_tile + ty + 16 * i, c = c_tile + tx + 16 * j;
      if (r >= g.p_h || c >= g.p_w) continue;
      const long pix = (long)r * g.p_w + c;
      const float ap = (g.aper_true != nullptr) ? g.aper_true[pix] : 1.f;
      dst[pix] = cscale(acc[i][j], g.parameter * ap);
    }
}

// ---------------------------------------------------------------------------------------------
// By species through Gaussian gridding (a type-1 non-uniform FFT), for uniform separable grids
// kx(c) = kx0 + c dkx, ky(r) = ky0 + r dky.  With kx' = c - p_w/2, ky' = r - p_h/2,
//   S(r, c) = sum_a w_a exp(-i (kx' tx_a + ky' ty_a)),
//   tx_a = 2 pi frac(dkx x_a), ty_a = 2 pi frac(dky y_a),
//   w_a = exp(-2 pi i (kx(p_w/2) x_a + ky(p_h/2) y_a))   (1 on centred grids).
// Each atom is spread with a periodic Gaussian exp(-d^2 / (4 tau)) onto a grid twice as fine as
// the potential (GR_W x GR_W points), the fine grid is transformed, and the Gaussian's transform
// sqrt(pi / tau) exp(-k^2 tau) is divided out: Greengard & Lee, "Accelerating the nonuniform
// fast Fourier transform", SIAM Review 46 (2004) 443-454, with oversampling R = 2, half-width
// M_sp = 7 and tau = pi M_sp / (P^2 R (R - 1/2)).  The relative L2 error of S is ~1e-7 (below
// the FP32 sums) whatever the atom count; the cost is O(atoms + P^2 log P) per species and
// slice instead of O(atoms P^2).
//
// The 2P x 2P fine grid is held as four P x P planes by the parity of its indices, plane
// (ey, ex) = points (2 qy + ey, 2 qx + ex), so its transform is four P x P FFTs and a half-bin
// phase: F(k) = sum_{ey, ex} exp(-i pi (ky ey / p_h + kx ex / p_w)) FFT(plane_{ey,ex})[k mod P].
// The x half of that sum is taken right after the row transforms (the rows of parity ex = 0
// and 1 of a fine row pair share a CTA), together with the x deconvolution, so two planes per
// job, ey = 0 and 1, go through the column transforms and the combine.
// Atoms are added in 32.32 fixed point (64-bit integer atomics), so the grid, and everything
// after it, is bit-reproducible whatever order the atomics land in.  The row pass writes its
// complex64 output in place into the ex = 0 row (the first half of its 16-byte-per-point
// storage), so the planes keep a pitch of 2 p_w complex64 values from then on.
// ---------------------------------------------------------------------------------------------
constexpr int GR_MSP = 7;
constexpr int GR_W = 2 * GR_MSP;
constexpr float GR_FIX = 4294967296.f;         // 2^32
constexpr float GR_UNFIX = 1.f / 4294967296.f;

__global__ void __launch_bounds__(256) k_grid_spread(GridPlanDev gp, int p_h, int p_w, SpeciesSet spset, int job0,
                                                     unsigned long long* __restrict__ grid,
                                                     unsigned* __restrict__ row_used) {
  const int4 jb = gp.jobs[job0 + blockIdx.y];  // kind, species, first atom, end atom
  const double* pos = spset.k[jb.x & 3].pos;
  const long plane = (long)p_h * p_w;
  unsigned long long* base = grid + (long)blockIdx.y * 8 * plane;  // 4 planes of (re, im) pairs
  const int total = (jb.w - jb.z) * GR_W;
  // h^2 / (4 tau) for the fine-grid spacing h = 2 pi / (2P): pi (R - 1/2) / (R M_sp)
  const float kappa = 3.f * 3.14159265358979f / (4.f * GR_MSP);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int q = t / GR_W, jy = t - q * GR_W;
    const int a = jb.z + q;
    const double x = pos[2L * a], y = pos[2L * a + 1];
    const double fx = gp.dkx * x, fy = gp.dky * y;
    const double u = (fx - floor(fx)) * (2.0 * p_w), v = (fy - floor(fy)) * (2.0 * p_h);
    const double fu = floor(u), fv = floor(v);
    const float du = (float)(u - fu), dv = (float)(v - fv);
    const float2 w = phase_of(gp.sx * x + gp.sy * y);
    const int my = ((int)fv + jy - (GR_MSP - 1)) & (2 * p_h - 1);
    row_used[(long)blockIdx.y * 2 * p_h + my] = 1u;  // the row pass skips fine rows nobody touched
    const float ey = (float)(jy - (GR_MSP - 1)) - dv;
    unsigned long long* row = base + (long)(my & 1) * 4 * plane + (long)(my >> 1) * 2 * p_w;
#pragma unroll 2
    for (int jx = 0; jx < GR_W; ++jx) {
      const int mx = ((int)fu + jx - (GR_MSP - 1)) & (2 * p_w - 1);
      const float ex = (float)(jx - (GR_MSP - 1)) - du;
      const float gw = __expf(-kappa * fmaf(ex, ex, ey * ey)) * GR_FIX;
      unsigned long long* dst = row + (long)(mx & 1) * 2 * plane + 2 * (mx >> 1);
      atomicAdd(dst, (unsigned long long)__float2ll_rn(w.x * gw));
      atomicAdd(dst + 1, (unsigned long long)__float2ll_rn(w.y * gw));
    }
  }
}

// Row pass: forward FFTs of the fine-grid rows of parity ex = 0 and 1 of one (job, ey, qy)
// (p_w = N points of fixed-point pairs, 16 bytes each) in one CTA, then
//   out[c] = ax[c][0] FFT(row_0)[k] + ax[c][1] FFT(row_1)[k],  k = (c + N/2) mod N,
// written as complex64 over the first half of the ex = 0 row.  Transform g of a CTA takes parity
// g & 1; the partner's spectrum comes through shared memory.  A fine row that no atom touched
// (row_used == 0; most rows of a crystal, whose atoms sit on lattice rows) is zero and so is its
// transform: the pair skips all work (from N = 256, where a pair never shares a warp with
// another pair's warp-level barriers).  A pair that ran zeroes the second half of both its rows;
// the first halves of all rows (where the column pass writes) and the flags are cleared in bulk
// before each batch.  (A 128-register bound: the forward transform of a 16-byte-per-point row
// does not fit 96.)
template <int N>
struct GridRowCfg {
  static constexpr int P = RowCfg<N>::P, T = RowCfg<N>::T;
  static constexpr int G = RowCfg<N>::G < 2 ? 2 : RowCfg<N>::G;
  static constexpr int MINB = (512 / (G * T) > 0) ? 512 / (G * T) : 1;
};
template <int N>
__global__ void __launch_bounds__(GridRowCfg<N>::G * GridRowCfg<N>::T, GridRowCfg<N>::MINB)
    k_grid_rows(void* __restrict__ grid, const unsigned* __restrict__ row_used, const float4* __restrict__ ax, int p_h,
                const float2* __restrict__ tw) {
  constexpr int P = GridRowCfg<N>::P, T = GridRowCfg<N>::T, G = GridRowCfg<N>::G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int g = threadIdx.x / T, j = threadIdx.x - g * T, ex = g & 1;
  const long pair = (long)blockIdx.x * (G / 2) + (g >> 1);
  const long qy = pair % p_h, t = pair / p_h;                 // t = 2 job + ey
  const long row0 = ((t >> 1) * 4 + 2 * (t & 1)) * p_h + qy;  // plane (ey, 0), row qy
  // fine row 2 qy + ey of job t / 2
  const bool live = N < 256 || row_used[(t >> 1) * 2 * p_h + 2 * qy + (t & 1)] != 0u;
  longlong2* src = static_cast<longlong2*>(grid) + (row0 + ex * p_h) * N;
  float2 v[P];
  if (live) {
#pragma unroll
    for (int m = 0; m < P; ++m) {
      const longlong2 q = src[j + m * T];
      v[m] = make_float2(__ll2float_rn(q.x) * GR_UNFIX, __ll2float_rn(q.y) * GR_UNFIX);
    }
  }
  load_twiddles<N>(s_tw, tw);
  __syncthreads();  // every point of the CTA's rows is in registers before any is overwritten
  const RowLayout<N> L;
  if (live) {
    // clear what the next batch's bulk clear leaves out: the second half of both rows
#pragma unroll
    for (int m = P / 2; m < P; ++m) src[j + m * T] = make_longlong2(0, 0);
    fft_regs<N, false>(v, j, g, s_tw, s_x, RowLayout<N>(), group_sync<N>(g));
#pragma unroll
    for (int m = 0; m < P; ++m) s_x[L(g, j + m * T)] = v[m];
  }
  __syncthreads();
  if (!live) return;  // the output row is still the zero the grid was cleared to
  float2* dst = static_cast<float2*>(grid) + row0 * 2 * N;
#pragma unroll
  for (int m = 0; m < P; ++m) {
    if ((m < P / 2) != (ex == 0)) continue;  // parity 0 finishes k < N/2, parity 1 the rest
    const int k = j + m * T;
    const float2 other = s_x[L(g ^ 1, k)];
    const float2 x0 = ex ? other : v[m], x1 = ex ? v[m] : other;
    const int c = (k + N / 2) & (N - 1);
    const float4 a = ax[c];
    dst[c] = cadd(cmul(make_float2(a.x, a.y), x0), cmul(make_float2(a.z, a.w), x1));
  }
}

// Forward FFT of the columns of pitched planes (width columns, rows ``pitch`` apart).  Plane pl is
// (job pl / 2, parity ey = pl % 2); its row q is fine row 2 q + ey, which is zero when no atom
// touched it (row_used == 0: the row pass left the cleared zeros there), so it is not read.
template <int N>
__global__ void __launch_bounds__(GridColCfg<N>::G * GridColCfg<N>::T, GridColCfg<N>::MINB)
    k_grid_cols(float2* __restrict__ data, int width, long pitch, long plane_stride, const unsigned* __restrict__ row_used,
                const float2* __restrict__ tw) {
  constexpr int P = GridColCfg<N>::P, T = GridColCfg<N>::T, G = GridColCfg<N>::G;
  extern __shared__ float2 sh[];
  float2* s_tw = sh;
  float2* s_x = sh + Fft<N>::tw_size;
  const int j = threadIdx.x / G, g = threadIdx.x - j * G;
  const int nblk = width / G;
  const long pl = blockIdx.x / nblk;
  const int cb = blockIdx.x - (int)pl * nblk;
  float2* p = data + pl * plane_stride + cb * G + g;
  const unsigned* used = row_used + (pl >> 1) * 2 * N + (pl & 1);  // row q: used[2 q]
  load_twiddles<N>(s_tw, tw);
  float2 v[P];
#pragma unroll
  for (int m = 0; m < P; ++m) {
    const int q = j + m * T;
    v[m] = __ldg(used + 2 * q) ? p[(long)q * pitch] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_regs<N, false>(v, j, g, s_tw, s_x, ColLayout<N, G>(), SyncBlock());
#pragma unroll
  for (int m = 0; m < P; ++m) p[(long)(j + m * T) * pitch] = v[m];
}

// V(r, c) of slices s_lo.. from the transformed planes of jobs [j_lo, j_hi): per job the y
// half-bin combination and deconvolution give S, then f_species(s^2) S is summed; PARAMETER *
// APERTURE as in k_tx_species.  A slice whose first jobs ran in an earlier batch adds to what
// that batch wrote.
__global__ void __launch_bounds__(256) k_grid_combine(TxGrid g, SpeciesSet spset, GridPlanDev gp,
                                                      const float2* __restrict__ grid, int s_lo, int j_lo, int j_hi,
                                                      float2* __restrict__ out) {
  const long plane = (long)g.p_h * g.p_w;
  const long pitch = 2L * g.p_w, pstride = (long)g.p_h * pitch;
  const int s = s_lo + blockIdx.y;
  const int jb0 = max(gp.job_beg[s], j_lo), jb1 = min(gp.job_beg[s + 1], j_hi);
  const bool add = gp.job_beg[s] < j_lo;
  float2* dst = out + (long)s * plane;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < plane; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / g.p_w), c = (int)(i - (long)r * g.p_w);
    const int qr = (r + g.p_h / 2) & (g.p_h - 1);
    const float2 y0 = gp.ay[2 * r], y1 = gp.ay[2 * r + 1];
    const float s2 = g.s2[i];
    float2 acc = make_float2(0.f, 0.f);
    for (int jj = jb0; jj < jb1; ++jj) {
      const int4 jb = gp.jobs[jj];
      const float2* F = grid + (long)(jj - j_lo) * 4 * pstride + (long)qr * pitch + c;
      const float2 S = cadd(cmul(y0, F[0]), cmul(y1, F[2 * pstride]));
      float fr, fi;
      species_form(jb.x & 3, g, spset.k[jb.x & 3], jb.y, s2, i, fr, fi);
      acc.x = fmaf(fr, S.x, fmaf(-fi, S.y, acc.x));
      acc.y = fmaf(fr, S.y, fmaf(fi, S.x, acc.y));
    }
    const float ap = (g.aper_true != nullptr) ? g.aper_true[i] : 1.f;
    float2 v = cscale(acc, g.parameter * ap);
    if (add) v = cadd(dst[i], v);
    dst[i] = v;
  }
}

template <int N>
Status grid_rows(void* grid, const unsigned* row_used, long pairs, const float2* ax, int p_h, const float2* tw,
                 cudaStream_t st) {
  constexpr int T = GridRowCfg<N>::T, G = GridRowCfg<N>::G;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_grid_rows<N>, smem));
  if (pairs % (G / 2)) return Status::Err(TOTEM_ERR_UNSUPPORTED, "row count not a multiple of the row tile");
  k_grid_rows<N><<<(unsigned)(pairs / (G / 2)), G * T, smem, st>>>(grid, row_used, reinterpret_cast<const float4*>(ax),
                                                                   p_h, tw);
  return cuda_status(cudaGetLastError(), "k_grid_rows");
}

template <int N>
Status grid_cols(float2* data, long planes, int width, long pitch, long plane_stride, const unsigned* row_used,
                 const float2* tw, cudaStream_t st) {
  constexpr int T = GridColCfg<N>::T, G = GridColCfg<N>::G;
  const size_t smem = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, G>::size(G));
  TOTEM_TRY(ensure_smem((const void*)k_grid_cols<N>, smem));
  if (width % G) return Status::Err(TOTEM_ERR_UNSUPPORTED, "grid width not a multiple of the column tile");
  k_grid_cols<N><<<(unsigned)(planes * (width / G)), G * T, smem, st>>>(data, width, pitch, plane_stride, row_used,
                                                                          tw);
  return cuda_status(cudaGetLastError(), "k_grid_cols");
}

__global__ void k_sign_exp(float2* __restrict__ data, long total, int p_h, int p_w, float sig) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long plane = (long)p_h * p_w;
    const long k = i % plane;
    const int r = (int)(k / p_w), c = (int)(k % p_w);
    // ifftshift of the input == multiplication of the output by (-1)^(r+c) (even sizes only;
    // the uploader rejects odd grids, as the reference's quadrant-swap ifftShift assumes).
    const float sgn = ((r + c) & 1) ? -1.f : 1.f;
    float2 v = data[i];
    const float re = sgn * v.x * sig, im = sgn * v.y * sig;
    const float amp = expf(-im);
    float sn, cs;
    sincosf(re, &sn, &cs);
    data[i] = make_float2(amp * cs, amp * sn);
  }
}

}  // namespace

bool gridding_size_ok(int n) { return n >= 64 && n <= 4096 && (n & (n - 1)) == 0; }
bool fused_fft_size_ok(int n) { return gridding_size_ok(n) || radix_window_ops(n) != nullptr; }

namespace {
template <int N>
constexpr int2 tx_tiles() { return make_int2(RowCfg<N>::G, GridColCfg<N>::G); }
// (rows per row tile, columns per column tile) of the transmission FFT at edge n; (0, 0) if none
int2 tx_tiles_of(int n) {
  switch (n) {
#define TOTEM_TX_TILES(NN) \
  case NN: return tx_tiles<NN>();
    TOTEM_TX_TILES(64) TOTEM_TX_TILES(128) TOTEM_TX_TILES(256) TOTEM_TX_TILES(512) TOTEM_TX_TILES(1024)
    TOTEM_TX_TILES(2048) TOTEM_TX_TILES(4096)
#undef TOTEM_TX_TILES
  }
  if (const WindowOps* o = radix_window_ops(n)) return make_int2(o->row_tile_rows, o->col_tile_cols);
  return make_int2(0, 0);
}
}  // namespace

bool tx_fft_shape_ok(int p_h, int p_w, int slices) {
  const int2 rw = tx_tiles_of(p_w), ch = tx_tiles_of(p_h);
  return rw.x > 0 && ch.y > 0 && ((long)slices * p_h) % rw.x == 0 && p_w % ch.y == 0;
}

Status launch_tx_structure(const TxGrid& g, const AtomRowsDev& neutral, const AtomRowsDev& ion,
                           const AtomRowsDev& corr_n, const AtomRowsDev& corr_i, float2* out, cudaStream_t st,
                           bool accumulate) {
  dim3 grid((g.p_w + TX_TC - 1) / TX_TC, (g.p_h + TX_TR - 1) / TX_TR, g.slices);
  if (g.slices == 0) return Status::Ok();
  if (g.separable) k_tx_structure<true><<<grid, 256, 0, st>>>(g, neutral, ion, corr_n, corr_i, out, accumulate);
  else k_tx_structure<false><<<grid, 256, 0, st>>>(g, neutral, ion, corr_n, corr_i, out, accumulate);
  return cuda_status(cudaGetLastError(), "k_tx_structure");
}

Status launch_tx_species(const TxGrid& g, const SpeciesSet& sp, float2* out, cudaStream_t st) {
  if (g.slices == 0) return Status::Ok();
  if (!g.separable) return Status::Err(TOTEM_ERR_UNSUPPORTED, "species builder needs separable reciprocal grids");
  dim3 grid((g.p_w + SP_T - 1) / SP_T, (g.p_h + SP_T - 1) / SP_T, g.slices);
  k_tx_species<<<grid, 256, 0, st>>>(g, sp, out);
  return cuda_status(cudaGetLastError(), "k_tx_species");
}

std::vector<float2> grid_deconvolution(int n) {
  // tau = pi M_sp / (n^2 R (R - 1/2)); the fine grid's FFT carries 1 / (R n) per axis
  const double pi = 3.14159265358979323846;
  const double tau = pi * GR_MSP / ((double)n * n * 2.0 * 1.5);
  const double pre = std::sqrt(pi / tau) / (2.0 * n);
  std::vector<float2> t(2 * (size_t)n);
  for (int c = 0; c < n; ++c) {
    const double k = c - n / 2;
    const double d = pre * std::exp(k * k * tau);
    t[2 * c] = make_float2((float)d, 0.f);
    t[2 * c + 1] = make_float2((float)(d * std::cos(pi * k / n)), (float)(-d * std::sin(pi * k / n)));
  }
  return t;
}

std::vector<GridBatch> grid_batches(const std::vector<int>& job_beg, int jobs_per_batch) {
  std::vector<GridBatch> out;
  const int slices = (int)job_beg.size() - 1;
  if (slices <= 0 || jobs_per_batch < 1) return out;
  const int total = job_beg[slices];
  int s_lo = 0, j_lo = 0;
  while (s_lo < slices) {
    const int j_hi = std::min(j_lo + jobs_per_batch, total);
    int s_hi = s_lo;
    if (j_hi == total) s_hi = slices;
    else
      while (s_hi < slices && job_beg[s_hi] < j_hi) ++s_hi;
    out.push_back(GridBatch{s_lo, s_hi, j_lo, j_hi});
    const bool partial = job_beg[s_hi] > j_hi;  // slice s_hi - 1 continues in the next batch
    s_lo = partial ? s_hi - 1 : s_hi;
    j_lo = j_hi;
  }
  return out;
}

Status launch_tx_gridding(const TxGrid& g, const SpeciesSet& sp, const GridPlanDev& gp,
                          const std::vector<int>& job_beg, const std::vector<int4>& jobs, const float2* tw_w,
                          const float2* tw_h, void* scratch, size_t scratch_bytes, bool scratch_zero, float2* out,
                          cudaStream_t st, int* launches) {
  if (g.slices == 0) return Status::Ok();
  if (!gridding_size_ok(g.p_h) || !gridding_size_ok(g.p_w))
    return Status::Err(TOTEM_ERR_UNSUPPORTED, "gridding builder needs power-of-two grids 64..4096");
  if ((int)job_beg.size() != g.slices + 1) return Status::Err(TOTEM_ERR_STATE, "gridding job table size");
  const long plane = (long)g.p_h * g.p_w;
  const size_t job_bytes = grid_job_bytes(g.p_h, g.p_w);
  const int per_batch = (int)std::min<size_t>(scratch_bytes / job_bytes, 65535);  // grid.y of the spread
  if (per_batch < 1) return Status::Err(TOTEM_ERR_STATE, "gridding scratch below one job");
  const long pitch = 2L * g.p_w, pstride = (long)g.p_h * pitch;
  const size_t plane_bytes = (size_t)plane * 64;  // four planes of 16-byte points per job
  unsigned* used = reinterpret_cast<unsigned*>(static_cast<char*>(scratch) + plane_bytes * per_batch);
  // Between batches the kernels leave the second half of every fine row zero; new scratch is
  // cleared whole once, and the first halves (dense after the column pass) and the row flags are
  // cleared in bulk before each batch (a strided memset; clearing the first halves in the combine
  // after reading was measured 7x slower than the combine itself).
  if (!scratch_zero) TOTEM_CUDA(cudaMemsetAsync(scratch, 0, job_bytes * per_batch, st));
  for (const GridBatch& b : grid_batches(job_beg, per_batch)) {
    const int nj = b.j_hi - b.j_lo;
    if (nj > 0) {
      TOTEM_CUDA(cudaMemset2DAsync(scratch, 16 * (size_t)g.p_w, 0, 8 * (size_t)g.p_w, 4 * (size_t)g.p_h * nj, st));
      TOTEM_CUDA(cudaMemsetAsync(used, 0, sizeof(unsigned) * 2 * g.p_h * nj, st));
      int most = 0;
      for (int j = b.j_lo; j < b.j_hi; ++j) most = std::max(most, jobs[j].w - jobs[j].z);
      const unsigned bx = (unsigned)std::min<long>(((long)most * GR_W + 255) / 256 + 1, 4096);
      k_grid_spread<<<dim3(bx, nj), 256, 0, st>>>(gp, g.p_h, g.p_w, sp, b.j_lo,
                                                  static_cast<unsigned long long*>(scratch), used);
      TOTEM_TRY(cuda_status(cudaGetLastError(), "k_grid_spread"));
      const long pairs = (long)nj * 2 * g.p_h, planes = (long)nj * 2;  // (job, ey) after the row pass
      float2* f = static_cast<float2*>(scratch);
      switch (g.p_w) {
        case 64: TOTEM_TRY(grid_rows<64>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 128: TOTEM_TRY(grid_rows<128>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 256: TOTEM_TRY(grid_rows<256>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 512: TOTEM_TRY(grid_rows<512>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 1024: TOTEM_TRY(grid_rows<1024>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 2048: TOTEM_TRY(grid_rows<2048>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
        case 4096: TOTEM_TRY(grid_rows<4096>(scratch, used, pairs, gp.ax, g.p_h, tw_w, st)); break;
      }
      switch (g.p_h) {
        case 64: TOTEM_TRY(grid_cols<64>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 128: TOTEM_TRY(grid_cols<128>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 256: TOTEM_TRY(grid_cols<256>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 512: TOTEM_TRY(grid_cols<512>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 1024: TOTEM_TRY(grid_cols<1024>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 2048: TOTEM_TRY(grid_cols<2048>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
        case 4096: TOTEM_TRY(grid_cols<4096>(f, planes, g.p_w, pitch, 2 * pstride, used, tw_h, st)); break;
      }
      *launches += 3;
    }
    const unsigned cx = (unsigned)std::min<long>((plane + 255) / 256, 2048);
    for (int s0 = b.s_lo; s0 < b.s_hi; s0 += 65535) {
      const int ns = std::min(b.s_hi - s0, 65535);
      k_grid_combine<<<dim3(cx, ns), 256, 0, st>>>(g, sp, gp, static_cast<const float2*>(scratch), s0, b.j_lo,
                                                   b.j_hi, out);
      TOTEM_TRY(cuda_status(cudaGetLastError(), "k_grid_combine"));
      ++*launches;
    }
  }
  return Status::Ok();
}

Status launch_tx_fft_exp(float2* data, int slices, int p_h, int p_w, float sig, const float2* tw_w,
                         const float2* tw_h, cudaStream_t st) {
  if (!tx_fft_shape_ok(p_h, p_w, slices))
    return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused transmission FFT: unsupported grid shape");
  const long nrows = (long)slices * p_h;
  switch (p_w) {
#define TOTEM_TX_ROWS_CASE(NN) \
  case NN: TOTEM_TRY(rows_inv<NN>(data, nrows, tw_w, st)); break;
    TOTEM_TX_ROWS_CASE(64) TOTEM_TX_ROWS_CASE(128) TOTEM_TX_ROWS_CASE(256) TOTEM_TX_ROWS_CASE(512)
    TOTEM_TX_ROWS_CASE(1024) TOTEM_TX_ROWS_CASE(2048) TOTEM_TX_ROWS_CASE(4096)
#undef TOTEM_TX_ROWS_CASE
    default: TOTEM_TRY(radix_window_ops(p_w)->tx_rows_inv(data, nrows, tw_w, st));
  }
  switch (p_h) {
#define TOTEM_TX_COLS_CASE(NN) \
  case NN: return cols_exp<NN>(data, slices, p_w, tw_h, sig, st);
    TOTEM_TX_COLS_CASE(64) TOTEM_TX_COLS_CASE(128) TOTEM_TX_COLS_CASE(256) TOTEM_TX_COLS_CASE(512)
    TOTEM_TX_COLS_CASE(1024) TOTEM_TX_COLS_CASE(2048) TOTEM_TX_COLS_CASE(4096)
#undef TOTEM_TX_COLS_CASE
  }
  return radix_window_ops(p_h)->tx_cols_exp(data, slices, p_w, tw_h, sig, st);
}

Status launch_sign_exp(float2* data, long total, int p_h, int p_w, float sig, cudaStream_t st) {
  if (total == 0) return Status::Ok();
  int blocks = (int)std::min<long>((total + 255) / 256, 148L * 16);
  k_sign_exp<<<blocks, 256, 0, st>>>(data, total, p_h, p_w, sig);
  return cuda_status(cudaGetLastError(), "k_sign_exp");
}

}  // namespace totem
