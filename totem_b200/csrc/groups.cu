// Continuous batching: row and column passes over groups of items of several requests, each
// group at its own slice; per window size, or (mixed) over 256^2 .. 1024^2 windows at once.
#include <map>
#include <mutex>

#include "passes.cuh"

namespace totem {

namespace {

// ---------------------------------------------------------------------------------------------
// Windows of different sizes in one launch.  A persistent CTA of kMixedThreads threads takes
// work units from a queue (an atomic counter) until the launch's units run out; a unit is
// kMixedThreads / T rows (row pass) or one column tile (column pass, the tile width of the
// single-size kernel, so the detector partial sums are the same) of one item of one group,
// groups of 256^2, 512^2 and 1024^2 windows mixed.  The per-tile code is the single-size
// kernels', so every result is bit-identical to the per-size launches.  Units are numbered group
// by group: work_begin[g] is the first unit of group g, work_begin[ngroups] the total.
// ---------------------------------------------------------------------------------------------
template <int N>
constexpr int mixed_row_units() { return N / (kMixedThreads / Fft<N>::T); }

__device__ __forceinline__ int take_unit(int* queue) {
  __shared__ int s_unit;
  __syncthreads();  // the previous unit is done with shared memory
  if (threadIdx.x == 0) s_unit = atomicAdd(queue, 1);
  __syncthreads();
  return s_unit;
}

__global__ void __launch_bounds__(kMixedThreads, 2)
    k_row_mixed(const GroupDesc* __restrict__ groups, const int* __restrict__ work_begin, int ngroups, int tick,
                MixedTwiddles tw, int* queue) {
  const int total = __ldg(work_begin + ngroups);
  for (int u = take_unit(queue); u < total; u = take_unit(queue)) {
    const int gidx = find_group(work_begin, ngroups, u);
    const GroupDesc& d = groups[gidx];
    const int lu = u - __ldg(work_begin + gidx);
    switch (d.n) {
#define TOTEM_ROW_MIXED(NN, TW)                                                                   \
  case NN: {                                                                                      \
    constexpr int rows = kMixedThreads / Fft<NN>::T, per_item = NN / rows;                        \
    row_group_tile<NN>(d, lu / per_item, (lu % per_item) * rows, tick, tw.TW);                    \
    break;                                                                                        \
  }
      TOTEM_ROW_MIXED(256, n256) TOTEM_ROW_MIXED(512, n512) TOTEM_ROW_MIXED(1024, n1024)
#undef TOTEM_ROW_MIXED
    }
  }
}

__global__ void __launch_bounds__(kMixedThreads, 2)
    k_col_mixed(const GroupDesc* __restrict__ groups, const int* __restrict__ work_begin, int ngroups, int tick,
                MixedTwiddles tw, int* queue) {
  const int total = __ldg(work_begin + ngroups);
  for (int u = take_unit(queue); u < total; u = take_unit(queue)) {
    const int gidx = find_group(work_begin, ngroups, u);
    const GroupDesc& d = groups[gidx];
    const int lu = u - __ldg(work_begin + gidx);
    switch (d.n) {
#define TOTEM_COL_MIXED(NN, TW)                                                                   \
  case NN: {                                                                                      \
    constexpr int G = ColCfg<NN>::G;                                                              \
    static_assert(G * ColCfg<NN>::T == kMixedThreads, "mixed column tiles use the single-size tile width"); \
    const int active = NN / G - d.skip.nskip;                                                     \
    const int t = lu % active;                                                                    \
    col_group_tile<NN, G>(d, lu / active, t < d.skip.z0 ? t : t + d.skip.nskip, tick, tw.TW);     \
    break;                                                                                        \
  }
      TOTEM_COL_MIXED(256, n256) TOTEM_COL_MIXED(512, n512) TOTEM_COL_MIXED(1024, n1024)
#undef TOTEM_COL_MIXED
    }
  }
}

}  // namespace

Status launch_row_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, cudaStream_t st) {
  if (items <= 0 || ngroups <= 0) return Status::Ok();
  switch (n) {
    case 64: return row_groups<64>(groups, item_begin, ngroups, items, tick, tw, st);
    case 128: return row_groups<128>(groups, item_begin, ngroups, items, tick, tw, st);
    case 256: return row_groups<256>(groups, item_begin, ngroups, items, tick, tw, st);
    case 512: return row_groups<512>(groups, item_begin, ngroups, items, tick, tw, st);
    case 1024: return row_groups<1024>(groups, item_begin, ngroups, items, tick, tw, st);
    case 2048: return row_groups<2048>(groups, item_begin, ngroups, items, tick, tw, st);
  }
  if (const WindowOps* o = radix_window_ops(n)) return o->row_groups(groups, item_begin, ngroups, items, tick, tw, st);
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "continuous batching: unsupported window edge");
}

Status launch_col_groups(int n, const GroupDesc* groups, const int* item_begin, int ngroups, long items, int tick,
                         const float2* tw, TileSkip skip, cudaStream_t st) {
  if (items <= 0 || ngroups <= 0) return Status::Ok();
  switch (n) {
    case 64: return col_groups<64>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 128: return col_groups<128>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 256: return col_groups<256>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 512: return col_groups<512>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 1024: return col_groups<1024>(groups, item_begin, ngroups, items, tick, tw, skip, st);
    case 2048: return col_groups<2048>(groups, item_begin, ngroups, items, tick, tw, skip, st);
  }
  if (const WindowOps* o = radix_window_ops(n))
    return o->col_groups(groups, item_begin, ngroups, items, tick, tw, skip, st);
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "continuous batching: unsupported window edge");
}

template <int N>
size_t mixed_smem() {
  constexpr int rows = kMixedThreads / Fft<N>::T;
  const size_t row = sizeof(float2) * (Fft<N>::tw_size + RowLayout<N>::size(rows));
  const size_t col = sizeof(float2) * (Fft<N>::tw_size + ColLayout<N, ColCfg<N>::G>::size(ColCfg<N>::G));
  return row > col ? row : col;
}

int mixed_units(int n, bool row, TileSkip skip) {
  switch (n) {
    case 256: return row ? mixed_row_units<256>() : 256 / ColCfg<256>::G - skip.nskip;
    case 512: return row ? mixed_row_units<512>() : 512 / ColCfg<512>::G - skip.nskip;
    case 1024: return row ? mixed_row_units<1024>() : 1024 / ColCfg<1024>::G - skip.nskip;
  }
  return 0;
}

bool mixed_window_ok(int n) { return n == 256 || n == 512 || n == 1024; }

Status launch_mixed_groups(bool row, const GroupDesc* groups, const int* work_begin, int ngroups, long units,
                           int tick, const MixedTwiddles& tw, int* queue, cudaStream_t st) {
  if (units <= 0 || ngroups <= 0) return Status::Ok();
  size_t smem = mixed_smem<256>();
  smem = std::max(smem, mixed_smem<512>());
  smem = std::max(smem, mixed_smem<1024>());
  const void* fn = row ? (const void*)k_row_mixed : (const void*)k_col_mixed;
  TOTEM_TRY(ensure_smem(fn, smem));
  // resident CTAs of the whole GPU (both kernels: same shape and bounds), per device
  static std::mutex mu;
  static std::map<int, int> ctas_of;
  int dev = 0;
  TOTEM_CUDA(cudaGetDevice(&dev));
  int ctas = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = ctas_of.find(dev);
    if (it != ctas_of.end()) ctas = it->second;
  }
  if (ctas == 0) {
    int sms = 0, per_sm = 0;
    TOTEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    TOTEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_row_mixed, kMixedThreads, smem));
    ctas = std::max(1, sms * std::max(per_sm, 1));
    std::lock_guard<std::mutex> lk(mu);
    ctas_of[dev] = ctas;
  }
  const unsigned grid = (unsigned)std::min<long>(units, ctas);
  if (row) k_row_mixed<<<grid, kMixedThreads, smem, st>>>(groups, work_begin, ngroups, tick, tw, queue);
  else k_col_mixed<<<grid, kMixedThreads, smem, st>>>(groups, work_begin, ngroups, tick, tw, queue);
  return cuda_status(cudaGetLastError(), row ? "k_row_mixed" : "k_col_mixed");
}

}  // namespace totem
