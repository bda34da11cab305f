// Row pass of the fused slice loop (single request): row IFFT -> * T[window] / N^2 -> row FFT
// (the first pass: probe * T -> row FFT) of the power-of-two windows, every register-cap variant
// and the zero-band skip; the mixed-radix windows come from their WindowOps table.
#include "passes.cuh"

namespace totem {

Status launch_row_pass(const SliceLoopArgs& a, const void* tslice, bool first, cudaStream_t st) {
  switch (a.n) {
#define TOTEM_ROW(NN) \
  case NN: return first ? row_pass<NN, true>(a, tslice, st) : row_pass<NN, false>(a, tslice, st);
    TOTEM_ROW(64) TOTEM_ROW(128) TOTEM_ROW(256) TOTEM_ROW(512) TOTEM_ROW(1024) TOTEM_ROW(2048)
#undef TOTEM_ROW
  }
  if (const WindowOps* o = radix_window_ops(a.n)) return o->row_pass(a, tslice, first, st);
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused slice loop: unsupported window edge");
}

}  // namespace totem
