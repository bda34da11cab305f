// Fused passes of the mixed-radix windows of TOTEM_MR_WINDOWS_D (the four quarters of the
// sizes compile in parallel).
#include "passes.cuh"

namespace totem {

const WindowOps* radix_window_ops_d(int n) {
  switch (n) {
#define TOTEM_MR_CASE(NN) \
  case NN: return window_ops<NN>();
    TOTEM_MR_WINDOWS_D(TOTEM_MR_CASE)
#undef TOTEM_MR_CASE
  }
  return nullptr;
}

}  // namespace totem
