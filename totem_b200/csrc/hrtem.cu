// HRTEM imaging from the exit-wave spectrum (hrtem_kernels.cuh): power-of-two grids here, the
// mixed-radix grids through their WindowOps table.
#include "hrtem_kernels.cuh"

namespace totem {

namespace {

Status image_dispatch(int n, const float2* spec, const float2* tf, int planes, const double* w, float2* work,
                      float2* out_c, float* out_i, const float2* tw, cudaStream_t st) {
  switch (n) {
    case 64: return image_n<64>(spec, tf, planes, w, work, out_c, out_i, tw, st);
    case 128: return image_n<128>(spec, tf, planes, w, work, out_c, out_i, tw, st);
    case 256: return image_n<256>(spec, tf, planes, w, work, out_c, out_i, tw, st);
    case 512: return image_n<512>(spec, tf, planes, w, work, out_c, out_i, tw, st);
    case 1024: return image_n<1024>(spec, tf, planes, w, work, out_c, out_i, tw, st);
    case 2048: return image_n<2048>(spec, tf, planes, w, work, out_c, out_i, tw, st);
  }
  if (const WindowOps* o = radix_window_ops(n)) return o->image(spec, tf, planes, w, work, out_c, out_i, tw, st);
  return Status::Err(TOTEM_ERR_UNSUPPORTED, "fused HRTEM imaging: unsupported grid edge");
}

}  // namespace

Status launch_exit_wave(int n, const float2* spec, float2* work, float2* out, const float2* tw, cudaStream_t st) {
  return image_dispatch(n, spec, nullptr, 1, nullptr, work, out, nullptr, tw, st);
}

Status launch_tcc_image(int n, const float2* spec, const float2* tf, int planes, const double* w, float2* work,
                        float* out, const float2* tw, cudaStream_t st) {
  if (planes <= 0) return Status::Ok();
  return image_dispatch(n, spec, tf, planes, w, work, nullptr, out, tw, st);
}

}  // namespace totem
