// cimx_fast_f32.cu — instantiations of the fast kernels (cimx_fast.cuh) for
// float input. Split by input dtype so the kernels compile in parallel.
#include "cimx_fast.cuh"
#include "cimx_vol.cuh"

namespace cimx {

int launch_stream_f32(const PassDesc& d, const float* w, int K, int anchor,
                      bool interior_zero, const void* in, int tout, void* out,
                      cudaStream_t st) {
  using namespace fast;
  if (tout == DT_F32)
    return launch_stream_td<float, float>(d, w, K, anchor, interior_zero, in, out, st);
  return CIMX_FUSED_DECLINED;
}

int launch_slab_f32(SlabArgs& a, int tout, cudaStream_t st) {
  using namespace fast;
  if (tout == DT_F32) return launch_slab_td<float, float>(a, st);
  return CIMX_FUSED_DECLINED;
}

int launch_vol_f32(const VolArgs& v, int tout, cudaStream_t st) {
  if (tout == DT_F32) return vol::launch_vol_td<float, float>(v, st);
  return CIMX_FUSED_DECLINED;
}

}  // namespace cimx
