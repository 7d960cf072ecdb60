// cimx_fast_u8.cu — instantiations of the fast kernels (cimx_fast.cuh) for
// uint8_t input. Split by input dtype so the kernels compile in parallel.
#include "cimx_fast.cuh"
#include "cimx_vol.cuh"

namespace cimx {

int launch_stream_u8(const PassDesc& d, const float* w, int K, int anchor,
                      bool interior_zero, const void* in, int tout, void* out,
                      cudaStream_t st) {
  using namespace fast;
  if (tout == DT_F32)
    return launch_stream_td<uint8_t, float>(d, w, K, anchor, interior_zero, in, out, st);
  if (tout == DT_U8)
    return launch_stream_td<uint8_t, uint8_t>(d, w, K, anchor, interior_zero, in, out, st);
  if (tout == DT_U16)
    return launch_stream_td<uint8_t, uint16_t>(d, w, K, anchor, interior_zero, in, out, st);
  return CIMX_FUSED_DECLINED;
}

int launch_slab_u8(SlabArgs& a, int tout, cudaStream_t st) {
  using namespace fast;
  if (tout == DT_F32) return launch_slab_td<uint8_t, float>(a, st);
  if (tout == DT_U8) return launch_slab_td<uint8_t, uint8_t>(a, st);
  if (tout == DT_U16) return launch_slab_td<uint8_t, uint16_t>(a, st);
  return CIMX_FUSED_DECLINED;
}

int launch_vol_u8(const VolArgs& v, int tout, cudaStream_t st) {
  if (tout == DT_F32) return vol::launch_vol_td<uint8_t, float>(v, st);
  if (tout == DT_U8) return vol::launch_vol_td<uint8_t, uint8_t>(v, st);
  if (tout == DT_U16) return vol::launch_vol_td<uint8_t, uint16_t>(v, st);
  return CIMX_FUSED_DECLINED;
}

}  // namespace cimx
