// cimx_edges.cu — the `mask=` argument of the skimage edge filters
// (python/cucim/src/cucim/skimage/filters/edges.py:75-85,
// _mask_filter_result): the mask is eroded with the full-connectivity
// footprint (every element of the 3 x ... x 3 neighbourhood,
// generate_binary_structure(ndim, ndim)) with border_value 0, and the
// filter result is multiplied by the eroded mask in place. One thread per
// output element reads the 3^ndim neighbourhood of the mask directly (the
// erosion is never stored).
#include <algorithm>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

struct MaskShape {
  int ndim;
  int64_t shape[CIMX_MAX_NDIM];
};

inline unsigned grid_for(int64_t n, int threads = 256) {
  const int64_t b = (n + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

// binary_erosion's truth value of one mask element (nonzero; NaN is nonzero)
__device__ __forceinline__ bool mask_true(const void* m, int t, int64_t i) {
  switch (t) {
    case 'H': case 'h': return static_cast<const uint16_t*>(m)[i] != 0;
    case 'e': return (static_cast<const uint16_t*>(m)[i] & 0x7fffu) != 0;
    case 'I': case 'i': return static_cast<const uint32_t*>(m)[i] != 0;
    case 'f': return static_cast<const float*>(m)[i] != 0.0f;
    case 'd': return static_cast<const double*>(m)[i] != 0.0;
    case 'L': case 'Q': case 'l': case 'q': return static_cast<const uint64_t*>(m)[i] != 0;
    default: return static_cast<const uint8_t*>(m)[i] != 0;  // '?', 'B', 'b'
  }
}

template <class F>
__global__ void k_mask_erode_mul(F* __restrict__ res, const void* __restrict__ mask, int tm,
                                 MaskShape s, int64_t n) {
  int nb = 1;
  for (int d = 0; d < s.ndim; ++d) nb *= 3;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t c[CIMX_MAX_NDIM];
    int64_t r = i;
    for (int d = s.ndim - 1; d >= 0; --d) {
      c[d] = r % s.shape[d];
      r /= s.shape[d];
    }
    bool keep = true;
    for (int o = 0; o < nb && keep; ++o) {
      int code = o;
      int64_t j = 0;
      for (int d = 0; d < s.ndim; ++d) {
        const int64_t x = c[d] + (code % 3) - 1;
        code /= 3;
        if (x < 0 || x >= s.shape[d]) {  // border_value=0
          keep = false;
          break;
        }
        j = j * s.shape[d] + x;
      }
      if (keep) keep = mask_true(mask, tm, j);
    }
    res[i] = res[i] * (keep ? F(1) : F(0));  // result *= mask
  }
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" int cimx_mask_erode_multiply(const CimxArray* result, const CimxArray* mask,
                                        void* stream) {
  if (!result || !mask) return fail(CIMX_E_INVALID, "NULL argument");
  if (result->dtype != DT_F32 && result->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "the filter result must be float32 or float64");
  if (mask->dtype != '?' && dtype_size(mask->dtype) == 0)
    return fail(CIMX_E_DTYPE, "unsupported mask dtype");
  if (mask->ndim != result->ndim || result->ndim < 1 || result->ndim > CIMX_MAX_NDIM)
    return fail(CIMX_E_INVALID, "mask shape must equal the image shape");
  MaskShape s{};
  s.ndim = result->ndim;
  int64_t n = 1;
  for (int d = 0; d < s.ndim; ++d) {
    if (mask->shape[d] != result->shape[d])
      return fail(CIMX_E_INVALID, "mask shape must equal the image shape");
    s.shape[d] = result->shape[d];
    n *= s.shape[d];
  }
  // both C-contiguous
  const int msize = mask->dtype == '?' ? 1 : dtype_size(mask->dtype);
  int64_t er = dtype_size(result->dtype), em = msize;
  for (int d = s.ndim - 1; d >= 0; --d) {
    if (s.shape[d] != 1 && (result->strides[d] != er || mask->strides[d] != em))
      return fail(CIMX_E_LAYOUT, "result and mask must be C-contiguous");
    er *= s.shape[d];
    em *= s.shape[d];
  }
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (result->dtype == DT_F32)
    k_mask_erode_mul<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(result->data),
                                                         mask->data, mask->dtype, s, n);
  else
    k_mask_erode_mul<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(result->data),
                                                          mask->data, mask->dtype, s, n);
  return cuda_fail(cudaGetLastError(), "mask launch");
}
