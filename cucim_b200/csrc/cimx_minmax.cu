// cimx_minmax.cu — minimum_filter1d / maximum_filter1d
// (_vendored/_ndimage_filters.py:1362-1497, kernel body from
// _get_min_or_max_kernel without weights): per output, the value starts at
// the input element itself as a double, then every window element in tap
// order (mapped by the boundary mode; the fill value cval itself, as a
// double, outside the array in constant mode) is folded in with fmin / fmax
// in double (nan-ignoring); the result is stored with cast<Y>().
//
// One thread per output of the view (outer, L, inner); the window is read
// through L1 and L2 (neighbouring threads of a row share it).
#include <algorithm>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

struct MinMaxArgs {
  const void* in;
  void* out;
  int tin, tout;
  long long outer, L, inner;
  int size, anchor, mode, is_max;
  double cval;
};

__global__ void __launch_bounds__(256) k_minmax1d(const MinMaxArgs a) {
  const long long n = a.outer * a.L * a.inner;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % a.inner;
    const long long l = (idx / a.inner) % a.L;
    const long long o = idx / (a.inner * a.L);
    const long long base = o * a.L * a.inner + i;
    double value = load_as<double>(a.in, idx, a.tin);
    for (int k = 0; k < a.size; ++k) {
      const long long c = l - a.anchor + k;
      const long long m = (c >= 0 && c < a.L) ? c : map_coord_near(c, a.L, a.mode);
      const double v = m < 0 ? a.cval : load_as<double>(a.in, base + m * a.inner, a.tin);
      value = a.is_max ? fmax(v, value) : fmin(v, value);
    }
    store_cast<double>(a.out, idx, value, a.tout);
  }
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" int cimx_min_max_1d(const CimxArray* in, const CimxArray* out, int size, int axis,
                               int origin, int mode, double cval, int is_max, void* stream) {
  if (!in || !out) return fail(CIMX_E_INVALID, "min/max filter: NULL array");
  if (size < 1) return fail(CIMX_E_INVALID, "incorrect filter size");
  if (in->ndim < 1 || in->ndim != out->ndim) return fail(CIMX_E_INVALID, "min/max filter: ndim");
  if (axis < 0 || axis >= in->ndim) return fail(CIMX_E_INVALID, "min/max filter: axis");
  if (mode < CIMX_MODE_REFLECT || mode > CIMX_MODE_CONSTANT)
    return fail(CIMX_E_INVALID, "boundary mode not supported");
  if (dtype_size(in->dtype) == 0 || dtype_size(out->dtype) == 0)
    return fail(CIMX_E_DTYPE, "min/max filter: unsupported dtype");
  long long outer = 1, inner = 1, n = 1;
  for (int d = 0; d < in->ndim; ++d) {
    if (in->shape[d] != out->shape[d]) return fail(CIMX_E_INVALID, "output shape not correct");
    if (d < axis) outer *= in->shape[d];
    if (d > axis) inner *= in->shape[d];
    n *= in->shape[d];
  }
  // C-contiguous layouts only (the Python layer makes them so)
  long long expect = dtype_size(in->dtype), expect_o = dtype_size(out->dtype);
  for (int d = in->ndim - 1; d >= 0; --d) {
    if (in->shape[d] > 1 && (in->strides[d] != expect || out->strides[d] != expect_o))
      return fail(CIMX_E_LAYOUT, "min/max filter: arrays must be C-contiguous");
    expect *= in->shape[d];
    expect_o *= out->shape[d];
  }
  if (n == 0) return CIMX_OK;
  const int anchor = size / 2 + origin;
  if (anchor < 0 || anchor >= size) return fail(CIMX_E_INVALID, "invalid origin");
  MinMaxArgs a{in->data, out->data, in->dtype, out->dtype, outer, in->shape[axis], inner,
               size, anchor, mode, is_max ? 1 : 0, cval};
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
  k_minmax1d<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  return cuda_fail(cudaGetLastError(), "min/max filter launch");
}
