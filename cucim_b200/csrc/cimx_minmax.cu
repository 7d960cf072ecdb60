// cimx_minmax.cu — minimum_filter1d / maximum_filter1d
// (_vendored/_ndimage_filters.py:1362-1497, kernel body from
// _get_min_or_max_kernel without weights): per output, the value starts at
// the input element itself as a double, then every window element in tap
// order (mapped by the boundary mode; the fill value cval itself, as a
// double, outside the array in constant mode) is folded in with fmin / fmax
// in double (nan-ignoring); the result is stored with cast<Y>().
//
// Tiled kernels stage a stretch of the line (k_minmax_rows, last axis) or
// of 32 columns (k_minmax_cols, strided axes) once in shared memory as
// doubles, with the boundary map applied while staging, and every output
// then folds its window from shared memory in the same order as above. The
// one-thread-per-output kernel (k_minmax1d) reads the window through L1 and
// L2 and takes windows too long for a shared-memory tile.
#include <algorithm>
#include <mutex>

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
  long long tiles_a, tiles_b;
};

constexpr int kRowT = 256, kRowP = 4, kRowSeg = kRowT * kRowP;  // 1024 outputs per CTA
constexpr int kColTI = 32, kColTY = 8, kColP = 8, kColTL = kColTY * kColP;  // 32 x 64 tile
constexpr int kMaxSmem = 227 * 1024;

__device__ __forceinline__ double fold(double v, double value, int is_max) {
  return is_max ? fmax(v, value) : fmin(v, value);
}

// Staged value of line coordinate c (boundary map outside [0, L)).
__device__ __forceinline__ double staged(const MinMaxArgs& a, long long line0, long long c,
                                         long long stride) {
  const long long m = (c >= 0 && c < a.L) ? c : map_coord_near(c, a.L, a.mode);
  return m < 0 ? a.cval : load_as<double>(a.in, line0 + m * stride, a.tin);
}

// Last axis (inner == 1): one CTA per 1024 outputs of a row; thread t folds
// outputs t, t + 256, t + 512, t + 768 of the segment (coalesced stores).
__global__ void __launch_bounds__(kRowT) k_minmax_rows(const MinMaxArgs a) {
  extern __shared__ double s_line[];
  const long long row = blockIdx.x / a.tiles_b;
  const long long x0 = (blockIdx.x % a.tiles_b) * kRowSeg;
  const long long base = row * a.L;
  // the staged stretch: only as far as the stored outputs (x < L) read
  const long long need = a.L - x0 + a.size - 1;
  const int n = need < kRowSeg + a.size - 1 ? static_cast<int>(need) : kRowSeg + a.size - 1;
  const long long c0 = x0 - a.anchor;
  for (int j = threadIdx.x; j < n; j += kRowT) s_line[j] = staged(a, base, c0 + j, 1);
  __syncthreads();
#pragma unroll
  for (int p = 0; p < kRowP; ++p) {
    const int lx = threadIdx.x + p * kRowT;
    if (x0 + lx >= a.L) break;
    const double* w = s_line + lx;
    double value = w[a.anchor];
    for (int k = 0; k < a.size; ++k) value = fold(w[k], value, a.is_max);
    store_cast<double>(a.out, base + x0 + lx, value, a.tout);
  }
}

// Strided axis (inner > 1): a tile of 32 columns x 64 outputs; thread
// (x, y) folds outputs y, y + 8, ..., y + 56 of column x.
__global__ void __launch_bounds__(kColTI * kColTY) k_minmax_cols(const MinMaxArgs a) {
  extern __shared__ double s_tile[];
  long long bid = blockIdx.x;
  const long long it = bid % a.tiles_a;
  bid /= a.tiles_a;
  const long long l0 = (bid % a.tiles_b) * kColTL;
  const long long o = bid / a.tiles_b;
  const long long i = it * kColTI + threadIdx.x;
  const long long line0 = o * a.L * a.inner + i;
  const long long need = a.L - l0 + a.size - 1;
  const int n = need < kColTL + a.size - 1 ? static_cast<int>(need) : kColTL + a.size - 1;
  const bool col_in = i < a.inner;
  for (int j = threadIdx.y; j < n; j += kColTY)
    s_tile[j * kColTI + threadIdx.x] = col_in ? staged(a, line0, l0 - a.anchor + j, a.inner) : 0.0;
  __syncthreads();
  if (!col_in) return;
#pragma unroll
  for (int p = 0; p < kColP; ++p) {
    const int ly = threadIdx.y + p * kColTY;
    if (l0 + ly >= a.L) break;
    const double* w = s_tile + ly * kColTI + threadIdx.x;
    double value = w[a.anchor * kColTI];
    for (int k = 0; k < a.size; ++k) value = fold(w[k * kColTI], value, a.is_max);
    store_cast<double>(a.out, line0 + (l0 + ly) * a.inner, value, a.tout);
  }
}

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
               size, anchor, mode, is_max ? 1 : 0, cval, 0, 0};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_minmax_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
    cudaFuncSetAttribute(k_minmax_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  });
  const long long L = a.L;
  const size_t row_smem = sizeof(double) * ((size_t)kRowSeg + size - 1);
  const size_t col_smem = sizeof(double) * kColTI * ((size_t)kColTL + size - 1);
  if (inner == 1 && row_smem <= (size_t)kMaxSmem) {
    a.tiles_b = (L + kRowSeg - 1) / kRowSeg;
    const long long blocks = outer * a.tiles_b;
    if (blocks <= 0x7fffffffLL) {
      k_minmax_rows<<<(unsigned)blocks, kRowT, row_smem, st>>>(a);
      return cuda_fail(cudaGetLastError(), "min/max filter launch");
    }
  } else if (inner > 1 && col_smem <= (size_t)kMaxSmem) {
    a.tiles_a = (inner + kColTI - 1) / kColTI;
    a.tiles_b = (L + kColTL - 1) / kColTL;
    const long long blocks = a.tiles_a * a.tiles_b * outer;
    if (blocks <= 0x7fffffffLL) {
      k_minmax_cols<<<(unsigned)blocks, dim3(kColTI, kColTY), col_smem, st>>>(a);
      return cuda_fail(cudaGetLastError(), "min/max filter launch");
    }
  }
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
  k_minmax1d<<<(unsigned)blocks, 256, 0, st>>>(a);
  return cuda_fail(cudaGetLastError(), "min/max filter launch");
}
