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

template <class F>
__device__ __forceinline__ F fold(F v, F value, int is_max) {
  return is_max ? fmax(v, value) : fmin(v, value);
}

// Staged value of line coordinate c (boundary map outside [0, L)), as F.
template <class F>
__device__ __forceinline__ F staged(const MinMaxArgs& a, long long line0, long long c,
                                    long long stride) {
  const long long m = (c >= 0 && c < a.L) ? c : map_coord_near(c, a.L, a.mode);
  return m < 0 ? static_cast<F>(a.cval) : load_as<F>(a.in, line0 + m * stride, a.tin);
}

// Folds P consecutive outputs: value[j] starts at window element j + anchor
// (the output's own input element) and takes window elements j + k, k = 0 ..
// size - 1, in order. `at(q)` returns window element q; the window slides in
// registers, reloaded once per P taps.
template <int P, class F, class At>
__device__ __forceinline__ void fold_block(F (&value)[P], int size, int anchor, int is_max,
                                           At at) {
#pragma unroll
  for (int j = 0; j < P; ++j) value[j] = at(j + anchor);
  F win[2 * P];
#pragma unroll
  for (int j = 0; j < P; ++j) win[j] = at(j);
  for (int k0 = 0; k0 < size; k0 += P) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int kk = 0; kk < P; ++kk) {
      if (k0 + kk < size) {
#pragma unroll
        for (int j = 0; j < P; ++j) value[j] = fold(win[j + kk], value[j], is_max);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) win[j] = win[P + j];
  }
}

// Last axis (inner == 1): one CTA per 1024 outputs of a row; thread t folds
// outputs 4t .. 4t + 3 of the segment. The staged stretch is padded by one
// double every 4, so that lanes reading at a stride of 4 hit distinct banks.
__device__ __forceinline__ int pad4(int j) { return j + (j >> 2); }

template <class F>
__global__ void __launch_bounds__(kRowT) k_minmax_rows(const MinMaxArgs a) {
  extern __shared__ __align__(16) unsigned char s_raw_rows[];
  F* s_line = reinterpret_cast<F*>(s_raw_rows);
  const long long row = blockIdx.x / a.tiles_b;
  const long long x0 = (blockIdx.x % a.tiles_b) * kRowSeg;
  const long long base = row * a.L;
  // the staged stretch: only as far as the stored outputs (x < L) read
  const long long need = a.L - x0 + a.size - 1;
  const int n = need < kRowSeg + a.size - 1 ? static_cast<int>(need) : kRowSeg + a.size - 1;
  const long long c0 = x0 - a.anchor;
  for (int j = threadIdx.x; j < n; j += kRowT) s_line[pad4(j)] = staged<F>(a, base, c0 + j, 1);
  __syncthreads();
  const int lx = kRowP * threadIdx.x;
  if (x0 + lx >= a.L) return;
  F value[kRowP];
  fold_block<kRowP>(value, a.size, a.anchor, a.is_max,
                    [&](int q) { return s_line[pad4(lx + q)]; });
#pragma unroll
  for (int j = 0; j < kRowP; ++j)
    if (x0 + lx + j < a.L) store_cast<F>(a.out, base + x0 + lx + j, value[j], a.tout);
}

// Strided axis (inner > 1): a tile of 32 columns x 64 outputs; thread
// (x, y) folds outputs 8y .. 8y + 7 of column x.
template <class F>
__global__ void __launch_bounds__(kColTI * kColTY) k_minmax_cols(const MinMaxArgs a) {
  extern __shared__ __align__(16) unsigned char s_raw_cols[];
  F* s_tile = reinterpret_cast<F*>(s_raw_cols);
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
    s_tile[j * kColTI + threadIdx.x] = col_in ? staged<F>(a, line0, l0 - a.anchor + j, a.inner) : F(0);
  __syncthreads();
  const int ly = kColP * threadIdx.y;
  if (!col_in || l0 + ly >= a.L) return;
  F value[kColP];
  fold_block<kColP>(value, a.size, a.anchor, a.is_max,
                    [&](int q) { return s_tile[(ly + q) * kColTI + threadIdx.x]; });
#pragma unroll
  for (int j = 0; j < kColP; ++j)
    if (l0 + ly + j < a.L)
      store_cast<F>(a.out, line0 + (l0 + ly + j) * a.inner, value[j], a.tout);
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
    cudaFuncSetAttribute(k_minmax_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_minmax_cols<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_minmax_rows<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_minmax_cols<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
  });
  // The fold is exact in float32 when every value it sees is: inputs of at
  // most float32 precision, and a fill value that float32 holds (or none).
  // Rounding is monotonic, so the float32 min / max of the rounded values is
  // the rounding of the float64 one, the same real number, stored with the
  // same cast; nan and the zeros' signs behave alike in both precisions.
  const int tin = in->dtype;
  const bool f32_in = tin == DT_U8 || tin == DT_I8 || tin == DT_U16 || tin == DT_I16 ||
                      tin == DT_F16 || tin == DT_F32;
  const bool fill_exact = mode != CIMX_MODE_CONSTANT ||
                          static_cast<double>(static_cast<float>(cval)) == cval;
  const bool use_f32 = f32_in && fill_exact;
  const size_t fsz = use_f32 ? sizeof(float) : sizeof(double);
  const long long L = a.L;
  // fold_block reads window elements up to (size rounded up to P) + P - 1
  // past a thread's first output: the tiles are sized for that
  const size_t row_span = (size_t)kRowSeg + (size + kRowP - 1) / kRowP * kRowP + kRowP;
  const size_t col_span = (size_t)kColTL + (size + kColP - 1) / kColP * kColP + kColP;
  const size_t row_smem = fsz * (row_span + row_span / 4 + 1);
  const size_t col_smem = fsz * kColTI * col_span;
  if (inner == 1 && row_smem <= (size_t)kMaxSmem) {
    a.tiles_b = (L + kRowSeg - 1) / kRowSeg;
    const long long blocks = outer * a.tiles_b;
    if (blocks <= 0x7fffffffLL) {
      if (use_f32) k_minmax_rows<float><<<(unsigned)blocks, kRowT, row_smem, st>>>(a);
      else k_minmax_rows<double><<<(unsigned)blocks, kRowT, row_smem, st>>>(a);
      return cuda_fail(cudaGetLastError(), "min/max filter launch");
    }
  } else if (inner > 1 && col_smem <= (size_t)kMaxSmem) {
    a.tiles_a = (inner + kColTI - 1) / kColTI;
    a.tiles_b = (L + kColTL - 1) / kColTL;
    const long long blocks = a.tiles_a * a.tiles_b * outer;
    if (blocks <= 0x7fffffffLL) {
      if (use_f32) k_minmax_cols<float><<<(unsigned)blocks, dim3(kColTI, kColTY), col_smem, st>>>(a);
      else k_minmax_cols<double><<<(unsigned)blocks, dim3(kColTI, kColTY), col_smem, st>>>(a);
      return cuda_fail(cudaGetLastError(), "min/max filter launch");
    }
  }
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
  k_minmax1d<<<(unsigned)blocks, 256, 0, st>>>(a);
  return cuda_fail(cudaGetLastError(), "min/max filter launch");
}
