// cimx_pass.cu — the generic single-pass separable correlation kernels.
//
// One launch applies one 1-D correlation along the middle axis of the
// C-contiguous view (outer, L, inner) of an n-D array: any axis, any real
// dtype pair, any tap count, every boundary mode. These kernels serve every
// call the fused kernels (cimx_fused.cu) do not take.
//
// Per output the arithmetic is cuCIM's: taps in ascending order, one fused
// multiply-add chain in W starting from +0, then cast<D>() (see
// cimx_common.cuh). The halo'd tile is staged in shared memory once, each
// thread keeps a sliding window of 2*P inputs in registers and produces P
// consecutive outputs, so a tap costs one broadcast shared load per P FMAs.
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

constexpr int P = 8;            // outputs per thread along the filtered axis
constexpr int kColTI = 32;      // column kernel: inner-axis width of a tile
constexpr int kColTY = 8;       // column kernel: threads along the filtered axis
constexpr int kColTL = kColTY * P;
constexpr int kCol2TY = 16;     // pair column kernel: threads along the filtered axis
constexpr int kCol2TL = kCol2TY * P;
constexpr int kMaxSmem = 227 * 1024;

template <class W>
struct TapBlock {
  W w[kParamTapBytes / sizeof(W)];
};

struct GArgs {
  const void* in;
  void* out;
  int tin, tout;
  long long outer, L, inner;
  int K, K8, anchor, mode;
  double cval;
  int cval_as_input;
  const void* gtaps;   // device copy of the taps when they exceed the parameter block
  long long tiles_a, tiles_b;
};

template <class W>
__device__ __forceinline__ void load_taps(W* taps, const GArgs& a, const TapBlock<W>& tb,
                                          int tid, int nthr) {
  const W* src = a.gtaps ? static_cast<const W*>(a.gtaps) : tb.w;
  for (int k = tid; k < a.K8; k += nthr) taps[k] = k < a.K ? src[k] : W(0);
}

// Sliding-window tap loop shared by the row and column kernels. `at(q)`
// returns the staged input at logical offset q from this thread's first
// output; the chain for output p is acc[p] = fma(x[p + k], w[k], acc[p]).
template <class W, bool SKIPZ, class At>
__device__ __forceinline__ void tap_loop(W (&acc)[P], const W* taps, int K, At at) {
  W win[2 * P];
#pragma unroll
  for (int j = 0; j < P; ++j) win[j] = at(j);
  int k0 = 0;
  // full chunks of P taps: no bound test
  for (; k0 + P <= K; k0 += P) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const W w = taps[k0 + j];
      if (!SKIPZ || w != W(0)) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma(win[p + j], w, acc[p]);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) win[j] = win[P + j];
  }
  if (k0 < K) {
    // the last K - k0 < P taps
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const W w = taps[k0 + j];
      if (k0 + j < K && (!SKIPZ || w != W(0))) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma(win[p + j], w, acc[p]);
      }
    }
  }
}

// Value of line coordinate c (boundary mode applied) of a float32 input.
__device__ __forceinline__ float staged_f32(const float* line, long long stride, long long c,
                                            long long L, int mode, float cv) {
  const long long m = (c >= 0 && c < L) ? c : map_coord_near(c, L, mode);
  return m < 0 ? cv : __ldg(line + m * stride);
}

// Element m of a line as W: typed for the common input dtypes (TI = the
// element type), by the runtime dtype code otherwise (TI = void). Plain
// loads: the read-only data cache path measured no faster on columns and
// slower on short rows (20000 x 100 float32: 28.5 -> 42.3 us).
template <class TI, class W>
__device__ __forceinline__ W line_value(const void* line, long long m, int dt) {
  if constexpr (std::is_void<TI>::value) return load_as<W>(line, m, dt);
  else return to_w<W>(static_cast<const TI*>(line)[m]);
}

// Stage columns c0 .. c0 + n - 1 of one line into the padded row buffer as
// W. The in-range columns load straight from the line, eight loads in flight
// per thread before the shared stores; the few beyond either end (at most
// the halo) go through the boundary map in a loop of their own, the fill
// value where it gives -1.
template <class TI, class W>
__device__ __forceinline__ void stage_row(W* rb, const void* line, int dt, long long c0, int n,
                                          long long L, int mode, W cv, int lane, int nl) {
  const long long lo = -c0, hi = L - c0;
  const int jlo = static_cast<int>(lo < 0 ? 0 : (lo > n ? n : lo));
  const int jhi = static_cast<int>(hi < jlo ? jlo : (hi > n ? n : hi));
  const void* base = static_cast<const unsigned char*>(line) +
                     c0 * static_cast<long long>(dtype_size(dt));  // column c0
  for (int jb = jlo + lane; jb < jhi; jb += 8 * nl) {
    W v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = jb + q * nl;
      if (j < jhi) v[q] = line_value<TI, W>(base, j, dt);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = jb + q * nl;
      if (j < jhi) rb[j + (j >> 3)] = v[q];
    }
  }
  const int nout = jlo + (n - jhi);
  for (int t = lane; t < nout; t += nl) {
    const int j = t < jlo ? t : jhi + (t - jlo);
    const long long m = map_coord_near(c0 + j, L, mode);
    rb[j + (j >> 3)] = m < 0 ? cv : line_value<TI, W>(line, m, dt);
  }
}

// Filter along the contiguous last axis (inner == 1). Block = (seg_threads,
// rows); each row buffer is padded by one word every 8 so that lanes reading
// at a stride of P words hit distinct banks. For 32- and 64-bit outputs the
// P outputs of a thread go back through the row buffer, so that the stores
// of a warp cover consecutive elements. TI: the input element type, or void
// for the runtime-typed loads. Six CTAs per SM with float weights (40
// registers, a few spilled), four with double: measured faster than the
// compiler's own choice (48-64 registers) on every dtype pair.
template <class W, bool SKIPZ, class TI>
__global__ void __launch_bounds__(256, sizeof(W) == 4 ? 6 : 4) k_rows(GArgs a, TapBlock<W> tb) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  W* taps = reinterpret_cast<W*>(sm_raw);
  const int nthr = blockDim.x * blockDim.y;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  load_taps(taps, a, tb, tid, nthr);
  const int seg = blockDim.x * P;
  const int span = seg + a.K8 + P;
  const int pspan = span + (span >> 3) + 1;
  W* rb = taps + a.K8 + threadIdx.y * pspan;

  const long long sg = blockIdx.x % a.tiles_b;
  const long long rg = blockIdx.x / a.tiles_b;
  const long long row = rg * blockDim.y + threadIdx.y;
  const long long x0 = sg * seg;
  const W cv = fill_value<W>(a.cval, a.cval_as_input, a.tin);
  const long long rbase = row * a.L;
  const bool live = row < a.outer;
  if (live) {
    // only the columns that the stored outputs (x < L) read: a row shorter
    // than the segment stages L - x0 + K8 + P columns, not the whole span
    const long long need = a.L - x0 + a.K8 + P;
    const int n = need < span ? static_cast<int>(need) : span;
    const void* line = static_cast<const unsigned char*>(a.in) +
                       rbase * static_cast<long long>(dtype_size(a.tin));
    stage_row<TI, W>(rb, line, a.tin, x0 - a.anchor, n, a.L, a.mode, cv, threadIdx.x,
                     blockDim.x);
  }
  __syncthreads();
  const int b = threadIdx.x * P;
  W acc[P];
#pragma unroll
  for (int p = 0; p < P; ++p) acc[p] = W(0);
  if (live)
    tap_loop<W, SKIPZ>(acc, taps, a.K, [&](int q) {
      const int x = b + q;
      return rb[x + (x >> 3)];
    });
  if (dtype_size(a.tout) < 4) {
    // 8- and 16-bit outputs: straight from the accumulators (measured faster
    // than going back through the buffer)
    if (!live) return;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const long long x = x0 + b + p;
      if (x < a.L) store_cast<W>(a.out, rbase + x, acc[p], a.tout);
    }
    return;
  }
  __syncthreads();  // every window read is done before the outputs overwrite the buffer
  if (live) {
#pragma unroll
    for (int p = 0; p < P; ++p) rb[b + p + ((b + p) >> 3)] = acc[p];
  }
  __syncthreads();  // a row spans blockDim.x / 32 warps
  if (!live) return;
  for (int j = threadIdx.x; j < seg; j += blockDim.x) {
    const long long x = x0 + j;
    if (x < a.L) store_cast<W>(a.out, rbase + x, rb[j + (j >> 3)], a.tout);
  }
}

// Filter along a strided axis (inner > 1). Block = (32 inner columns, 8);
// each thread produces P consecutive outputs of one column. With typed loads
// (TI: see with_input_type; void: runtime-typed) a tile inside the line
// walks its rows directly; otherwise each staged row's mapped offset comes
// from a table built once per CTA.
template <class W, bool SKIPZ, class TI>
__global__ void __launch_bounds__(256, sizeof(W) == 4 ? 6 : 4) k_cols(GArgs a, TapBlock<W> tb) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  W* taps = reinterpret_cast<W*>(sm_raw);
  const int tid = threadIdx.y * kColTI + threadIdx.x;
  load_taps(taps, a, tb, tid, kColTI * kColTY);
  W* buf = taps + a.K8;
  const int span = kColTL + a.K8 + P;
  // element index of each staged row's mapped line coordinate (column 0),
  // -1 for the fill value: the boundary map runs once per row
  long long* rowoff = reinterpret_cast<long long*>(buf + (size_t)span * kColTI);

  long long bid = blockIdx.x;
  const long long it = bid % a.tiles_a;
  bid /= a.tiles_a;
  const long long lt = bid % a.tiles_b;
  const long long o = bid / a.tiles_b;
  const long long i = it * kColTI + threadIdx.x;
  const long long l0 = lt * kColTL;
  const W cv = fill_value<W>(a.cval, a.cval_as_input, a.tin);
  const long long obase = o * a.L;
  const bool interior = l0 - a.anchor >= 0 && l0 - a.anchor + span <= a.L;
  // typed loads: an interior tile walks its rows, eight loads in flight;
  // the other dtypes take one runtime-typed load per row (measured at six
  // CTAs per SM: typed staging 1.6x faster for float64, 4-5 % for uint16 /
  // uint8; eight-wide runtime-typed staging 5-8 % slower)
  constexpr bool kTyped = !std::is_void<TI>::value;
  const bool walk = interior && kTyped;
  if (!walk) {  // the same for every thread of the CTA
    for (int j = tid; j < span; j += kColTI * kColTY) {
      const long long cj = l0 - a.anchor + j;
      const long long m = map_coord_near(cj, a.L, a.mode);
      rowoff[j] = m < 0 ? -1 : (obase + m) * a.inner;
    }
    __syncthreads();
  }
  if constexpr (kTyped) {
    // element offset of staged row j (column 0): a walk inside the line,
    // the table otherwise (-1: the fill value); eight loads in flight
    const long long walk0 = (obase + l0 - a.anchor) * a.inner;
    for (int jb = threadIdx.y; jb < span; jb += 8 * kColTY) {
      W v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = jb + q * kColTY;
        v[q] = W(0);
        if (j < span && i < a.inner) {
          const long long off = walk ? walk0 + (long long)j * a.inner : rowoff[j];
          v[q] = off < 0 ? cv : line_value<TI, W>(a.in, off + i, a.tin);
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = jb + q * kColTY;
        if (j < span) buf[j * kColTI + threadIdx.x] = v[q];
      }
    }
  } else {
    for (int j = threadIdx.y; j < span; j += kColTY) {
      W v = W(0);
      if (i < a.inner) {
        const long long off = rowoff[j];
        v = off < 0 ? cv : load_as<W>(a.in, off + i, a.tin);
      }
      buf[j * kColTI + threadIdx.x] = v;
    }
  }
  __syncthreads();
  if (i >= a.inner) return;
  const int b = threadIdx.y * P;
  W acc[P];
#pragma unroll
  for (int p = 0; p < P; ++p) acc[p] = W(0);
  tap_loop<W, SKIPZ>(acc, taps, a.K, [&](int q) { return buf[(b + q) * kColTI + threadIdx.x]; });
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const long long l = l0 + b + p;
    if (l < a.L) store_cast<W>(a.out, (obase + l) * a.inner + i, acc[p], a.tout);
  }
}

// Two float32 lanes in one 64-bit register (x in the low half) and their
// lane-wise fused multiply-add, each lane an IEEE float32 FMA rounded to
// nearest (bit-identical to fmaf on each lane).
using u64 = unsigned long long;
__device__ __forceinline__ u64 pair2(float x, float y) {
  return (static_cast<u64>(__float_as_uint(y)) << 32) | __float_as_uint(x);
}
__device__ __forceinline__ float lane_lo(u64 v) { return __uint_as_float(static_cast<unsigned>(v)); }
__device__ __forceinline__ float lane_hi(u64 v) {
  return __uint_as_float(static_cast<unsigned>(v >> 32));
}
__device__ __forceinline__ u64 fma_pair(u64 a, u64 b, u64 c) {
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// tap_loop on column pairs: `at(q)` returns the staged pair at offset q,
// taps hold (w, w); each lane is the same chain as tap_loop's.
template <bool SKIPZ, class At>
__device__ __forceinline__ void tap_loop_pairs(u64 (&acc)[P], const u64* taps, int K, At at) {
  u64 win[2 * P];
#pragma unroll
  for (int j = 0; j < P; ++j) win[j] = at(j);
  int k0 = 0;
  for (; k0 + P <= K; k0 += P) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const u64 w = taps[k0 + j];
      if (!SKIPZ || lane_lo(w) != 0.f) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma_pair(win[p + j], w, acc[p]);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) win[j] = win[P + j];
  }
  if (k0 < K) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const u64 w = taps[k0 + j];
      if (k0 + j < K && (!SKIPZ || lane_lo(w) != 0.f)) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma_pair(win[p + j], w, acc[p]);
      }
    }
  }
}

// k_cols for float32 input and float32 taps: block = (16 column pairs, 16);
// each thread produces P consecutive outputs of two adjacent columns with
// one f32x2 FMA per tap and output pair, and a tile is 32 columns x 128
// outputs (half the halo share of k_cols' 64-output tiles). Four CTAs per
// SM: with three (80 registers) the staging loads of short-tap passes had
// too few warps in flight. The boundary map runs once per staged row (a
// table of row offsets in shared memory) rather than per element, which
// took a fifth of the time off every pass. 256^3 float32, axis 0: 70, 95
// and 152 us at 23, 57 and 143 taps, against 89, 129 and 242 us for k_cols.
// TI: the input element type (float32, or uint16 / uint8 widened exactly
// to float32 as they are staged).
template <bool SKIPZ, class TI>
__global__ void __launch_bounds__(256, 4) k_cols_pairs(GArgs a, TapBlock<float> tb) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  u64* taps = reinterpret_cast<u64*>(sm_raw);
  const int tid = threadIdx.y * 16 + threadIdx.x;
  {
    const float* src = a.gtaps ? static_cast<const float*>(a.gtaps) : tb.w;
    for (int k = tid; k < a.K8; k += 256) {
      const float w = k < a.K ? src[k] : 0.f;
      taps[k] = pair2(w, w);
    }
  }
  float* buf = reinterpret_cast<float*>(taps + a.K8);  // span rows x 32 columns
  const int span = kCol2TL + a.K8 + P;
  // element offset of each staged row's mapped line coordinate, -1 for the
  // fill value: the boundary map runs once per row, not per element
  long long* rowoff = reinterpret_cast<long long*>(buf + (size_t)span * 32);

  long long bid = blockIdx.x;
  const long long it = bid % a.tiles_a;
  bid /= a.tiles_a;
  const long long lt = bid % a.tiles_b;
  const long long o = bid / a.tiles_b;
  const long long l0 = lt * kCol2TL;
  const float cv = fill_value<float>(a.cval, a.cval_as_input, a.tin);
  const long long obase = o * a.L;
  const long long c0 = l0 - a.anchor;
  for (int j = tid; j < span; j += 256) {
    const long long cj = c0 + j;
    const long long m = (cj >= 0 && cj < a.L) ? cj : map_coord_near(cj, a.L, a.mode);
    rowoff[j] = m < 0 ? -1 : m * a.inner;
  }
  __syncthreads();
  {
    // staging: thread (c, r) loads column c of rows r, r + 8, ..., eight
    // loads in flight before the stores
    const int c = tid & 31, r = tid >> 5;
    const long long ic = it * 32 + c;
    const TI* col = static_cast<const TI*>(a.in) + obase * a.inner + ic;
    const bool cin = ic < a.inner;
    for (int jb = r; jb < span; jb += 64) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = jb + q * 8;
        v[q] = 0.f;
        if (j < span && cin) {
          const long long off = rowoff[j];
          v[q] = off < 0 ? cv : static_cast<float>(__ldg(col + off));
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = jb + q * 8;
        if (j < span) buf[j * 32 + c] = v[q];
      }
    }
  }
  __syncthreads();
  const long long i = it * 32 + 2 * threadIdx.x;
  if (i >= a.inner) return;
  const int b = threadIdx.y * P;
  u64 acc[P];
#pragma unroll
  for (int p = 0; p < P; ++p) acc[p] = 0ull;
  const u64* pcol = reinterpret_cast<const u64*>(buf) + threadIdx.x;
  tap_loop_pairs<SKIPZ>(acc, taps, a.K, [&](int q) { return pcol[(b + q) * 16]; });
  const bool second = i + 1 < a.inner;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const long long l = l0 + b + p;
    if (l < a.L) {
      store_cast<float>(a.out, (obase + l) * a.inner + i, lane_lo(acc[p]), a.tout);
      if (second) store_cast<float>(a.out, (obase + l) * a.inner + i + 1, lane_hi(acc[p]), a.tout);
    }
  }
}

// Tap counts whose halo does not fit in shared memory: one thread per
// output, reading global memory per tap (taps in global memory).
template <class W, bool SKIPZ>
__global__ void __launch_bounds__(256) k_direct(GArgs a) {
  const W* taps = static_cast<const W*>(a.gtaps);
  const W cv = fill_value<W>(a.cval, a.cval_as_input, a.tin);
  const long long total = a.outer * a.L * a.inner;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % a.inner;
    const long long ol = e / a.inner;
    const long long l = ol % a.L;
    const long long obase = (ol - l);
    W acc = W(0);
    for (int k = 0; k < a.K; ++k) {
      const W w = taps[k];
      if (SKIPZ && w == W(0)) continue;
      const long long m = map_coord_near(l - a.anchor + k, a.L, a.mode);
      const W x = m < 0 ? cv : load_as<W>(a.in, (obase + m) * a.inner + i, a.tin);
      acc = fma(x, w, acc);
    }
    store_cast<W>(a.out, e, acc, a.tout);
  }
}

// Row kernel geometry for lines of L samples: threads per segment, rows per
// CTA and the dynamic shared memory (taps, padded row buffers).
struct RowGeom {
  int seg_threads, ry, seg;
  size_t smem;
};
inline RowGeom row_geom(long long L, int K8, size_t wsize) {
  RowGeom g;
  g.seg_threads = 256;
  while (g.seg_threads > 32 && (long long)(g.seg_threads / 2) * P >= L) g.seg_threads /= 2;
  g.ry = 256 / g.seg_threads;
  g.seg = g.seg_threads * P;
  const int span = g.seg + K8 + P;
  const int pspan = span + (span >> 3) + 1;
  g.smem = wsize * ((size_t)K8 + (size_t)g.ry * pspan);
  return g;
}

template <class Kern>
void allow_big_smem(Kern k) {
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
}

// The input dtypes with typed loads in k_cols / k_rows: float32, float16,
// uint16, int16, uint8 and int8 with float weights, float64, int32 and
// uint32 with double weights; the 64-bit integers are loaded by their
// runtime dtype code (TI = void).
template <class W, class F>
void with_input_type(int dt, F&& f) {
  if constexpr (std::is_same<W, float>::value) {
    switch (dt) {
      case DT_F32: f(static_cast<float*>(nullptr)); return;
      case DT_F16: f(static_cast<__half*>(nullptr)); return;
      case DT_U16: f(static_cast<uint16_t*>(nullptr)); return;
      case DT_I16: f(static_cast<int16_t*>(nullptr)); return;
      case DT_U8: f(static_cast<uint8_t*>(nullptr)); return;
      case DT_I8: f(static_cast<int8_t*>(nullptr)); return;
      default: break;
    }
  } else {
    switch (dt) {
      case DT_F64: f(static_cast<double*>(nullptr)); return;
      case DT_I32: f(static_cast<int32_t*>(nullptr)); return;
      case DT_U32: f(static_cast<uint32_t*>(nullptr)); return;
      default: break;
    }
  }
  f(static_cast<void*>(nullptr));
}

template <class W, bool SKIPZ>
void launch_cols(const GArgs& a, const TapBlock<W>& tb, dim3 grid, dim3 block, size_t smem,
                 cudaStream_t st) {
  with_input_type<W>(a.tin, [&](auto* tag) {
    using TI = std::remove_pointer_t<decltype(tag)>;
    static std::once_flag once;
    std::call_once(once, [] { allow_big_smem(k_cols<W, SKIPZ, TI>); });
    k_cols<W, SKIPZ, TI><<<grid, block, smem, st>>>(a, tb);
  });
}

template <class W, bool SKIPZ>
void launch_rows(const GArgs& a, const TapBlock<W>& tb, dim3 grid, dim3 block, size_t smem,
                 cudaStream_t st) {
  with_input_type<W>(a.tin, [&](auto* tag) {
    using TI = std::remove_pointer_t<decltype(tag)>;
    static std::once_flag once;
    std::call_once(once, [] { allow_big_smem(k_rows<W, SKIPZ, TI>); });
    k_rows<W, SKIPZ, TI><<<grid, block, smem, st>>>(a, tb);
  });
}

template <class W, bool SKIPZ>
int launch_t(GArgs a, const TapBlock<W>& tb, bool direct, cudaStream_t st) {
  static std::once_flag once;
  std::call_once(once, [] {
    if constexpr (std::is_same<W, float>::value) {
      allow_big_smem(k_cols_pairs<SKIPZ, float>);
      allow_big_smem(k_cols_pairs<SKIPZ, uint16_t>);
      allow_big_smem(k_cols_pairs<SKIPZ, uint8_t>);
    }
  });
  const long long total = a.outer * a.L * a.inner;
  if (total == 0) return CIMX_OK;
  if (direct) {
    const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 64);
    k_direct<W, SKIPZ><<<(unsigned)blocks, 256, 0, st>>>(a);
  } else if (a.inner == 1) {
    const RowGeom g = row_geom(a.L, a.K8, sizeof(W));
    a.tiles_b = (a.L + g.seg - 1) / g.seg;
    const long long blocks = ((a.outer + g.ry - 1) / g.ry) * a.tiles_b;
    launch_rows<W, SKIPZ>(a, tb, dim3((unsigned)blocks), dim3(g.seg_threads, g.ry), g.smem, st);
  } else {
    if constexpr (std::is_same<W, float>::value) {
      // float32 input (float32 taps) along lines longer than one k_cols tile:
      // column pairs
      const size_t span2 = (size_t)(kCol2TL + a.K8 + P);
      const size_t smem2 = 8 * (size_t)a.K8 + sizeof(float) * span2 * 32 + 8 * span2;
      // float32 input only: uint16 / uint8 input measured slower here than on
      // the typed k_cols for short taps (9 taps, 256 x 512^2 along axis 0:
      // 374 / 353 us against 350 / 338 us) and within 0-4 % for 21-33 taps
      const bool pair_in = a.tin == DT_F32;
      if (pair_in && a.inner >= 2 && a.L > kColTL && smem2 <= (size_t)kMaxSmem) {
        a.tiles_a = (a.inner + 31) / 32;
        a.tiles_b = (a.L + kCol2TL - 1) / kCol2TL;
        const long long blocks = a.tiles_a * a.tiles_b * a.outer;
        const dim3 grid((unsigned)blocks), block(16, kCol2TY);
        if (a.tin == DT_F32) k_cols_pairs<SKIPZ, float><<<grid, block, smem2, st>>>(a, tb);
        else if (a.tin == DT_U16) k_cols_pairs<SKIPZ, uint16_t><<<grid, block, smem2, st>>>(a, tb);
        else k_cols_pairs<SKIPZ, uint8_t><<<grid, block, smem2, st>>>(a, tb);
        return cuda_fail(cudaGetLastError(), "generic pass launch");
      }
    }
    const size_t smem = sizeof(W) * ((size_t)a.K8 + (size_t)(kColTL + a.K8 + P) * kColTI) +
                        8 * (size_t)(kColTL + a.K8 + P);
    a.tiles_a = (a.inner + kColTI - 1) / kColTI;
    a.tiles_b = (a.L + kColTL - 1) / kColTL;
    const long long blocks = a.tiles_a * a.tiles_b * a.outer;
    launch_cols<W, SKIPZ>(a, tb, dim3((unsigned)blocks), dim3(kColTI, kColTY), smem, st);
  }
  return cuda_fail(cudaGetLastError(), "generic pass launch");
}

template <class W>
int launch_w(const PassDesc& d, cudaStream_t st) {
  // Round the taps to W, then (elementwise-kernel rule) drop zero taps at
  // both ends: skipping them is exact whatever the input holds.
  std::vector<W> w(d.K);
  for (int k = 0; k < d.K; ++k) w[k] = static_cast<W>(d.taps[k]);
  int lo = 0, hi = d.K;
  if (d.skip_zero) {
    while (lo < hi && w[lo] == W(0)) ++lo;
    while (hi > lo && w[hi - 1] == W(0)) --hi;
  }
  const int K = hi - lo;
  bool interior_zero = false;
  if (d.skip_zero)
    for (int k = lo; k < hi; ++k) interior_zero |= (w[k] == W(0));

  GArgs a{};
  a.in = d.in;
  a.out = d.out;
  a.tin = d.tin;
  a.tout = d.tout;
  a.outer = d.outer;
  a.L = d.L;
  a.inner = d.inner;
  a.K = K;
  a.K8 = (K + P - 1) / P * P;
  a.anchor = d.anchor - lo;
  a.mode = d.mode;
  a.cval = d.cval;
  a.cval_as_input = d.cval_as_input ? 1 : 0;

  TapBlock<W> tb;
  std::fill(std::begin(tb.w), std::end(tb.w), W(0));
  const bool fits_param = K * sizeof(W) <= sizeof(tb.w);
  const size_t smem_rows = row_geom(a.L, a.K8, sizeof(W)).smem;
  const size_t smem_cols = sizeof(W) * ((size_t)a.K8 + (size_t)(kColTL + a.K8 + P) * kColTI) +
                           8 * (size_t)(kColTL + a.K8 + P);
  const bool direct = (a.inner == 1 ? smem_rows : smem_cols) > (size_t)kMaxSmem;
  void* gt = nullptr;
  const size_t gbytes = sizeof(W) * std::max(K, 1);
  if (fits_param && !direct) {
    std::copy(w.begin() + lo, w.begin() + hi, tb.w);
  } else {
    if (d.no_alloc)
      return fail(CIMX_E_INVALID,
                  "this pass needs device scratch memory for its " + std::to_string(K) +
                      " taps (beyond the launch parameters or the shared-memory budget), "
                      "which an entry point that allocates nothing cannot take");
    gt = scratch_alloc(gbytes, st);
    if (!gt) return fail(CIMX_E_NOMEM, "scratch allocation for taps failed");
    cudaError_t e = cudaMemcpyAsync(gt, w.data() + lo, sizeof(W) * K, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      scratch_free(gt, gbytes, st);
      return cuda_fail(e, "tap upload");
    }
    a.gtaps = gt;
  }
  int rc = interior_zero ? launch_t<W, true>(a, tb, direct, st)
                         : launch_t<W, false>(a, tb, direct, st);
  if (gt) scratch_free(gt, gbytes, st);
  return rc;
}

}  // namespace

int launch_generic_pass(const PassDesc& d, cudaStream_t stream) {
  return d.w64 ? launch_w<double>(d, stream) : launch_w<float>(d, stream);
}

}  // namespace cimx
