// cimx_common.cuh — element access, the output cast rule and boundary index
// maps shared by all libcimx kernels.
//
// Semantics follow cuCIM (paths relative to python/cucim/src/cucim/skimage):
//   cast<D>(): _vendored/_ndimage_filters_core.py:227-244 — a plain C cast,
//     except float -> unsigned which is (a >= 0) ? (D)a : -(D)(-a). The C
//     casts below are compiled by the same NVVM backend cuCIM's NVRTC kernels
//     use, so saturation and wrap-around of out-of-range values match.
//   boundary maps: _vendored/_ndimage_util.py:186-308.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/cimx.h"

namespace cimx {

// dtype codes are numpy dtype.char values
enum : int {
  DT_U8 = 'B', DT_I8 = 'b', DT_U16 = 'H', DT_I16 = 'h', DT_U32 = 'I', DT_I32 = 'i',
  DT_U64 = 'L', DT_U64Q = 'Q', DT_I64 = 'l', DT_I64Q = 'q', DT_F16 = 'e', DT_F32 = 'f',
  DT_F64 = 'd', DT_C64 = 'F', DT_C128 = 'D',
};

__host__ __device__ inline int dtype_size(int dt) {
  switch (dt) {
    case DT_U8: case DT_I8: return 1;
    case DT_U16: case DT_I16: case DT_F16: return 2;
    case DT_U32: case DT_I32: case DT_F32: return 4;
    case DT_U64: case DT_U64Q: case DT_I64: case DT_I64Q: case DT_F64: return 8;
    default: return 0;
  }
}

// complex64 / complex128: taken only by the entries that filter complex
// arrays (cimx_correlate1d, cimx_separable); dtype_size() leaves them out so
// every other entry rejects them as unsupported
__host__ __device__ inline bool is_complex_dt(int dt) { return dt == DT_C64 || dt == DT_C128; }
__host__ __device__ inline int element_size(int dt) {
  return dt == DT_C64 ? 8 : dt == DT_C128 ? 16 : dtype_size(dt);
}

// ---------------------------------------------------------------- casts

// Float -> 8/16-bit integer conversion of the GPU: truncation toward zero,
// saturation to the 16-bit range (unsigned for a uint16 target, signed for
// the 8-bit and int16 targets), NaN -> 0; an 8-bit target keeps the low 8
// bits. This is the conversion a scalar store of the C cast compiles to. It
// is written out in PTX because an out-of-range C cast is undefined, and the
// compiler may fold a narrow conversion whose result is widened again (packed
// into a vector, merged with another store, converted back to float) into
// one wider conversion, which wraps instead of saturating.
template <class B, class A>
__device__ __forceinline__ uint32_t cvt_rzi16(A a) {
  unsigned short u;
  if constexpr (std::is_same<A, double>::value) {
    if constexpr (std::is_same<B, unsigned short>::value)
      asm("cvt.rzi.u16.f64 %0, %1;" : "=h"(u) : "d"(a));
    else
      asm("cvt.rzi.s16.f64 %0, %1;" : "=h"(u) : "d"(a));
  } else {
    const float f = static_cast<float>(a);
    if constexpr (std::is_same<B, unsigned short>::value)
      asm("cvt.rzi.u16.f32 %0, %1;" : "=h"(u) : "f"(f));
    else
      asm("cvt.rzi.s16.f32 %0, %1;" : "=h"(u) : "f"(f));
  }
  return u;
}

template <class B, class A>
__device__ __forceinline__ B out_cast(A a) {
  if constexpr (std::is_same<B, __half>::value) {
    return __float2half_rn(static_cast<float>(a));
  } else if constexpr (std::is_floating_point<A>::value && std::is_integral<B>::value &&
                       sizeof(B) <= 2) {
    if constexpr (!std::is_signed<B>::value) {
      // (a >= 0) ? (B)a : -(B)(-a); NaN takes the second side and gives 0
      const bool neg = !(a >= 0);
      const uint32_t v = cvt_rzi16<B>(neg ? -a : a);
      return static_cast<B>(neg ? 0u - v : v);
    } else {
      return static_cast<B>(cvt_rzi16<B>(a));
    }
  } else if constexpr (std::is_floating_point<A>::value && !std::is_signed<B>::value) {
    return (a >= 0) ? static_cast<B>(a) : static_cast<B>(-static_cast<B>(-a));
  } else {
    return static_cast<B>(a);
  }
}

template <class W, class T>
__device__ __forceinline__ W to_w(T v) {
  if constexpr (std::is_same<T, __half>::value) {
    return static_cast<W>(__half2float(v));
  } else {
    return static_cast<W>(v);
  }
}

// Runtime-typed load of element i as W (used by the generic kernels).
template <class W>
__device__ __forceinline__ W load_as(const void* __restrict__ p, int64_t i, int dt) {
  switch (dt) {
    case DT_F32: return to_w<W>(static_cast<const float*>(p)[i]);
    case DT_U16: return to_w<W>(static_cast<const uint16_t*>(p)[i]);
    case DT_U8: return to_w<W>(static_cast<const uint8_t*>(p)[i]);
    case DT_F64: return to_w<W>(static_cast<const double*>(p)[i]);
    case DT_I16: return to_w<W>(static_cast<const int16_t*>(p)[i]);
    case DT_I8: return to_w<W>(static_cast<const int8_t*>(p)[i]);
    case DT_U32: return to_w<W>(static_cast<const uint32_t*>(p)[i]);
    case DT_I32: return to_w<W>(static_cast<const int32_t*>(p)[i]);
    case DT_U64: case DT_U64Q: return to_w<W>(static_cast<const unsigned long long*>(p)[i]);
    case DT_I64: case DT_I64Q: return to_w<W>(static_cast<const long long*>(p)[i]);
    case DT_F16: return to_w<W>(static_cast<const __half*>(p)[i]);
    default: return W(0);
  }
}

// Runtime-typed store of a W value with the cast<D>() rule.
template <class W>
__device__ __forceinline__ void store_cast(void* __restrict__ p, int64_t i, W v, int dt) {
  switch (dt) {
    case DT_F32: static_cast<float*>(p)[i] = out_cast<float>(v); break;
    case DT_U16: static_cast<uint16_t*>(p)[i] = out_cast<unsigned short>(v); break;
    case DT_U8: static_cast<uint8_t*>(p)[i] = out_cast<unsigned char>(v); break;
    case DT_F64: static_cast<double*>(p)[i] = out_cast<double>(v); break;
    case DT_I16: static_cast<int16_t*>(p)[i] = out_cast<short>(v); break;
    case DT_I8: static_cast<int8_t*>(p)[i] = out_cast<signed char>(v); break;
    case DT_U32: static_cast<uint32_t*>(p)[i] = out_cast<unsigned int>(v); break;
    case DT_I32: static_cast<int32_t*>(p)[i] = out_cast<int>(v); break;
    case DT_U64: case DT_U64Q:
      static_cast<unsigned long long*>(p)[i] = out_cast<unsigned long long>(v); break;
    case DT_I64: case DT_I64Q: static_cast<long long*>(p)[i] = out_cast<long long>(v); break;
    case DT_F16: static_cast<__half*>(p)[i] = out_cast<__half>(v); break;
    default: break;
  }
}

// Fill value of constant mode as a W value: (W)cval for the elementwise
// kernel's rule, (W)static_cast<T>(cval) for the shared-memory kernel's
// (T = the dtype the pass reads).
template <class W>
__device__ __forceinline__ W fill_value(double cval, int as_input, int dt) {
  if (!as_input) return static_cast<W>(cval);
  switch (dt) {
    case DT_F32: return static_cast<W>(static_cast<float>(cval));
    case DT_F64: return static_cast<W>(cval);
    // 8/16-bit: the GPU conversion of the C cast, written out (cvt_rzi16)
    case DT_U8: return static_cast<W>(static_cast<unsigned char>(cvt_rzi16<unsigned char>(cval)));
    case DT_I8: return static_cast<W>(static_cast<signed char>(cvt_rzi16<signed char>(cval)));
    case DT_U16: return static_cast<W>(static_cast<unsigned short>(cvt_rzi16<unsigned short>(cval)));
    case DT_I16: return static_cast<W>(static_cast<short>(cvt_rzi16<short>(cval)));
    case DT_U32: return static_cast<W>(static_cast<unsigned int>(cval));
    case DT_I32: return static_cast<W>(static_cast<int>(cval));
    case DT_U64: case DT_U64Q: return static_cast<W>(static_cast<unsigned long long>(cval));
    case DT_I64: case DT_I64Q: return static_cast<W>(static_cast<long long>(cval));
    case DT_F16: return static_cast<W>(__half2float(__float2half_rn(static_cast<float>(cval))));
    default: return W(0);
  }
}

// ------------------------------------------------------- boundary maps
//
// Map a (possibly out-of-range) coordinate along an axis of length n to the
// coordinate it reads. Returns -1 for constant mode outside the array.
__host__ __device__ __forceinline__ int64_t map_coord(int64_t ix, int64_t n, int mode) {
  if (ix >= 0 && ix < n) return ix;
  switch (mode) {
    case CIMX_MODE_REFLECT: {
      if (ix < 0) ix = -1 - ix;
      ix %= 2 * n;
      const int64_t r = 2 * n - 1 - ix;
      return r < ix ? r : ix;
    }
    case CIMX_MODE_MIRROR: {
      if (n == 1) return 0;
      if (ix < 0) ix = -ix;
      ix = 1 + (ix - 1) % ((n - 1) * 2);
      const int64_t r = 2 * n - 2 - ix;
      return r < ix ? r : ix;
    }
    case CIMX_MODE_NEAREST:
      return ix < 0 ? 0 : n - 1;
    case CIMX_MODE_GRID_WRAP: {
      ix %= n;
      return ix < 0 ? ix + n : ix;
    }
    default:
      return -1;
  }
}

// 32-bit variant for kernels whose axis length fits in int.
__host__ __device__ __forceinline__ int map_coord32(int ix, int n, int mode) {
  if (ix >= 0 && ix < n) return ix;
  switch (mode) {
    case CIMX_MODE_REFLECT: {
      if (ix < 0) ix = -1 - ix;
      ix %= 2 * n;
      const int r = 2 * n - 1 - ix;
      return r < ix ? r : ix;
    }
    case CIMX_MODE_MIRROR: {
      if (n == 1) return 0;
      if (ix < 0) ix = -ix;
      ix = 1 + (ix - 1) % ((n - 1) * 2);
      const int r = 2 * n - 2 - ix;
      return r < ix ? r : ix;
    }
    case CIMX_MODE_NEAREST:
      return ix < 0 ? 0 : n - 1;
    case CIMX_MODE_GRID_WRAP: {
      ix %= n;
      return ix < 0 ? ix + n : ix;
    }
    default:
      return -1;
  }
}

// map_coord with the common case first: an overhang of at most one axis
// length (every tap window shorter than the axis) needs one reflection or
// shift, computed without a division; longer ones take map_coord's periodic
// formula. The same index as map_coord. For code that maps many elements
// (tile borders, generic passes); the streaming kernels keep the plain
// map_coord, whose smaller inlined body suits their per-row loops.
__host__ __device__ __forceinline__ int64_t map_coord_near(int64_t ix, int64_t n, int mode) {
  if (ix >= 0 && ix < n) return ix;
  switch (mode) {
    case CIMX_MODE_REFLECT:
      if (ix >= -n && ix < 2 * n) return ix < 0 ? -1 - ix : 2 * n - 1 - ix;
      break;
    case CIMX_MODE_MIRROR:
      if (n == 1) return 0;
      if (ix > -n && ix < 2 * n - 1) return ix < 0 ? -ix : 2 * n - 2 - ix;
      break;
    case CIMX_MODE_NEAREST:
      return ix < 0 ? 0 : n - 1;
    case CIMX_MODE_GRID_WRAP:
      if (ix >= -n && ix < 2 * n) return ix < 0 ? ix + n : ix - n;
      break;
    default:
      return -1;
  }
  return map_coord(ix, n, mode);
}

}  // namespace cimx
