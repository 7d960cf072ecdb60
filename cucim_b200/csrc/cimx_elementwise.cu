// cimx_elementwise.cu — elementwise epilogues of the separable path:
// conversion copies, the square/accumulate/sqrt of gradient magnitudes,
// closed-form symmetric eigenvalues and rgb2gray.
//
// Each kernel evaluates the same expression, statement by statement, as the
// cuCIM kernel it replaces (cited per kernel), so the compiler's rounding and
// contraction decisions are the same ones cuCIM's kernels get.
#include <algorithm>
#include <cmath>
#include <vector>

#include <type_traits>

#include "cimx_common.cuh"
#include "cimx_fused.h"
#include "cimx_internal.h"

namespace cimx {
namespace {

inline unsigned grid_for(int64_t n, int threads = 256) {
  const int64_t b = (n + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

__global__ void k_copy_cast(const void* in, int tin, void* out, int tout, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = load_as<double>(in, i, tin);
    switch (tout) {
      case DT_F32: static_cast<float*>(out)[i] = static_cast<float>(v); break;
      case DT_F64: static_cast<double*>(out)[i] = v; break;
      case DT_F16: static_cast<__half*>(out)[i] = __float2half_rn(static_cast<float>(v)); break;
      case DT_U8: static_cast<uint8_t*>(out)[i] = static_cast<unsigned char>(v); break;
      case DT_I8: static_cast<int8_t*>(out)[i] = static_cast<signed char>(v); break;
      case DT_U16: static_cast<uint16_t*>(out)[i] = static_cast<unsigned short>(v); break;
      case DT_I16: static_cast<int16_t*>(out)[i] = static_cast<short>(v); break;
      case DT_U32: static_cast<uint32_t*>(out)[i] = static_cast<unsigned int>(v); break;
      case DT_I32: static_cast<int32_t*>(out)[i] = static_cast<int>(v); break;
      case DT_U64: case DT_U64Q:
        static_cast<unsigned long long*>(out)[i] = static_cast<unsigned long long>(v); break;
      default: static_cast<long long*>(out)[i] = static_cast<long long>(v); break;
    }
  }
}

// acc = t*t (first) or acc = acc + t*t, each product and sum rounded on its
// own: cuCIM runs `output *= output` and `output += tmp` as separate kernels
// (_vendored/_ndimage_filters.py:1080-1096, filters/edges.py:229-235).
template <class F>
__global__ void k_square_acc(F* acc, const F* t, int64_t n, int first) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (sizeof(F) == 4) {
      const float sq = __fmul_rn(t[i], t[i]);
      acc[i] = first ? sq : __fadd_rn(acc[i], sq);
    } else {
      const double sq = __dmul_rn(t[i], t[i]);
      acc[i] = first ? sq : __dadd_rn(acc[i], sq);
    }
  }
}

// acc = acc + t or acc - t in acc's dtype, as CuPy's `output += tmp`
// (_vendored/_ndimage_filters.py:888, generic_laplace) and `out -= ...`
// (filters/_gaussian.py:164, difference_of_gaussians) compute it: integers
// wrap around, floats round to nearest.
template <class T>
__global__ void k_combine(T* acc, const T* t, int64_t n, int sub) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (std::is_same<T, float>::value) {
      acc[i] = sub ? __fsub_rn(acc[i], t[i]) : __fadd_rn(acc[i], t[i]);
    } else if constexpr (std::is_same<T, double>::value) {
      acc[i] = sub ? __dsub_rn(acc[i], t[i]) : __dadd_rn(acc[i], t[i]);
    } else if constexpr (std::is_same<T, __half>::value) {
      acc[i] = sub ? __hsub(acc[i], t[i]) : __hadd(acc[i], t[i]);
    } else {
      using U = typename std::make_unsigned<T>::type;
      using W = typename std::conditional<(sizeof(T) < 4), uint32_t, U>::type;
      const W a = static_cast<W>(static_cast<U>(acc[i])), b = static_cast<W>(static_cast<U>(t[i]));
      acc[i] = static_cast<T>(static_cast<U>(sub ? a - b : a + b));
    }
  }
}

template <class T>
int launch_combine_t(void* acc, const void* t, int64_t n, int sub, cudaStream_t st) {
  k_combine<T><<<grid_for(n), 256, 0, st>>>(static_cast<T*>(acc), static_cast<const T*>(t), n, sub);
  return cuda_fail(cudaGetLastError(), "combine launch");
}

int launch_combine(void* acc, const void* t, int dt, int64_t n, int sub, cudaStream_t st) {
  switch (dt) {
    case DT_F32: return launch_combine_t<float>(acc, t, n, sub, st);
    case DT_F64: return launch_combine_t<double>(acc, t, n, sub, st);
    case DT_F16: return launch_combine_t<__half>(acc, t, n, sub, st);
    case DT_U8: return launch_combine_t<uint8_t>(acc, t, n, sub, st);
    case DT_I8: return launch_combine_t<int8_t>(acc, t, n, sub, st);
    case DT_U16: return launch_combine_t<uint16_t>(acc, t, n, sub, st);
    case DT_I16: return launch_combine_t<int16_t>(acc, t, n, sub, st);
    case DT_U32: return launch_combine_t<uint32_t>(acc, t, n, sub, st);
    case DT_I32: return launch_combine_t<int32_t>(acc, t, n, sub, st);
    case DT_U64: case DT_U64Q: return launch_combine_t<unsigned long long>(acc, t, n, sub, st);
    case DT_I64: case DT_I64Q: return launch_combine_t<long long>(acc, t, n, sub, st);
    default: return fail(CIMX_E_DTYPE, "combine: unsupported dtype");
  }
}

// filters/_unsharp_mask.py:12-20: result = image + (image - blurred) * amount,
// each operation a separate CuPy kernel (rounded on its own, no contraction),
// then cp.clip(result, lo, hi) when a range is given (nan passes through).
template <class F>
__global__ void k_unsharp(const F* __restrict__ img, const F* __restrict__ blur, F* out,
                          int64_t n, F amount, int clip, F lo, F hi) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    F r;
    if constexpr (sizeof(F) == 4) {
      r = __fadd_rn(img[i], __fmul_rn(__fsub_rn(img[i], blur[i]), amount));
    } else {
      r = __dadd_rn(img[i], __dmul_rn(__dsub_rn(img[i], blur[i]), amount));
    }
    if (clip) r = r < lo ? lo : (r > hi ? hi : r);
    out[i] = r;
  }
}

// any element < 0 (filters/_unsharp_mask.py:145, cp.any(fimg < 0))
template <class F>
__global__ void k_any_negative(const F* __restrict__ a, int64_t n, int* flag) {
  int found = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    found |= a[i] < F(0);
  if (__syncthreads_or(found) && threadIdx.x == 0) atomicOr(flag, 1);
}

template <class F>
__global__ void k_sqrt(F* acc, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc[i] = sqrt(acc[i]);
}

// feature/corner.py:473-527 — symmetric 2x2 eigenvalues.
template <class F>
__global__ void k_eig22(const F* __restrict__ M00, const F* __restrict__ M01,
                        const F* __restrict__ M11, F* lam1o, F* lam2o, int64_t n,
                        int descending, int abs_sort) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    F tmp1, tmp2;
    double m00 = static_cast<double>(M00[i]);
    double m01 = static_cast<double>(M01[i]);
    double m11 = static_cast<double>(M11[i]);
    tmp1 = m01 * m01;
    tmp1 *= 4;
    tmp2 = m00 - m11;
    tmp2 *= tmp2;
    tmp2 += tmp1;
    tmp2 = sqrt(tmp2);
    tmp2 /= 2;
    tmp1 = m00 + m11;
    tmp1 /= 2;
    F lam1, lam2;
    if (!descending) {
      lam1 = tmp1 - tmp2;
      lam2 = tmp1 + tmp2;
      if (abs_sort && abs(lam1) > abs(lam2)) {
        F s = lam1; lam1 = lam2; lam2 = s;
      }
    } else {
      lam1 = tmp1 + tmp2;
      lam2 = tmp1 - tmp2;
      if (abs_sort && abs(lam1) < abs(lam2)) {
        F s = lam1; lam1 = lam2; lam2 = s;
      }
    }
    lam1o[i] = lam1;
    lam2o[i] = lam2;
  }
}

// feature/corner.py:566-647 — symmetric 3x3 eigenvalues, float64 inside
// (Deledalle et al. closed form with the max(.,0) guards). Arguments are the
// matrix [[a d f] [d b e] [f e c]].
template <class F>
__device__ __forceinline__ void eig33(double a, double b, double c, double d, double e, double f,
                                      F& lam1, F& lam2, F& lam3) {
  double x1, x2, phi;
  double d_sq = d * d;
  double e_sq = e * e;
  double f_sq = f * f;
  double tmpa = (2 * a - b - c);
  double tmpb = (2 * b - a - c);
  double tmpc = (2 * c - a - b);
  x2 = -tmpa * tmpb * tmpc;
  x2 += 9 * (tmpc * d_sq + tmpb * f_sq + tmpa * e_sq);
  x2 -= 54 * (d * e * f);
  x1 = a * a + b * b + c * c - a * b - a * c - b * c + 3 * (d_sq + e_sq + f_sq);
  x1 = max(x1, 0.0);
  if (x2 == 0.0) {
    phi = M_PI / 2.0;
  } else {
    double arg = max(4 * x1 * x1 * x1 - x2 * x2, 0.0);
    phi = atan(sqrt(arg) / x2);
    if (x2 < 0) phi += M_PI;
  }
  double x1_term = (2.0 / 3.0) * sqrt(x1);
  double abc = (a + b + c) / 3.0;
  lam1 = abc - x1_term * cos(phi / 3.0);
  lam2 = abc + x1_term * cos((phi - M_PI) / 3.0);
  lam3 = abc + x1_term * cos((phi + M_PI) / 3.0);
}

// The three compare-and-swap steps of corner.py:607-629. With abs_sort the
// magnitudes are read once before any swap and stay attached to their
// original slots, exactly as in cuCIM.
template <class F>
__device__ __forceinline__ void sort3(F& l1, F& l2, F& l3, int descending, int abs_sort) {
  F* v1 = descending ? &l3 : &l1;
  F* v2 = &l2;
  F* v3 = descending ? &l1 : &l3;
  F k1, k2, k3;
  if (abs_sort) {
    const F a1 = abs(l1), a2 = abs(l2), a3 = abs(l3);
    k1 = descending ? a3 : a1;
    k2 = a2;
    k3 = descending ? a1 : a3;
    F s;
    if (k1 > k2) { s = *v2; *v2 = *v1; *v1 = s; }
    if (k1 > k3) { s = *v3; *v3 = *v1; *v1 = s; }
    if (k2 > k3) { s = *v3; *v3 = *v2; *v2 = s; }
  } else {
    F s;
    if (*v1 > *v2) { s = *v2; *v2 = *v1; *v1 = s; }
    if (*v1 > *v3) { s = *v3; *v3 = *v1; *v1 = s; }
    if (*v2 > *v3) { s = *v3; *v3 = *v2; *v2 = s; }
  }
}

template <class F>
__global__ void k_eig33(const F* __restrict__ a_, const F* __restrict__ d_,
                        const F* __restrict__ f_, const F* __restrict__ b_,
                        const F* __restrict__ e_, const F* __restrict__ c_, F* o1, F* o2, F* o3,
                        int64_t n, int descending, int abs_sort) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    F l1, l2, l3;
    eig33<F>(a_[i], b_[i], c_[i], d_[i], e_[i], f_[i], l1, l2, l3);
    sort3(l1, l2, l3, descending, abs_sort);
    o1[i] = l1;
    o2[i] = l2;
    o3[i] = l3;
  }
}

// color/colorconv.py:1038-1046 (+ util/dtype.py:360-361 for uint8 input).
template <class X>
__global__ void k_rgb2gray(const void* rgb, int trgb, X* gray, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    X r, g, b;
    if (trgb == DT_U8) {
      const uint8_t* p = static_cast<const uint8_t*>(rgb);
      const float s = static_cast<float>(1.0 / 255.0);
      r = __fmul_rn(static_cast<float>(p[3 * i]), s);
      g = __fmul_rn(static_cast<float>(p[3 * i + 1]), s);
      b = __fmul_rn(static_cast<float>(p[3 * i + 2]), s);
    } else {
      const X* p = static_cast<const X*>(rgb);
      r = p[3 * i];
      g = p[3 * i + 1];
      b = p[3 * i + 2];
    }
    gray[i] = 0.2125 * r + 0.7154 * g + 0.0721 * b;
  }
}

// util/dtype.py:219-372 restricted to what the path needs:
//   op 0: plain astype (C conversion);
//   op 1: img_as_float — unsigned: x * fl(1/imax) in the computation type C
//         (float32 for <=16-bit input and float32 output, else float64);
//         signed: the same, then max(., -1); floats are converted as by astype;
//   op 2: astype followed by negation (frangi's black_ridges=False, ridges.py:411-413).
template <class C, class D>
__global__ void k_convert(const void* in, int tin, D* out, int64_t n, int op, C scale,
                          int is_signed_int) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    C v = load_as<C>(in, i, tin);
    if (op == 1 && scale != C(0)) {
      v = v * scale;
      if (is_signed_int) v = v < C(-1) ? C(-1) : v;
    }
    D d = static_cast<D>(v);
    if (op == 2) d = -d;
    out[i] = d;
  }
}

// numpy/cupy gradient along one axis with unit spacing and edge_order=1:
// interior (f[i+1] - f[i-1]) / 2, ends f[1] - f[0] and f[n-1] - f[n-2].
template <class F>
__global__ void k_gradient(const F* __restrict__ f, F* __restrict__ g, int64_t outer, int64_t L,
                           int64_t inner) {
  const int64_t n = outer * L * inner;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t l = (e / inner) % L;
    F v;
    if (l == 0) v = f[e + inner] - f[e];
    else if (l == L - 1) v = f[e] - f[e - inner];
    else v = (f[e + inner] - f[e - inner]) / F(2.0);
    g[e] = v;
  }
}

// frangi epilogue for one scale (filters/ridges.py:228-319, :436-475):
// r_g = sum of squared eigenvalues in F, gamma from the first scale's
// max(r_g), the vesselness formula with float64 exponentials, and the
// running maximum over scales.
//
// cuCIM's sum kernels are `r_g = l1 * l1; r_g += l2 * l2; [r_g += l3 * l3;]`
// compiled with contraction on: the CUDA compiler fuses the first product
// into the first addition, fma(l1, l1, l2 * l2) (on 1 M GPU results of the
// compiled 2-D statements, that form matched all and the other two
// associations did not), and the third product into the second addition. Written out with explicit
// fused multiply-adds so that no loop or inlining decision can change it.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

template <class F>
__device__ __forceinline__ F frangi_rg(const F* const* ev, int nd, int64_t i) {
  const F l1 = ev[0][i], l2 = ev[1][i];
  F r = fma(l1, l1, mul_rn(l2, l2));
  if (nd == 3) {
    const F l3 = ev[2][i];
    r = fma(l3, l3, r);
  }
  return r;
}

template <class F>
__global__ void k_frangi_max_rg(const F* __restrict__ l0, const F* __restrict__ l1,
                                const F* __restrict__ l2, int nd, int64_t n,
                                unsigned long long* maxbits) {
  const F* ev[3] = {l0, l1, l2};
  F m = F(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const F r = frangi_rg<F>(ev, nd, i);
    if (r > m) m = r;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const F other = __shfl_xor_sync(0xffffffffu, m, o);
    m = other > m ? other : m;
  }
  if ((threadIdx.x & 31) == 0 && m > F(0)) {
    const double md = static_cast<double>(m);
    atomicMax(maxbits, static_cast<unsigned long long>(__double_as_longlong(md)));
  }
}

// gamma^2 of the automatic gamma: half the square root of the first scale's
// largest r_g (ridges.py:447-453), or the fixed value
__device__ __forceinline__ double frangi_gamma_sq(double gamma_sq_fixed,
                                                  const unsigned long long* maxbits) {
  if (!maxbits) return gamma_sq_fixed;
  const double s_max = __longlong_as_double(static_cast<long long>(*maxbits));
  const double gamma = sqrt(s_max) / 2.0;
  return (s_max == 0) ? 2.0 : max(2 * gamma * gamma, 1e-10);
}

// The vesselness of one voxel from its eigenvalues (ascending by magnitude)
// and r_g: cuCIM's 2-D and 3-D inner kernels, statement by statement.
template <class F>
__device__ __forceinline__ F frangi_value(F lambda1, F lambda2, F lambda3, int nd, F r_g,
                                          double alpha_sq, double beta_sq, double gamma_sq) {
  F result;
  if (nd == 2) {
    F r_b;
    r_b = abs(lambda1) / max(lambda2, static_cast<F>(1.0e-10));
    r_b *= r_b;
    result = exp(-r_b / beta_sq);
    result *= 1.0 - exp(-r_g / gamma_sq);
  } else {
    F r_a, r_b;
    F lam2 = max(lambda2, static_cast<F>(1.0e-10));
    F lam3 = max(lambda3, static_cast<F>(1.0e-10));
    r_a = lam2 / lam3;
    r_a *= r_a;
    r_b = (lambda1 * lambda1) / (lam2 * lam3);
    result = 1.0 - exp(-r_a / alpha_sq);
    result *= exp(-r_b / beta_sq);
    result *= 1.0 - exp(-r_g / gamma_sq);
  }
  return result;
}

// cupy.maximum: NaN in either operand propagates
template <class F>
__device__ __forceinline__ F frangi_fold(F prev, F result) {
  return (prev != prev) ? prev : ((result != result) ? result : (prev > result ? prev : result));
}

template <class F>
__global__ void k_frangi_inner(const F* __restrict__ l0, const F* __restrict__ l1,
                               const F* __restrict__ l2, int nd, int64_t n, double alpha_sq,
                               double beta_sq, double gamma_sq_fixed,
                               const unsigned long long* maxbits, F* out, int first) {
  const double gamma_sq = frangi_gamma_sq(gamma_sq_fixed, maxbits);
  const F* ev[3] = {l0, l1, l2};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const F r_g = frangi_rg<F>(ev, nd, i);
    const F result = frangi_value<F>(l0[i], l1[i], nd == 3 ? l2[i] : F(0), nd, r_g, alpha_sq,
                                     beta_sq, gamma_sq);
    out[i] = first ? result : frangi_fold(out[i], result);
  }
}

// Eigenvalues (ascending by magnitude) and the vesselness in one pass over
// the Hessian elements (00, 01, 11) or (00, 01, 02, 11, 12, 22): the
// eigenvalue images are never stored. The same statements as k_eig22 /
// eig33 + sort3 and k_frangi_inner.
template <class F>
__global__ void k_frangi_fused(const F* __restrict__ h0, const F* __restrict__ h1,
                               const F* __restrict__ h2, const F* __restrict__ h3,
                               const F* __restrict__ h4, const F* __restrict__ h5, int nd,
                               int64_t n, double alpha_sq, double beta_sq,
                               double gamma_sq_fixed, const unsigned long long* maxbits, F* out,
                               int first) {
  const double gamma_sq = frangi_gamma_sq(gamma_sq_fixed, maxbits);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    F lam1, lam2, lam3 = F(0);
    if (nd == 2) {
      // k_eig22's statements with each operation rounded on its own (the
      // form the compiled k_eig22 was measured to take)
      F tmp1, tmp2;
      double m00 = static_cast<double>(h0[i]);
      double m01 = static_cast<double>(h1[i]);
      double m11 = static_cast<double>(h2[i]);
      tmp1 = m01 * m01;
      tmp1 *= 4;
      tmp2 = m00 - m11;
      tmp2 = mul_rn(tmp2, tmp2);
      tmp2 = add_rn(tmp2, tmp1);
      tmp2 = sqrt(tmp2);
      tmp2 /= 2;
      tmp1 = m00 + m11;
      tmp1 /= 2;
      lam1 = tmp1 - tmp2;
      lam2 = tmp1 + tmp2;
      if (abs(lam1) > abs(lam2)) {
        F s = lam1; lam1 = lam2; lam2 = s;
      }
    } else {
      // elements (00, 01, 02, 11, 12, 22) = (a, d, f, b, e, c)
      eig33<F>(h0[i], h3[i], h5[i], h1[i], h4[i], h2[i], lam1, lam2, lam3);
      sort3(lam1, lam2, lam3, 0, 1);
    }
    F r_g = fma(lam1, lam1, mul_rn(lam2, lam2));
    if (nd == 3) r_g = fma(lam3, lam3, r_g);
    const F result = frangi_value<F>(lam1, lam2, lam3, nd, r_g, alpha_sq, beta_sq, gamma_sq);
    out[i] = first ? result : frangi_fold(out[i], result);
  }
}

int64_t numel(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

bool same_shape(const CimxArray* a, const CimxArray* b) {
  if (a->ndim != b->ndim) return false;
  for (int d = 0; d < a->ndim; ++d)
    if (a->shape[d] != b->shape[d]) return false;
  return true;
}

bool contiguous(const CimxArray* a) {
  if (numel(a) == 0) return true;
  int64_t expect = dtype_size(a->dtype);
  for (int d = a->ndim - 1; d >= 0; --d) {
    if (a->shape[d] != 1 && a->strides[d] != expect) return false;
    expect *= a->shape[d];
  }
  return true;
}

}  // namespace

int launch_copy_cast(const void* in, int tin, void* out, int tout, int64_t n, cudaStream_t st) {
  if (n == 0) return CIMX_OK;
  if (tin == tout)
    return cuda_fail(cudaMemcpyAsync(out, in, (size_t)n * dtype_size(tin),
                                     cudaMemcpyDeviceToDevice, st),
                     "copy");
  k_copy_cast<<<grid_for(n), 256, 0, st>>>(in, tin, out, tout, n);
  return cuda_fail(cudaGetLastError(), "copy_cast launch");
}

int launch_square_accumulate(void* acc, const void* term, int dt, int64_t n, bool first,
                             cudaStream_t st) {
  if (dt == DT_F32)
    k_square_acc<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(acc),
                                                      static_cast<const float*>(term), n, first);
  else
    k_square_acc<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(acc),
                                                       static_cast<const double*>(term), n, first);
  return cuda_fail(cudaGetLastError(), "square_accumulate launch");
}

int launch_sqrt_inplace(void* acc, int dt, int64_t n, cudaStream_t st) {
  if (dt == DT_F32)
    k_sqrt<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(acc), n);
  else
    k_sqrt<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(acc), n);
  return cuda_fail(cudaGetLastError(), "sqrt launch");
}

}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_gradient_magnitude(const CimxArray* in, const CimxArray* out, const CimxPass* passes,
                            int naxes, int passes_per_axis, void* stream) {
  if (!in || !out || !passes || naxes < 1 || passes_per_axis < 0)
    return fail(CIMX_E_INVALID, "bad gradient-magnitude arguments");
  if (out->dtype != DT_F32 && out->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "gradient magnitude output must be float32 or float64");
  if (!same_shape(in, out)) return fail(CIMX_E_INVALID, "output shape not correct");
  if (!contiguous(out)) return fail(CIMX_E_LAYOUT, "output is not C-contiguous");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = numel(out);
  if (n == 0) return CIMX_OK;
  const size_t bytes = (size_t)n * dtype_size(out->dtype);
  void* tmp = nullptr;
  if (naxes > 1) {
    tmp = scratch_alloc(bytes, st);
    if (!tmp) return fail(CIMX_E_NOMEM, "scratch allocation for gradient magnitude failed");
  }
  CimxArray t = *out;
  t.data = tmp;
  int rc = CIMX_OK;
  for (int a = 0; a < naxes && rc == CIMX_OK; ++a) {
    const CimxArray* dst = a == 0 ? out : &t;
    rc = cimx_separable(in, dst, passes + (size_t)a * passes_per_axis, passes_per_axis, 0, stream);
    if (rc == CIMX_OK)
      rc = launch_square_accumulate(out->data, dst->data, out->dtype, n, a == 0, st);
  }
  if (rc == CIMX_OK) rc = launch_sqrt_inplace(out->data, out->dtype, n, st);
  scratch_free(tmp, bytes, st);
  return rc;
}

int cimx_square_accumulate(const CimxArray* acc, const CimxArray* term, int first,
                           void* stream) {
  if (!acc || !term) return fail(CIMX_E_INVALID, "bad square-accumulate arguments");
  if (acc->dtype != DT_F32 && acc->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "square-accumulate: float32 or float64");
  if (term->dtype != acc->dtype) return fail(CIMX_E_DTYPE, "square-accumulate: dtypes differ");
  if (!same_shape(acc, term)) return fail(CIMX_E_INVALID, "square-accumulate: shapes differ");
  if (!contiguous(acc) || !contiguous(term))
    return fail(CIMX_E_LAYOUT, "square-accumulate: arrays must be C-contiguous");
  const int64_t n = numel(acc);
  if (n == 0) return CIMX_OK;
  return launch_square_accumulate(acc->data, term->data, acc->dtype, n, first != 0,
                                  static_cast<cudaStream_t>(stream));
}

int cimx_sqrt(const CimxArray* a, void* stream) {
  if (!a) return fail(CIMX_E_INVALID, "bad sqrt arguments");
  if (a->dtype != DT_F32 && a->dtype != DT_F64) return fail(CIMX_E_DTYPE, "sqrt: float32 or float64");
  if (!contiguous(a)) return fail(CIMX_E_LAYOUT, "sqrt: array must be C-contiguous");
  const int64_t n = numel(a);
  if (n == 0) return CIMX_OK;
  return launch_sqrt_inplace(a->data, a->dtype, n, static_cast<cudaStream_t>(stream));
}

int cimx_combine(const CimxArray* acc, const CimxArray* term, int op, void* stream) {
  if (!acc || !term || (op != CIMX_COMBINE_ADD && op != CIMX_COMBINE_SUBTRACT))
    return fail(CIMX_E_INVALID, "bad combine arguments");
  if (acc->dtype != term->dtype) return fail(CIMX_E_DTYPE, "combine: dtypes differ");
  if (!same_shape(acc, term)) return fail(CIMX_E_INVALID, "combine: shapes differ");
  if (!contiguous(acc) || !contiguous(term))
    return fail(CIMX_E_LAYOUT, "combine: arrays must be C-contiguous");
  const int64_t n = numel(acc);
  if (n == 0) return CIMX_OK;
  return launch_combine(acc->data, term->data, acc->dtype, n, op == CIMX_COMBINE_SUBTRACT,
                        static_cast<cudaStream_t>(stream));
}

int cimx_unsharp(const CimxArray* image, const CimxArray* blurred, const CimxArray* out,
                 double amount, int clip, double lo, double hi, void* stream) {
  if (!image || !blurred || !out) return fail(CIMX_E_INVALID, "bad unsharp arguments");
  const int dt = image->dtype;
  if (dt != DT_F32 && dt != DT_F64) return fail(CIMX_E_DTYPE, "unsharp: float32 or float64");
  if (blurred->dtype != dt || out->dtype != dt) return fail(CIMX_E_DTYPE, "unsharp: dtypes differ");
  if (!same_shape(image, blurred) || !same_shape(image, out))
    return fail(CIMX_E_INVALID, "unsharp: shapes differ");
  if (!contiguous(image) || !contiguous(blurred) || !contiguous(out))
    return fail(CIMX_E_LAYOUT, "unsharp: arrays must be C-contiguous");
  const int64_t n = numel(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dt == DT_F32)
    k_unsharp<float><<<grid_for(n), 256, 0, st>>>(
        static_cast<const float*>(image->data), static_cast<const float*>(blurred->data),
        static_cast<float*>(out->data), n, static_cast<float>(amount), clip,
        static_cast<float>(lo), static_cast<float>(hi));
  else
    k_unsharp<double><<<grid_for(n), 256, 0, st>>>(
        static_cast<const double*>(image->data), static_cast<const double*>(blurred->data),
        static_cast<double*>(out->data), n, amount, clip, lo, hi);
  return cuda_fail(cudaGetLastError(), "unsharp launch");
}

int cimx_any_negative(const CimxArray* a, int* result, void* stream) {
  if (!a || !result) return fail(CIMX_E_INVALID, "bad any_negative arguments");
  if (a->dtype != DT_F32 && a->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "any_negative: float32 or float64");
  if (!contiguous(a)) return fail(CIMX_E_LAYOUT, "any_negative: array must be C-contiguous");
  *result = 0;
  const int64_t n = numel(a);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* flag = static_cast<int*>(scratch_alloc(sizeof(int), st));
  if (!flag) return fail(CIMX_E_NOMEM, "scratch allocation for any_negative failed");
  int rc = cuda_fail(cudaMemsetAsync(flag, 0, sizeof(int), st), "any_negative memset");
  if (rc == CIMX_OK) {
    if (a->dtype == DT_F32)
      k_any_negative<float><<<grid_for(n), 256, 0, st>>>(static_cast<const float*>(a->data), n, flag);
    else
      k_any_negative<double><<<grid_for(n), 256, 0, st>>>(static_cast<const double*>(a->data), n, flag);
    rc = cuda_fail(cudaGetLastError(), "any_negative launch");
  }
  if (rc == CIMX_OK)
    rc = cuda_fail(cudaMemcpyAsync(result, flag, sizeof(int), cudaMemcpyDeviceToHost, st),
                   "any_negative readback");
  if (rc == CIMX_OK) rc = cuda_fail(cudaStreamSynchronize(st), "any_negative synchronize");
  scratch_free(flag, sizeof(int), st);
  return rc;
}

int cimx_laplace(const CimxArray* in, const CimxArray* out, const CimxPass* passes, int naxes,
                 int passes_per_axis, void* stream) {
  if (!in || !out || !passes || naxes < 1 || passes_per_axis < 0)
    return fail(CIMX_E_INVALID, "bad laplace arguments");
  if (!same_shape(in, out)) return fail(CIMX_E_INVALID, "output shape not correct");
  if (!contiguous(out)) return fail(CIMX_E_LAYOUT, "output is not C-contiguous");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = numel(out);
  if (n == 0) return CIMX_OK;
  const size_t bytes = (size_t)n * dtype_size(out->dtype);
  void* tmp = nullptr;
  if (naxes > 1) {
    tmp = scratch_alloc(bytes, st);
    if (!tmp) return fail(CIMX_E_NOMEM, "scratch allocation for laplace failed");
  }
  CimxArray t = *out;
  t.data = tmp;
  int rc = cimx_separable(in, out, passes, passes_per_axis, 0, stream);
  for (int a = 1; a < naxes && rc == CIMX_OK; ++a) {
    rc = cimx_separable(in, &t, passes + (size_t)a * passes_per_axis, passes_per_axis, 0, stream);
    if (rc == CIMX_OK) rc = launch_combine(out->data, tmp, out->dtype, n, 0, st);
  }
  scratch_free(tmp, bytes, st);
  return rc;
}

int cimx_eigvals_sym(const CimxArray* elems, int nelems, const CimxArray* out, int sort,
                     int abs_sort, void* stream) {
  if (!elems || !out || (nelems != 3 && nelems != 6))
    return fail(CIMX_E_INVALID, "eigvals: expected 3 or 6 element images");
  const int nout = nelems == 3 ? 2 : 3;
  const int dt = elems[0].dtype;
  if (dt != DT_F32 && dt != DT_F64)
    return fail(CIMX_E_DTYPE, "expected real-valued floating point matrices");
  for (int i = 0; i < nelems; ++i)
    if (elems[i].dtype != dt || !same_shape(&elems[0], &elems[i]) || !contiguous(&elems[i]))
      return fail(CIMX_E_INVALID, "eigvals: element images must share dtype, shape, layout");
  for (int i = 0; i < nout; ++i)
    if (out[i].dtype != dt || !same_shape(&elems[0], &out[i]) || !contiguous(&out[i]))
      return fail(CIMX_E_INVALID, "eigvals: outputs must match the element images");
  const int64_t n = numel(&elems[0]);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int desc = sort != 0;
  if (dt == DT_F32) {
    auto E = [&](int i) { return static_cast<const float*>(elems[i].data); };
    auto O = [&](int i) { return static_cast<float*>(out[i].data); };
    if (nelems == 3)
      k_eig22<float><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), O(0), O(1), n, desc, abs_sort);
    else  // elems = (00,01,02,11,12,22) = (a,d,f,b,e,c)
      k_eig33<float><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), E(3), E(4), E(5), O(0), O(1),
                                                  O(2), n, desc, abs_sort);
  } else {
    auto E = [&](int i) { return static_cast<const double*>(elems[i].data); };
    auto O = [&](int i) { return static_cast<double*>(out[i].data); };
    if (nelems == 3)
      k_eig22<double><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), O(0), O(1), n, desc, abs_sort);
    else
      k_eig33<double><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), E(3), E(4), E(5), O(0), O(1),
                                                   O(2), n, desc, abs_sort);
  }
  return cuda_fail(cudaGetLastError(), "eigvals launch");
}

int cimx_rgb2gray(const CimxArray* rgb, const CimxArray* gray, void* stream) {
  if (!rgb || !gray) return fail(CIMX_E_INVALID, "rgb2gray: NULL argument");
  if (rgb->ndim < 1 || rgb->shape[rgb->ndim - 1] != 3 || gray->ndim != rgb->ndim - 1)
    return fail(CIMX_E_INVALID, "the input array must have size 3 along `channel_axis`");
  for (int d = 0; d < gray->ndim; ++d)
    if (gray->shape[d] != rgb->shape[d]) return fail(CIMX_E_INVALID, "output shape not correct");
  if (!contiguous(rgb) || !contiguous(gray)) return fail(CIMX_E_LAYOUT, "not C-contiguous");
  const int64_t n = numel(gray);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) return CIMX_OK;
  if (gray->dtype == DT_F32 && (rgb->dtype == DT_F32 || rgb->dtype == DT_U8))
    k_rgb2gray<float><<<grid_for(n), 256, 0, st>>>(rgb->data, rgb->dtype,
                                                   static_cast<float*>(gray->data), n);
  else if (gray->dtype == DT_F64 && rgb->dtype == DT_F64)
    k_rgb2gray<double><<<grid_for(n), 256, 0, st>>>(rgb->data, rgb->dtype,
                                                    static_cast<double*>(gray->data), n);
  else
    return fail(CIMX_E_DTYPE, "rgb2gray: unsupported dtype pair");
  return cuda_fail(cudaGetLastError(), "rgb2gray launch");
}

int cimx_convert(const CimxArray* in, const CimxArray* out, int op, void* stream) {
  if (!in || !out || op < 0 || op > 2) return fail(CIMX_E_INVALID, "convert: bad arguments");
  if (!same_shape(in, out)) return fail(CIMX_E_INVALID, "output shape not correct");
  if (!contiguous(in) || !contiguous(out)) return fail(CIMX_E_LAYOUT, "not C-contiguous");
  if (dtype_size(in->dtype) == 0) return fail(CIMX_E_DTYPE, "convert: unsupported input dtype");
  if (out->dtype != DT_F32 && out->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "convert: output must be float32 or float64");
  const int64_t n = numel(in);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int t = in->dtype;
  const bool is_int = !(t == DT_F16 || t == DT_F32 || t == DT_F64);
  const bool is_signed = t == DT_I8 || t == DT_I16 || t == DT_I32 || t == DT_I64 || t == DT_I64Q;
  double imax = 0;
  switch (t) {
    case DT_U8: imax = 255.0; break;
    case DT_I8: imax = 127.0; break;
    case DT_U16: imax = 65535.0; break;
    case DT_I16: imax = 32767.0; break;
    case DT_U32: imax = 4294967295.0; break;
    case DT_I32: imax = 2147483647.0; break;
    case DT_U64: case DT_U64Q: imax = 18446744073709551615.0; break;
    case DT_I64: case DT_I64Q: imax = 9223372036854775807.0; break;
    default: break;
  }
  const bool scale = op == 1 && is_int;
  // float32 computation only for <= 16-bit integers converted to float32
  const bool c32 = out->dtype == DT_F32 && (!scale || dtype_size(t) <= 2);
  if (c32) {
    const float s = scale ? static_cast<float>(1.0 / imax) : 0.0f;
    k_convert<float, float><<<grid_for(n), 256, 0, st>>>(in->data, t,
        static_cast<float*>(out->data), n, scale ? 1 : (op == 2 ? 2 : 0), s, is_signed);
  } else if (out->dtype == DT_F32) {
    k_convert<double, float><<<grid_for(n), 256, 0, st>>>(in->data, t,
        static_cast<float*>(out->data), n, scale ? 1 : (op == 2 ? 2 : 0), 1.0 / imax, is_signed);
  } else {
    const double s = scale ? 1.0 / imax : 0.0;
    k_convert<double, double><<<grid_for(n), 256, 0, st>>>(in->data, t,
        static_cast<double*>(out->data), n, scale ? 1 : (op == 2 ? 2 : 0), s, is_signed);
  }
  return cuda_fail(cudaGetLastError(), "convert launch");
}

int cimx_gradient_fd(const CimxArray* in, const CimxArray* out, int axis, void* stream) {
  if (!in || !out) return fail(CIMX_E_INVALID, "gradient: NULL argument");
  if (!same_shape(in, out) || in->dtype != out->dtype)
    return fail(CIMX_E_INVALID, "gradient: output must match the input");
  if (in->dtype != DT_F32 && in->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "gradient: float32/float64 only");
  if (!contiguous(in) || !contiguous(out)) return fail(CIMX_E_LAYOUT, "not C-contiguous");
  if (axis < 0) axis += in->ndim;
  if (axis < 0 || axis >= in->ndim) return fail(CIMX_E_INVALID, "axis out of range");
  if (in->shape[axis] < 2)
    return fail(CIMX_E_INVALID,
                "Shape of array too small to calculate a numerical gradient, at least "
                "(edge_order + 1) elements are required.");
  int64_t outer = 1, inner = 1;
  for (int d = 0; d < axis; ++d) outer *= in->shape[d];
  for (int d = axis + 1; d < in->ndim; ++d) inner *= in->shape[d];
  const int64_t n = numel(in);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->dtype == DT_F32)
    k_gradient<float><<<grid_for(n), 256, 0, st>>>(static_cast<const float*>(in->data),
        static_cast<float*>(out->data), outer, in->shape[axis], inner);
  else
    k_gradient<double><<<grid_for(n), 256, 0, st>>>(static_cast<const double*>(in->data),
        static_cast<double*>(out->data), outer, in->shape[axis], inner);
  return cuda_fail(cudaGetLastError(), "gradient launch");
}

int cimx_frangi_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out, double alpha,
                           double beta, double gamma, int first, void* gamma_state,
                           void* stream) {
  if (!eigs || !out || (ndim != 2 && ndim != 3))
    return fail(CIMX_E_INVALID, "frangi: expected 2 or 3 eigenvalue images");
  const int dt = out->dtype;
  if (dt != DT_F32 && dt != DT_F64) return fail(CIMX_E_DTYPE, "frangi: float32/float64 only");
  for (int k = 0; k < ndim; ++k)
    if (eigs[k].dtype != dt || !same_shape(&eigs[k], out) || !contiguous(&eigs[k]))
      return fail(CIMX_E_INVALID, "frangi: eigenvalue images must match the output");
  if (!contiguous(out)) return fail(CIMX_E_LAYOUT, "not C-contiguous");
  const int64_t n = numel(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double alpha_sq = 2 * alpha * alpha, beta_sq = 2 * beta * beta;
  const bool auto_gamma = gamma != gamma;  // NaN: half the max Hessian norm of the first scale
  unsigned long long* maxbits = static_cast<unsigned long long*>(gamma_state);
  if (auto_gamma && !maxbits) return fail(CIMX_E_INVALID, "frangi: auto gamma needs a state word");
  const double gamma_sq = auto_gamma ? 0.0 : 2 * gamma * gamma;
  const void* e2 = ndim == 3 ? eigs[2].data : eigs[1].data;
  if (dt == DT_F32) {
    auto E = [&](int k) { return static_cast<const float*>(k == 2 ? e2 : eigs[k].data); };
    if (auto_gamma && first) {
      cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), st);
      if (e != cudaSuccess) return cuda_fail(e, "frangi state reset");
      k_frangi_max_rg<float><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), ndim, n, maxbits);
    }
    k_frangi_inner<float><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), ndim, n, alpha_sq,
        beta_sq, gamma_sq, auto_gamma ? maxbits : nullptr, static_cast<float*>(out->data), first);
  } else {
    auto E = [&](int k) { return static_cast<const double*>(k == 2 ? e2 : eigs[k].data); };
    if (auto_gamma && first) {
      cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), st);
      if (e != cudaSuccess) return cuda_fail(e, "frangi state reset");
      k_frangi_max_rg<double><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), ndim, n, maxbits);
    }
    k_frangi_inner<double><<<grid_for(n), 256, 0, st>>>(E(0), E(1), E(2), ndim, n, alpha_sq,
        beta_sq, gamma_sq, auto_gamma ? maxbits : nullptr, static_cast<double*>(out->data),
        first);
  }
  return cuda_fail(cudaGetLastError(), "frangi launch");
}

}  // extern "C"

extern "C" int cimx_frangi_hessian_accumulate(const CimxArray* H, int nelems,
                                              const CimxArray* out, double alpha, double beta,
                                              double gamma, int first, void* gamma_state,
                                              void* stream) {
  using namespace cimx;
  if (!H || !out || (nelems != 3 && nelems != 6))
    return fail(CIMX_E_INVALID, "frangi: expected 3 or 6 Hessian element images");
  const int nd = nelems == 3 ? 2 : 3;
  const int dt = out->dtype;
  if (dt != DT_F32 && dt != DT_F64) return fail(CIMX_E_DTYPE, "frangi: float32/float64 only");
  for (int k = 0; k < nelems; ++k)
    if (H[k].dtype != dt || !same_shape(&H[k], out) || !contiguous(&H[k]))
      return fail(CIMX_E_INVALID, "frangi: Hessian images must match the output");
  if (!contiguous(out)) return fail(CIMX_E_LAYOUT, "not C-contiguous");
  const int64_t n = numel(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool auto_gamma = gamma != gamma;
  auto* maxbits = static_cast<unsigned long long*>(gamma_state);
  if (auto_gamma && !maxbits) return fail(CIMX_E_INVALID, "frangi: auto gamma needs a state word");
  if ((auto_gamma && first) || dt == DT_F64) {
    // the first scale's gamma needs the image-wide max of r_g before any
    // vesselness: eigenvalue images, the max, then the vesselness. float64
    // takes this path on every scale: its eigenvalues are not rounded to
    // float, so the last bit of the float64 solve would show how the
    // compiler contracted it inside the fused kernel, where the standalone
    // eigenvalue kernel is compiled like cuCIM's own
    const size_t bytes = (size_t)n * dtype_size(dt);
    void* buf = scratch_alloc(bytes * nd, st);
    if (!buf) return fail(CIMX_E_NOMEM, "scratch allocation for the eigenvalues failed");
    CimxArray ev[3];
    for (int k = 0; k < nd; ++k) {
      ev[k] = *out;
      ev[k].data = static_cast<char*>(buf) + k * bytes;
    }
    int rc = cimx_eigvals_sym(H, nelems, ev, 0, 1, stream);
    if (!rc) rc = cimx_frangi_accumulate(ev, nd, out, alpha, beta, gamma, first, gamma_state,
                                         stream);
    scratch_free(buf, bytes * nd, st);
    return rc;
  }
  const double alpha_sq = 2 * alpha * alpha, beta_sq = 2 * beta * beta;
  const double gamma_sq = auto_gamma ? 0.0 : 2 * gamma * gamma;
  const unsigned long long* mb = auto_gamma ? maxbits : nullptr;
  auto E = [&](int k) { return H[k < nelems ? k : 0].data; };
  if (dt == DT_F32) {
    auto P = [&](int k) { return static_cast<const float*>(E(k)); };
    k_frangi_fused<float><<<grid_for(n), 256, 0, st>>>(P(0), P(1), P(2), P(3), P(4), P(5), nd, n,
                                                       alpha_sq, beta_sq, gamma_sq, mb,
                                                       static_cast<float*>(out->data), first);
  } else {
    auto P = [&](int k) { return static_cast<const double*>(E(k)); };
    k_frangi_fused<double><<<grid_for(n), 256, 0, st>>>(P(0), P(1), P(2), P(3), P(4), P(5), nd,
                                                        n, alpha_sq, beta_sq, gamma_sq, mb,
                                                        static_cast<double*>(out->data), first);
  }
  return cuda_fail(cudaGetLastError(), "frangi launch");
}
