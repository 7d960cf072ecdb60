// cimx_corner.cu — the elementwise parts of structure_tensor and the corner
// measures of python/cucim/src/cucim/skimage/feature/corner.py: the
// products of derivative images (:146-156) and the response kernels of
// corner_kitchen_rosenfeld (:940-1004), corner_harris (:1007-1113),
// corner_shi_tomasi (:1116-1189) and corner_foerstner (:1192-1284).
//
// Each kernel body evaluates cuCIM's expression statement by statement in
// the same types (F and, for Harris' parameter, double), so the CUDA
// compiler contracts it the way NVRTC contracts cuCIM's kernels.
#include <algorithm>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

inline unsigned grid_for(int64_t n, int threads = 256) {
  const int64_t b = (n + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

#define CIMX_GRID_LOOP(i, n)                                                \
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); \
       i += (int64_t)gridDim.x * blockDim.x)

template <class F>
__global__ void k_multiply(const F* __restrict__ a, const F* __restrict__ b, F* __restrict__ out,
                           int64_t n) {
  CIMX_GRID_LOOP(i, n) out[i] = a[i] * b[i];
}

template <class F>
__global__ void k_kitchen_rosenfeld(const F* imx, const F* imy, const F* imxx, const F* imxy,
                                    const F* imyy, F* response, int64_t n) {
  CIMX_GRID_LOOP(i, n) {
    F numerator, denominator, imx_sq, imy_sq;
    imx_sq = imx[i] * imx[i];
    imy_sq = imy[i] * imy[i];
    denominator = imx_sq;
    denominator += imy_sq;
    if (denominator == 0) {
      response[i] = 0.0;
    } else {
      numerator = imxx[i] * imy_sq + imyy[i] * imx_sq - 2 * imxy[i] * imx[i] * imy[i];
      response[i] = numerator / denominator;
    }
  }
}

template <class F>
__global__ void k_harris_k(const F* Arr, const F* Acc, const F* Arc, double k, F* response,
                           int64_t n) {
  CIMX_GRID_LOOP(i, n) {
    F detA, traceA;
    detA = Arr[i] * Acc[i] - Arc[i] * Arc[i];
    traceA = Arr[i] + Acc[i];
    response[i] = detA - k * traceA * traceA;
  }
}

template <class F>
__global__ void k_harris_eps(const F* Arr, const F* Acc, const F* Arc, double eps, F* response,
                             int64_t n) {
  CIMX_GRID_LOOP(i, n) {
    F detA, traceA;
    detA = Arr[i] * Acc[i] - Arc[i] * Arc[i];
    traceA = Arr[i] + Acc[i];
    response[i] = 2 * detA / (traceA + eps);
  }
}

template <class F>
__global__ void k_shi_tomasi(const F* Arr, const F* Acc, const F* Arc, F* response, int64_t n) {
  CIMX_GRID_LOOP(i, n) {
    F tmp;
    tmp = (Arr[i] - Acc[i]);
    tmp *= tmp;
    response[i] = (Arr[i] + Acc[i] - sqrt(tmp + 4 * Arc[i] * Arc[i])) / 2.0;
  }
}

template <class F>
__global__ void k_foerstner(const F* Arr, const F* Acc, const F* Arc, F* w, F* q, int64_t n) {
  CIMX_GRID_LOOP(i, n) {
    F detA, traceA;
    detA = Arr[i] * Acc[i] - Arc[i] * Arc[i];
    traceA = Arr[i] + Acc[i];
    if (traceA == 0) {
      w[i] = 0;
      q[i] = 0;
    } else {
      w[i] = detA / traceA;
      q[i] = 4 * detA / (traceA * traceA);
    }
  }
}

int64_t count(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

bool dense(const CimxArray* a) {
  int64_t e = dtype_size(a->dtype);
  for (int d = a->ndim - 1; d >= 0; --d) {
    if (a->shape[d] != 1 && a->strides[d] != e) return false;
    e *= a->shape[d];
  }
  return true;
}

// every array float32/float64, C-contiguous, with the dtype and element
// count of `ref`
int check_like(const CimxArray* ref, const CimxArray* a) {
  if (!a || !a->data) return fail(CIMX_E_INVALID, "NULL array");
  if (a->dtype != ref->dtype) return fail(CIMX_E_DTYPE, "arrays must share one float dtype");
  if (a->ndim != ref->ndim) return fail(CIMX_E_INVALID, "arrays must share one shape");
  for (int d = 0; d < a->ndim; ++d)
    if (a->shape[d] != ref->shape[d]) return fail(CIMX_E_INVALID, "arrays must share one shape");
  if (!dense(a)) return fail(CIMX_E_LAYOUT, "arrays must be C-contiguous");
  return CIMX_OK;
}

template <class F>
int launch_corner(int kind, const CimxArray* in, const CimxArray* out, const CimxArray* out2,
                  double param, int64_t n, cudaStream_t st) {
  auto I = [&](int k) { return static_cast<const F*>(in[k].data); };
  F* o = static_cast<F*>(out->data);
  switch (kind) {
    case CIMX_CORNER_KITCHEN_ROSENFELD:
      k_kitchen_rosenfeld<F><<<grid_for(n), 256, 0, st>>>(I(0), I(1), I(2), I(3), I(4), o, n);
      break;
    case CIMX_CORNER_HARRIS_K:
      k_harris_k<F><<<grid_for(n), 256, 0, st>>>(I(0), I(1), I(2), param, o, n);
      break;
    case CIMX_CORNER_HARRIS_EPS:
      k_harris_eps<F><<<grid_for(n), 256, 0, st>>>(I(0), I(1), I(2), param, o, n);
      break;
    case CIMX_CORNER_SHI_TOMASI:
      k_shi_tomasi<F><<<grid_for(n), 256, 0, st>>>(I(0), I(1), I(2), o, n);
      break;
    default:
      k_foerstner<F><<<grid_for(n), 256, 0, st>>>(I(0), I(1), I(2), o,
                                                   static_cast<F*>(out2->data), n);
  }
  return cuda_fail(cudaGetLastError(), "corner launch");
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_multiply(const CimxArray* a, const CimxArray* b, const CimxArray* out, void* stream) {
  if (!a || !b || !out) return fail(CIMX_E_INVALID, "NULL argument");
  if (out->dtype != DT_F32 && out->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "multiply: float32/float64 only");
  int rc;
  if ((rc = check_like(out, a)) || (rc = check_like(out, b)) || (rc = check_like(out, out)))
    return rc;
  const int64_t n = count(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (out->dtype == DT_F32)
    k_multiply<float><<<grid_for(n), 256, 0, st>>>(static_cast<const float*>(a->data),
                                                   static_cast<const float*>(b->data),
                                                   static_cast<float*>(out->data), n);
  else
    k_multiply<double><<<grid_for(n), 256, 0, st>>>(static_cast<const double*>(a->data),
                                                    static_cast<const double*>(b->data),
                                                    static_cast<double*>(out->data), n);
  return cuda_fail(cudaGetLastError(), "multiply launch");
}

int cimx_corner_response(int kind, const CimxArray* inputs, int ninputs, const CimxArray* out,
                         const CimxArray* out2, double param, void* stream) {
  if (!inputs || !out) return fail(CIMX_E_INVALID, "NULL argument");
  if (kind < CIMX_CORNER_KITCHEN_ROSENFELD || kind > CIMX_CORNER_FOERSTNER)
    return fail(CIMX_E_INVALID, "unknown corner measure");
  const int need = kind == CIMX_CORNER_KITCHEN_ROSENFELD ? 5 : 3;
  if (ninputs != need)
    return fail(CIMX_E_INVALID, "expected " + std::to_string(need) + " input images");
  if (out->dtype != DT_F32 && out->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "corner measures: float32/float64 only");
  int rc = check_like(out, out);
  for (int k = 0; k < ninputs && !rc; ++k) rc = check_like(out, &inputs[k]);
  if (!rc && kind == CIMX_CORNER_FOERSTNER) rc = out2 ? check_like(out, out2)
                                                      : fail(CIMX_E_INVALID, "q is NULL");
  if (rc) return rc;
  const int64_t n = count(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return out->dtype == DT_F32 ? launch_corner<float>(kind, inputs, out, out2, param, n, st)
                              : launch_corner<double>(kind, inputs, out, out2, param, n, st);
}

}  // extern "C"
