// cimx_ridges.cu — per-scale epilogues of the meijering, sato and hybrid
// Hessian ridge filters (python/cucim/src/cucim/skimage/filters/ridges.py),
// applied to the eigenvalues of the Gaussian-derivative Hessian.
//
// meijering (ridges.py:50-146): the eigenvalues (descending) below 1e-12 in
// magnitude are zeroed, mixed by the circulant matrix (1 on the diagonal,
// alpha elsewhere), the mixed value of largest magnitude is kept, clipped at
// 0, normalised by its image-wide maximum and folded into the running
// maximum over scales. cuCIM reads that maximum on the host; here a first
// kernel reduces it into device memory and a second one normalises and
// folds, so no host synchronisation is needed.
// sato (ridges.py:148-225): the eigenvalues but the lowest, clipped at 0,
// their geometric mean (powf with exponent 1 / (ndim - 1)) times sigma^2.
// hessian (ridges.py:479-595): frangi with gamma 15, then outputs <= 0 set
// to 1.
#include <cmath>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

inline unsigned grid_for(int64_t n, int threads = 256) {
  const int64_t b = (n + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * 32));
}

// eigvals[abs(eigvals) < 1e-12] = 0 (ridges.py:116, :209); the threshold is
// the Python float compared in the array's type
template <class F>
__device__ __forceinline__ F zero_tiny(F v) {
  return abs(v) < static_cast<F>(1e-12) ? F(0) : v;
}

// cupy.maximum(a, b): NaN in either operand propagates
template <class F>
__device__ __forceinline__ F nan_max(F a, F b) {
  return (a != a) ? a : ((b != b) ? b : (a > b ? a : b));
}

// vals = tensordot(mtx, eigvals, 1) for row r of the circulant matrix, each
// row an ascending-index multiply-add chain (the order the float32 GEMM of
// cupy.tensordot accumulates its ndim products in), then the value of
// largest magnitude (first on ties, NaN first, like argmax), clipped at 0.
template <class F>
__device__ __forceinline__ F meijering_value(const F* const* ev, int nd, F alpha, int64_t i) {
  F e[3];
  for (int k = 0; k < nd; ++k) e[k] = zero_tiny(ev[k][i]);
  F best = F(0), best_abs = F(-1);
  for (int r = 0; r < nd; ++r) {
    F v = (r == 0 ? F(1) : alpha) * e[0];
    for (int k = 1; k < nd; ++k) v = fma(r == k ? F(1) : alpha, e[k], v);
    const F a = abs(v);
    if (r == 0 || (a != a && best_abs == best_abs) || a > best_abs) {
      best = v;
      best_abs = a;
    }
  }
  // cupy.maximum(vals, 0)
  return (best != best) ? best : (best > F(0) ? best : F(0));
}

// state[0]: the maximum's bit pattern as a float64 (values are >= 0, so the
// bit patterns order like the values); state[1]: set when a value is NaN
// (cupy's max is then NaN and cuCIM skips the normalisation)
template <class F>
__global__ void k_meijering_max(const F* __restrict__ l0, const F* __restrict__ l1,
                                const F* __restrict__ l2, int nd, F alpha, int64_t n,
                                unsigned long long* state) {
  const F* ev[3] = {l0, l1, l2};
  F m = F(0);
  bool nan = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const F v = meijering_value<F>(ev, nd, alpha, i);
    if (v != v) nan = true;
    else if (v > m) m = v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const F other = __shfl_xor_sync(0xffffffffu, m, o);
    m = other > m ? other : m;
  }
  nan = __any_sync(0xffffffffu, nan);
  if ((threadIdx.x & 31) == 0) {
    if (m > F(0))
      atomicMax(&state[0], static_cast<unsigned long long>(
                               __double_as_longlong(static_cast<double>(m))));
    if (nan) atomicOr(&state[1], 1ull);
  }
}

template <class F>
__global__ void k_meijering_fold(const F* __restrict__ l0, const F* __restrict__ l1,
                                 const F* __restrict__ l2, int nd, F alpha, int64_t n,
                                 const unsigned long long* state, F* out, int first) {
  const F* ev[3] = {l0, l1, l2};
  const F m = static_cast<F>(__longlong_as_double(static_cast<long long>(state[0])));
  const bool scale = state[1] == 0 && m > F(0);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    F v = meijering_value<F>(ev, nd, alpha, i);
    if (scale) v = v / m;
    out[i] = nan_max(first ? F(0) : out[i], v);
  }
}

template <class F>
__global__ void k_sato(const F* __restrict__ l0, const F* __restrict__ l1, int nd, F s2,
                       int64_t n, F* out, int first) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    // cupy.maximum(eigvals[:-1], 0), their product, ** (1 / (ndim - 1))
    const F a = nan_max(zero_tiny(l0[i]), F(0));
    F v;
    if (nd == 2) {
      v = pow(a, F(1));
    } else {
      const F b = nan_max(zero_tiny(l1[i]), F(0));
      v = pow(a * b, static_cast<F>(0.5));
    }
    v = v * s2;
    out[i] = nan_max(first ? F(0) : out[i], v);
  }
}

template <class F>
__global__ void k_le0_to_one(F* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (out[i] <= F(0)) out[i] = F(1);
}

int64_t count(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

int check_eigs(const CimxArray* eigs, int ndim, const CimxArray* out) {
  if (!eigs || !out || (ndim != 2 && ndim != 3))
    return fail(CIMX_E_INVALID, "expected 2 or 3 eigenvalue images");
  if (out->dtype != DT_F32 && out->dtype != DT_F64)
    return fail(CIMX_E_DTYPE, "float32/float64 only");
  const int64_t n = count(out);
  for (int k = 0; k < ndim; ++k) {
    if (eigs[k].dtype != out->dtype || count(&eigs[k]) != n)
      return fail(CIMX_E_INVALID, "eigenvalue images must match the output");
  }
  return CIMX_OK;
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_meijering_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out,
                              double alpha, int first, void* state, void* stream) {
  int rc = check_eigs(eigs, ndim, out);
  if (rc) return rc;
  if (!state) return fail(CIMX_E_INVALID, "state is NULL");
  const int64_t n = count(out);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the maximum of this scale starts from zero
  cudaError_t e = cudaMemsetAsync(state, 0, 16, st);
  if (e != cudaSuccess) return cuda_fail(e, "meijering state");
  if (n == 0) return CIMX_OK;
  auto* s = static_cast<unsigned long long*>(state);
  auto E = [&](int k) { return eigs[k < ndim ? k : 0].data; };
  if (out->dtype == DT_F32) {
    const float a = static_cast<float>(alpha);
    auto P = [&](int k) { return static_cast<const float*>(E(k)); };
    k_meijering_max<float><<<grid_for(n), 256, 0, st>>>(P(0), P(1), P(2), ndim, a, n, s);
    k_meijering_fold<float><<<grid_for(n), 256, 0, st>>>(P(0), P(1), P(2), ndim, a, n, s,
                                                         static_cast<float*>(out->data), first);
  } else {
    auto P = [&](int k) { return static_cast<const double*>(E(k)); };
    k_meijering_max<double><<<grid_for(n), 256, 0, st>>>(P(0), P(1), P(2), ndim, alpha, n, s);
    k_meijering_fold<double><<<grid_for(n), 256, 0, st>>>(
        P(0), P(1), P(2), ndim, alpha, n, s, static_cast<double*>(out->data), first);
  }
  return cuda_fail(cudaGetLastError(), "meijering launch");
}

int cimx_sato_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out, double sigma,
                         int first, void* stream) {
  int rc = check_eigs(eigs, ndim, out);
  if (rc) return rc;
  const int64_t n = count(out);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double s2 = sigma * sigma;  // sigma**2 in Python, then the array's type
  if (out->dtype == DT_F32)
    k_sato<float><<<grid_for(n), 256, 0, st>>>(
        static_cast<const float*>(eigs[0].data), static_cast<const float*>(eigs[1].data),
        ndim, static_cast<float>(s2), n, static_cast<float*>(out->data), first);
  else
    k_sato<double><<<grid_for(n), 256, 0, st>>>(
        static_cast<const double*>(eigs[0].data), static_cast<const double*>(eigs[1].data),
        ndim, s2, n, static_cast<double*>(out->data), first);
  return cuda_fail(cudaGetLastError(), "sato launch");
}

int cimx_nonpositive_to_one(const CimxArray* a, void* stream) {
  if (!a) return fail(CIMX_E_INVALID, "NULL argument");
  if (a->dtype != DT_F32 && a->dtype != DT_F64) return fail(CIMX_E_DTYPE, "float32/float64 only");
  const int64_t n = count(a);
  if (n == 0) return CIMX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->dtype == DT_F32)
    k_le0_to_one<float><<<grid_for(n), 256, 0, st>>>(static_cast<float*>(a->data), n);
  else
    k_le0_to_one<double><<<grid_for(n), 256, 0, st>>>(static_cast<double*>(a->data), n);
  return cuda_fail(cudaGetLastError(), "hessian ridge launch");
}

}  // extern "C"
