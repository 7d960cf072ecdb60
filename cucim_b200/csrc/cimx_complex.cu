// cimx_complex.cu — 1-D correlation passes over complex arrays, or with
// complex taps: cuCIM's elementwise and shared-memory kernels instantiated
// with W = complex<float> / complex<double>
// (_vendored/_ndimage_filters.py:224-244, _vendored/_ndimage_util.py:35-37,
// filters/_separable_filtering.py:720-760). Rare in practice, so one plain
// kernel serves every pass: one thread per output, taps ascending.
//
// Arithmetic of one output, as the generated kernels compute it:
//   sum = (W)0;  for k: if (the elementwise kernel && w[k] == 0 + 0i) skip;
//                      sum = sum + value(x) * w[k];
//   y = (D)sum  (component-wise conversion)
// The complex product is the textbook form of the complex header the kernels
// include, (x.r w.r - x.i w.i, x.i w.r + x.r w.i), which the compiler's
// contraction turns into one fused multiply-add per part:
//   p.r = fma(x.r, w.r, -(x.i * w.i)),  p.i = fma(x.i, w.r, x.r * w.i);
// each part of the sum is a separate rounded add. With real taps (w.i = +0)
// every part of the sum is a chain of adds of rounded products, whatever the
// contraction.
//
// value(x), the input converted to W:
//   complex input: its parts (complex128 input always has W = complex<double>);
//   real input: (x, 0), where the elementwise kernel's cast<W>() rule
//   ((a >= 0) ? (W)a : -(W)(-a), _vendored/_ndimage_filters_core.py:234-244)
//   gives a negative (or NaN) floating-point value the imaginary part -0. In
//   constant mode the elementwise kernel converts in-bounds values implicitly
//   (imaginary part +0) and only the fill value goes through cast<W>(); the
//   shared-memory kernel converts with static_cast (+0), its fill value being
//   (W)(T)cval.
#include <algorithm>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

template <class R>
struct CArgs {
  const void* in;
  void* out;
  int tin, tout;
  long long outer, L, inner, n;
  int K, anchor, mode;
  int skip;       // skip taps equal to 0 + 0i (elementwise kernel)
  int sign_rule;  // in-bounds real values take cast<W>()'s sign rule
  int cval_as_input;
  double cval;
  const R* taps;  // K (re, im) pairs, rounded to R
};

__device__ __forceinline__ float f_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double f_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double f_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double f_add(double a, double b) { return __dadd_rn(a, b); }

__host__ __device__ inline bool float_dt(int dt) {
  return dt == DT_F32 || dt == DT_F64 || dt == DT_F16;
}

// element i of an array of dtype dt as the parts of W (parts loaded one by
// one: the caller's buffer need only be aligned to its component type)
template <class R>
__device__ __forceinline__ void load_c(const void* p, long long i, int dt, bool sign_rule, R& re,
                                       R& im) {
  if (dt == DT_C64) {
    const float* q = static_cast<const float*>(p) + 2 * i;
    re = static_cast<R>(q[0]);
    im = static_cast<R>(q[1]);
  } else if (dt == DT_C128) {
    const double* q = static_cast<const double*>(p) + 2 * i;
    re = static_cast<R>(q[0]);
    im = static_cast<R>(q[1]);
  } else {
    re = load_as<R>(p, i, dt);
    im = (sign_rule && float_dt(dt) && !(re >= R(0))) ? R(-0.0) : R(0);
  }
}

template <class R>
__device__ __forceinline__ void store_c(void* p, long long i, int dt, R re, R im) {
  if (dt == DT_C64) {
    float* q = static_cast<float*>(p) + 2 * i;
    q[0] = static_cast<float>(re);
    q[1] = static_cast<float>(im);
  } else {
    double* q = static_cast<double*>(p) + 2 * i;
    q[0] = static_cast<double>(re);
    q[1] = static_cast<double>(im);
  }
}

template <class R>
__global__ void __launch_bounds__(256) k_complex_pass(const CArgs<R> a) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < a.n;
       idx += stride) {
    const long long i = idx % a.inner;
    const long long t = idx / a.inner;
    const long long l = t % a.L, o = t / a.L;
    const long long base = o * a.L * a.inner + i;
    // constant mode's fill value as W: (W)(T)cval in the shared-memory
    // kernel (T = the dtype this pass reads), cast<W>(cval) in the
    // elementwise kernel
    R cre, cim = R(0);
    if (a.cval_as_input) {
      if (a.tin == DT_C64) cre = static_cast<R>(static_cast<float>(a.cval));
      else if (a.tin == DT_C128) cre = static_cast<R>(a.cval);
      else cre = fill_value<R>(a.cval, 1, a.tin);
    } else {
      cre = static_cast<R>(a.cval);
      if (!(a.cval >= 0)) cim = R(-0.0);
    }
    R sr = R(0), si = R(0);
    for (int k = 0; k < a.K; ++k) {
      const R wr = a.taps[2 * k], wi = a.taps[2 * k + 1];
      if (a.skip && wr == R(0) && wi == R(0)) continue;
      const long long m = map_coord(l - a.anchor + k, a.L, a.mode);
      R xr, xi;
      if (m < 0) {
        xr = cre;
        xi = cim;
      } else {
        load_c<R>(a.in, base + m * a.inner, a.tin, a.sign_rule != 0, xr, xi);
      }
      const R pr = f_fma(xr, wr, -f_mul(xi, wi));
      const R pi = f_fma(xi, wr, f_mul(xr, wi));
      sr = f_add(sr, pr);
      si = f_add(si, pi);
    }
    store_c<R>(a.out, idx, a.tout, sr, si);
  }
}

// in -> out with a conversion to the output's complex type (no filter)
__global__ void __launch_bounds__(256) k_complex_copy(const void* in, int tin, void* out, int tout,
                                                      long long n) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < n;
       idx += stride) {
    double re, im;  // every part converts to double exactly
    load_c<double>(in, idx, tin, false, re, im);
    store_c<double>(out, idx, tout, re, im);
  }
}

unsigned grid_for(long long n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long blocks = (n + 255) / 256;
  return static_cast<unsigned>(std::max<long long>(1, std::min<long long>(blocks, 8LL * sms)));
}

template <class R>
int launch_cpass(const PassDesc& d, int64_t n, cudaStream_t st) {
  CArgs<R> a{};
  a.in = d.in;
  a.out = d.out;
  a.tin = d.tin;
  a.tout = d.tout;
  a.outer = d.outer;
  a.L = d.L;
  a.inner = d.inner;
  a.n = n;
  a.K = d.K;
  a.anchor = d.anchor;
  a.mode = d.mode;
  a.skip = d.skip_zero ? 1 : 0;
  // the elementwise kernel (zero taps skipped) in a non-constant mode takes
  // cast<W>()'s sign rule for every value; in constant mode only the fill
  // value does
  a.sign_rule = (d.skip_zero && d.mode != CIMX_MODE_CONSTANT) ? 1 : 0;
  a.cval_as_input = d.cval_as_input ? 1 : 0;
  a.cval = d.cval;
  std::vector<R> w(2 * static_cast<size_t>(d.K));
  for (int k = 0; k < d.K; ++k) {
    w[2 * k] = static_cast<R>(d.ctaps ? d.taps[2 * k] : d.taps[k]);
    w[2 * k + 1] = d.ctaps ? static_cast<R>(d.taps[2 * k + 1]) : R(0);
  }
  const size_t wbytes = w.size() * sizeof(R);
  void* gt = scratch_alloc(wbytes, st);
  if (!gt) return fail(CIMX_E_NOMEM, "scratch allocation for taps failed");
  cudaError_t e = cudaMemcpyAsync(gt, w.data(), wbytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    scratch_free(gt, wbytes, st);
    return cuda_fail(e, "tap upload");
  }
  a.taps = static_cast<const R*>(gt);
  k_complex_pass<R><<<grid_for(n), 256, 0, st>>>(a);
  e = cudaGetLastError();
  scratch_free(gt, wbytes, st);
  return cuda_fail(e, "complex pass launch");
}

}  // namespace

int complex_separable(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
                      cudaStream_t st) {
  if (!is_complex_dt(out->dtype)) return fail(CIMX_E_DTYPE, "output must have complex dtype");
  int64_t n = 1;
  for (int d = 0; d < in->ndim; ++d) n *= in->shape[d];
  if (n == 0) return CIMX_OK;
  if (npasses == 0) {
    k_complex_copy<<<grid_for(n), 256, 0, st>>>(in->data, in->dtype, out->data, out->dtype, n);
    return cuda_fail(cudaGetLastError(), "complex copy launch");
  }
  void* temp = nullptr;
  const size_t tbytes = static_cast<size_t>(n) * element_size(out->dtype);
  if (npasses > 1) {
    temp = scratch_alloc(tbytes, st);
    if (!temp) return fail(CIMX_E_NOMEM, "scratch allocation for the ping-pong buffer failed");
  }
  const void* src = in->data;
  int tsrc = in->dtype;
  void* dst = (npasses % 2 == 0) ? temp : out->data;
  int rc = CIMX_OK;
  for (int i = 0; i < npasses && rc == CIMX_OK; ++i) {
    ds[i].in = src;
    ds[i].tin = tsrc;
    ds[i].out = dst;
    ds[i].tout = out->dtype;
    rc = ds[i].w64 ? launch_cpass<double>(ds[i], n, st) : launch_cpass<float>(ds[i], n, st);
    src = dst;
    tsrc = out->dtype;
    dst = (dst == out->data) ? temp : out->data;
  }
  scratch_free(temp, tbytes, st);
  return rc;
}

}  // namespace cimx
