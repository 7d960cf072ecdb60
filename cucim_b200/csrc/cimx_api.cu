// cimx_api.cu — the extern "C" entry points of libcimx.so (declared in
// include/cimx.h): argument validation, the scratch allocator, error
// reporting and the choice between fused and per-pass kernels.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"
#include "cimx_fused.h"
#include "cimx_tc.h"

namespace cimx {

namespace {
thread_local std::string g_last_error;

// Keep freed blocks in the device's default pool instead of returning them
// to the driver at every synchronisation (the pool otherwise releases down to
// zero bytes, so each call would map its scratch afresh).
void retain_pool_memory() {
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  });
}

void* default_alloc(size_t n, void* stream, void*) {
  retain_pool_memory();
  void* p = nullptr;
  if (cudaMallocAsync(&p, n, static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void default_free(void* p, size_t, void* stream, void*) {
  cudaFreeAsync(p, static_cast<cudaStream_t>(stream));
}

std::mutex g_alloc_mu;
cimx_alloc_fn g_alloc = default_alloc;
cimx_free_fn g_free = default_free;
void* g_alloc_user = nullptr;
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CIMX_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return CIMX_E_CUDA;
}

void* scratch_alloc(size_t nbytes, cudaStream_t s) {
  cimx_alloc_fn f;
  void* u;
  {
    std::lock_guard<std::mutex> g(g_alloc_mu);
    f = g_alloc;
    u = g_alloc_user;
  }
  return f(nbytes, s, u);
}

void scratch_free(void* p, size_t nbytes, cudaStream_t s) {
  if (!p) return;
  cimx_free_fn f;
  void* u;
  {
    std::lock_guard<std::mutex> g(g_alloc_mu);
    f = g_free;
    u = g_alloc_user;
  }
  f(p, nbytes, s, u);
}

namespace {

bool supported_dtype(int dt) { return element_size(dt) > 0; }

int64_t numel(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

bool c_contiguous(const CimxArray* a) {
  if (numel(a) == 0) return true;
  int64_t expect = element_size(a->dtype);
  for (int d = a->ndim - 1; d >= 0; --d) {
    if (a->shape[d] != 1 && a->strides[d] != expect) return false;
    expect *= a->shape[d];
  }
  return true;
}

int check_array(const CimxArray* a, const char* name) {
  if (!a) return fail(CIMX_E_INVALID, std::string(name) + " is NULL");
  if (a->ndim < 0 || a->ndim > CIMX_MAX_NDIM)
    return fail(CIMX_E_INVALID, std::string(name) + ": ndim out of range");
  if (!supported_dtype(a->dtype))
    return fail(CIMX_E_DTYPE, std::string(name) + ": unsupported dtype code " +
                                  std::to_string(a->dtype));
  for (int d = 0; d < a->ndim; ++d)
    if (a->shape[d] < 0) return fail(CIMX_E_INVALID, std::string(name) + ": negative extent");
  if (!c_contiguous(a)) return fail(CIMX_E_LAYOUT, std::string(name) + " is not C-contiguous");
  if (numel(a) > 0 && !a->data) return fail(CIMX_E_INVALID, std::string(name) + ": NULL data");
  return CIMX_OK;
}

int check_same_shape(const CimxArray* a, const CimxArray* b) {
  if (a->ndim != b->ndim) return fail(CIMX_E_INVALID, "output shape not correct");
  for (int d = 0; d < a->ndim; ++d)
    if (a->shape[d] != b->shape[d]) return fail(CIMX_E_INVALID, "output shape not correct");
  return CIMX_OK;
}

bool overlaps(const CimxArray* a, const CimxArray* b) {
  const char* a0 = static_cast<const char*>(a->data);
  const char* b0 = static_cast<const char*>(b->data);
  const char* a1 = a0 + numel(a) * element_size(a->dtype);
  const char* b1 = b0 + numel(b) * element_size(b->dtype);
  return numel(a) > 0 && numel(b) > 0 && a0 < b1 && b0 < a1;
}

}  // namespace

int check_mode(int mode) {
  if (mode < CIMX_MODE_REFLECT || mode > CIMX_MODE_CONSTANT)
    return fail(CIMX_E_INVALID, "boundary mode not supported");
  return CIMX_OK;
}

// Resolve one pass against an array shape into a PassDesc (taps flipped for
// convolution, origin checked, anchor computed).
int make_pass(const CimxArray* shape_of, const CimxPass& p, std::vector<double>& taps_store,
              PassDesc& d) {
  if (p.ntaps < 1) return fail(CIMX_E_INVALID, "incorrect filter size");
  if (!p.taps) return fail(CIMX_E_INVALID, "taps is NULL");
  int axis = p.axis;
  if (axis < 0) axis += shape_of->ndim;
  if (axis < 0 || axis >= shape_of->ndim) return fail(CIMX_E_INVALID, "axis out of range");
  int rc = check_mode(p.mode);
  if (rc) return rc;
  const int K = p.ntaps;
  int origin = p.origin;
  if (K / 2 + origin < 0 || K / 2 + origin >= K) return fail(CIMX_E_INVALID, "invalid origin");
  const bool ctaps = (p.flags & CIMX_F_COMPLEX_TAPS) != 0;
  taps_store.assign(p.taps, p.taps + (ctaps ? 2 * K : K));
  if (p.flags & CIMX_F_CONVOLVE) {
    if (ctaps) {
      // reverse the (re, im) pairs
      for (int i = 0, j = K - 1; i < j; ++i, --j) {
        std::swap(taps_store[2 * i], taps_store[2 * j]);
        std::swap(taps_store[2 * i + 1], taps_store[2 * j + 1]);
      }
    } else {
      std::reverse(taps_store.begin(), taps_store.end());
    }
    origin = -origin;
    if (K % 2 == 0) origin -= 1;
  }
  d.outer = 1;
  for (int i = 0; i < axis; ++i) d.outer *= shape_of->shape[i];
  d.L = shape_of->shape[axis];
  d.inner = 1;
  for (int i = axis + 1; i < shape_of->ndim; ++i) d.inner *= shape_of->shape[i];
  d.axis = axis;
  d.K = K;
  d.anchor = K / 2 + origin;
  d.mode = p.mode;
  d.cval = p.cval;
  d.w64 = (p.flags & CIMX_F_W64) != 0;
  d.cval_as_input = (p.flags & CIMX_F_CVAL_AS_INPUT) != 0;
  d.skip_zero = (p.flags & CIMX_F_SKIP_ZERO_TAPS) != 0;
  d.ctaps = ctaps;
  d.taps = taps_store.data();
  return CIMX_OK;
}

}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_abi_version(void) { return 101; }

const char* cimx_last_error_string(void) { return g_last_error.c_str(); }

int cimx_set_allocator(cimx_alloc_fn alloc, cimx_free_fn release, void* user) {
  std::lock_guard<std::mutex> g(g_alloc_mu);
  if (!alloc || !release) {
    g_alloc = default_alloc;
    g_free = default_free;
    g_alloc_user = nullptr;
  } else {
    g_alloc = alloc;
    g_free = release;
    g_alloc_user = user;
  }
  return CIMX_OK;
}

int cimx_correlate1d(const CimxArray* in, const CimxArray* out, const double* taps, int ntaps,
                     int axis, int origin, int mode, double cval, int flags, void* stream) {
  int rc;
  if ((rc = check_array(in, "input")) || (rc = check_array(out, "output")) ||
      (rc = check_same_shape(in, out)))
    return rc;
  if (in->ndim == 0) return fail(CIMX_E_INVALID, "correlate1d needs ndim >= 1");
  if (overlaps(in, out)) return fail(CIMX_E_INVALID, "input and output overlap");
  CimxPass p{axis, ntaps, origin, mode, cval, flags, 0, taps};
  std::vector<double> ts;
  PassDesc d{};
  if ((rc = make_pass(in, p, ts, d))) return rc;
  d.in = in->data;
  d.out = out->data;
  d.tin = in->dtype;
  d.tout = out->dtype;
  if (is_complex_dt(in->dtype) || is_complex_dt(out->dtype) || d.ctaps)
    return complex_separable(in, out, &d, 1, static_cast<cudaStream_t>(stream));
  return launch_generic_pass(d, static_cast<cudaStream_t>(stream));
}

int cimx_separable(const CimxArray* in, const CimxArray* out, const CimxPass* passes,
                   int npasses, int lib_flags, void* stream) {
  int rc;
  if ((rc = check_array(in, "input")) || (rc = check_array(out, "output")) ||
      (rc = check_same_shape(in, out)))
    return rc;
  if (overlaps(in, out)) return fail(CIMX_E_INVALID, "input and output overlap");
  if (npasses < 0 || (npasses > 0 && !passes)) return fail(CIMX_E_INVALID, "bad pass list");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = numel(in);
  const bool cplx = is_complex_dt(in->dtype) || is_complex_dt(out->dtype);
  if (npasses == 0) {
    if (cplx) return complex_separable(in, out, nullptr, 0, st);
    return launch_copy_cast(in->data, in->dtype, out->data, out->dtype, n, st);
  }
  if (in->ndim == 0) return fail(CIMX_E_INVALID, "separable filtering needs ndim >= 1");

  std::vector<std::vector<double>> taps(npasses);
  std::vector<PassDesc> ds(npasses);
  bool ctaps = false;
  for (int i = 0; i < npasses; ++i) {
    if ((rc = make_pass(in, passes[i], taps[i], ds[i]))) return rc;
    ctaps = ctaps || ds[i].ctaps;
  }
  // complex arrays or taps: cuCIM's complex<float> / complex<double> kernels,
  // one launch per pass
  if (cplx || ctaps) return complex_separable(in, out, ds.data(), npasses, st);
  if (n == 0) return CIMX_OK;

  // the autotuner's schedule for this signature (or the caller's flags)
  if (!(lib_flags & CIMX_L_NO_TUNE) && tuning_needed(lib_flags)) {
    const std::string key = tune_key(in, out, ds.data(), npasses, lib_flags);
    lib_flags = tuned_flags(key, lib_flags, st, [&](int f) {
      return cimx_separable(in, out, passes, npasses, f, stream);
    });
  }

  const bool tf32x3 = (lib_flags & CIMX_L_TENSOR_TF32X3) != 0;
  const bool tensor = tf32x3 || (lib_flags & CIMX_L_TENSOR_BF16X3) != 0;
  // Tensor-core passes where they measured faster than the plain kernels: on
  // a B200, 1.2-2.3x for 23-143 taps along 8192-sample lines, slower or even
  // for every length along 256-sample lines (the band's halo and the strip
  // set-up dominate short lines). CIMX_L_TENSOR_ALL_LINES lifts the limit.
  constexpr int64_t kTensorMinLine = 2048;
  const bool all_lines = (lib_flags & CIMX_L_TENSOR_ALL_LINES) != 0;
  auto tensor_kind = [&](const PassDesc& d) {
    if (!tensor || d.K < 16 || (!all_lines && d.L < kTensorMinLine)) return 0;
    if (tf32x3) return tcs_supports(d) ? 1 : 0;
    return tc_supports(d) ? 2 : 0;
  };
  bool any_tensor = false;
  for (int i = 0; i < npasses; ++i) {
    PassDesc d = ds[i];  // the dtypes each pass will see
    d.in = in->data;
    d.out = out->data;
    d.tin = i == 0 ? in->dtype : out->dtype;
    d.tout = out->dtype;
    any_tensor = any_tensor || tensor_kind(d) != 0;
  }
  // fused kernels take whole runs of passes in one launch
  if (!any_tensor && !(lib_flags & CIMX_L_NO_FUSION)) {
    rc = try_fused(in, out, ds.data(), npasses, lib_flags, st);
    if (rc != CIMX_FUSED_DECLINED) return rc;
    rc = CIMX_OK;
  }

  // one launch per pass, ping-pong between `out` and one temporary of the
  // output dtype exactly like _run_1d_filters
  void* temp = nullptr;
  const size_t tbytes = (size_t)n * dtype_size(out->dtype);
  if (npasses > 1) {
    temp = scratch_alloc(tbytes, st);
    if (!temp) return fail(CIMX_E_NOMEM, "scratch allocation for the ping-pong buffer failed");
  }
  const void* src = in->data;
  int tsrc = in->dtype;
  void* dst = (npasses % 2 == 0) ? temp : out->data;
  for (int i = 0; i < npasses && rc == CIMX_OK; ++i) {
    ds[i].in = src;
    ds[i].tin = tsrc;
    ds[i].out = dst;
    ds[i].tout = out->dtype;
    const int kind = tensor_kind(ds[i]);
    if (kind == 1) {
      rc = launch_tcs_pass(ds[i], st);
    } else if (kind == 2) {
      rc = launch_tc_pass(ds[i], st);
    } else {
      // a pass list the fused kernels do not take as a whole (axes out of
      // ascending order, as the edge filters' edge-then-smooth chains along
      // axis 1 or 2): each pass on its own still runs on a fast kernel when
      // one covers it (the stream kernel for a leading axis, the slab for a
      // pass along the second-to-last axis), the same chain as the generic
      // kernel. CIMX_L_NO_FUSION keeps the generic kernels.
      rc = CIMX_FUSED_DECLINED;
      if (!(lib_flags & CIMX_L_NO_FUSION)) {
        CimxArray s_arr = i == 0 ? *in : *out, d_arr = *out;
        s_arr.data = const_cast<void*>(src);
        d_arr.data = dst;
        rc = try_fused(&s_arr, &d_arr, &ds[i], 1, lib_flags, st);
      }
      if (rc == CIMX_FUSED_DECLINED) rc = launch_generic_pass(ds[i], st);
    }
    src = dst;
    tsrc = out->dtype;
    dst = (dst == out->data) ? temp : out->data;
  }
  scratch_free(temp, tbytes, st);
  return rc;
}

}  // extern "C"
