// cimx_noalloc.cu — cimx_separable_noalloc: the multi-pass separable filter
// for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc or any allocating routine: code that
// runs while a CUDA graph is being captured by someone else, plug-ins that
// live inside a host application owning every device allocation, or
// real-time pipelines that forbid allocation after start-up. cimx_separable
// takes its ping-pong buffer from an allocator; this entry point takes it
// from a file-scope static device array instead, so a call allocates
// nothing.
//
// The array holds kNoAllocScratchBytes (64 MiB) on every GPU that loads the
// library, until the process exits. A call whose intermediate does not fit,
// or whose tap vector does not fit in the launch parameters, is rejected.
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_fused.h"
#include "cimx_internal.h"

namespace cimx {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code cannot use g_noalloc_scratch's name as a device address: the
// address is resolved with cudaGetSymbolAddress, with the device current, the
// first time a device is used. The cache is keyed on the device's current
// context as well, so that after cudaDeviceReset (which gives the module, and
// the array, a new address in a new primary context) the address is resolved
// again instead of reused.
using CtxGetCurrentFn = int (*)(void**);  // cuCtxGetCurrent(CUcontext*)

CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  });
  return fn;
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};
void* g_scratch_ctx[kMaxDevices] = {nullptr};

int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(CIMX_E_INVALID, "device ordinal out of range");
  CtxGetCurrentFn get = ctx_get_current();
  if (!get) return fail(CIMX_E_CUDA, "cuCtxGetCurrent is not available");
  // NULL before the runtime has made the device's primary context current
  void* ctx = nullptr;
  if (get(&ctx) != 0) return fail(CIMX_E_CUDA, "cuCtxGetCurrent failed");
  std::lock_guard<std::mutex> g(g_mu);
  if (!ctx || !g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    // resolving the symbol also creates the primary context when needed
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    if (get(&ctx) != 0 || !ctx) return fail(CIMX_E_CUDA, "no current context");
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return CIMX_OK;
}

int64_t count(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

bool dense(const CimxArray* a) {
  if (count(a) == 0) return true;
  int64_t expect = dtype_size(a->dtype);
  for (int d = a->ndim - 1; d >= 0; --d) {
    if (a->shape[d] != 1 && a->strides[d] != expect) return false;
    expect *= a->shape[d];
  }
  return true;
}

int check(const CimxArray* a, const char* name) {
  if (!a) return fail(CIMX_E_INVALID, std::string(name) + " is NULL");
  if (a->ndim < 1 || a->ndim > CIMX_MAX_NDIM)
    return fail(CIMX_E_INVALID, std::string(name) + ": ndim out of range");
  if (dtype_size(a->dtype) == 0) return fail(CIMX_E_DTYPE, std::string(name) + ": unsupported dtype");
  if (!dense(a)) return fail(CIMX_E_LAYOUT, std::string(name) + " is not C-contiguous");
  if (count(a) > 0 && !a->data) return fail(CIMX_E_INVALID, std::string(name) + ": NULL data");
  return CIMX_OK;
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" CIMX_API int cimx_separable_noalloc(const CimxArray* in, const CimxArray* out,
                                               const CimxPass* passes, int npasses,
                                               void* stream) {
  int rc;
  if ((rc = check(in, "input")) || (rc = check(out, "output"))) return rc;
  if (in->ndim != out->ndim) return fail(CIMX_E_INVALID, "output shape not correct");
  for (int d = 0; d < in->ndim; ++d)
    if (in->shape[d] != out->shape[d]) return fail(CIMX_E_INVALID, "output shape not correct");
  if (npasses < 0 || (npasses > 0 && !passes)) return fail(CIMX_E_INVALID, "bad pass list");
  const int64_t n = count(in);
  {
    const char* a0 = static_cast<const char*>(in->data);
    const char* b0 = static_cast<const char*>(out->data);
    if (n > 0 && a0 < b0 + n * dtype_size(out->dtype) && b0 < a0 + n * dtype_size(in->dtype))
      return fail(CIMX_E_INVALID, "input and output overlap");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // resolve every pass and check the limits before touching the device
  std::vector<std::vector<double>> taps(npasses);
  std::vector<PassDesc> ds(npasses);
  for (int i = 0; i < npasses; ++i) {
    if ((rc = make_pass(in, passes[i], taps[i], ds[i]))) return rc;
    const size_t max_taps = kParamTapBytes / (ds[i].w64 ? sizeof(double) : sizeof(float));
    if ((size_t)ds[i].K > max_taps)
      return fail(CIMX_E_INVALID,
                  "cimx_separable_noalloc: a pass has " + std::to_string(ds[i].K) +
                      " taps; without scratch memory at most " + std::to_string(max_taps) +
                      " fit in the launch parameters");
    // a pass whose taps would have to go to device memory fails instead
    ds[i].no_alloc = true;
  }
  const size_t need = npasses > 1 ? (size_t)n * dtype_size(out->dtype) : 0;
  if (need > kNoAllocScratchBytes)
    return fail(CIMX_E_INVALID, "cimx_separable_noalloc: the intermediate needs " +
                                    std::to_string(need) + " bytes; the static scratch holds " +
                                    std::to_string(kNoAllocScratchBytes) + " bytes");
  if (n == 0) return CIMX_OK;
  if (npasses == 0) return launch_copy_cast(in->data, in->dtype, out->data, out->dtype, n, st);

  void* temp = nullptr;
  if (need > 0 && (rc = scratch_address(&temp))) return rc;

  // ping-pong between `out` and the static scratch, as _run_1d_filters does:
  // the last pass writes `out`; every scratch element a pass reads was
  // written by the previous pass of this call, so nothing needs clearing
  const void* src = in->data;
  int tsrc = in->dtype;
  void* dst = (npasses % 2 == 0) ? temp : out->data;
  for (int i = 0; i < npasses; ++i) {
    ds[i].in = src;
    ds[i].tin = tsrc;
    ds[i].out = dst;
    ds[i].tout = out->dtype;
    if ((rc = launch_generic_pass(ds[i], st))) return rc;
    src = dst;
    tsrc = out->dtype;
    dst = (dst == out->data) ? temp : out->data;
  }
  return CIMX_OK;
}
