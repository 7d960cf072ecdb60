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

// Host code cannot use g_noalloc_scratch's name as a device address: resolve
// it once per device with that device current.
std::mutex g_mu;
void* g_scratch_ptr[64] = {nullptr};

int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(CIMX_E_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_scratch_ptr[dev] = p;
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
    const CimxPass& p = passes[i];
    if (p.ntaps < 1 || !p.taps) return fail(CIMX_E_INVALID, "incorrect filter size");
    int axis = p.axis < 0 ? p.axis + in->ndim : p.axis;
    if (axis < 0 || axis >= in->ndim) return fail(CIMX_E_INVALID, "axis out of range");
    if (p.mode < CIMX_MODE_REFLECT || p.mode > CIMX_MODE_CONSTANT)
      return fail(CIMX_E_INVALID, "boundary mode not supported");
    const int K = p.ntaps;
    int origin = p.origin;
    if (K / 2 + origin < 0 || K / 2 + origin >= K) return fail(CIMX_E_INVALID, "invalid origin");
    const bool w64 = (p.flags & CIMX_F_W64) != 0;
    const size_t max_taps = kParamTapBytes / (w64 ? sizeof(double) : sizeof(float));
    if ((size_t)K > max_taps)
      return fail(CIMX_E_INVALID,
                  "cimx_separable_noalloc: a pass has " + std::to_string(K) +
                      " taps; without scratch memory at most " + std::to_string(max_taps) +
                      " fit in the launch parameters");
    taps[i].assign(p.taps, p.taps + K);
    if (p.flags & CIMX_F_CONVOLVE) {
      std::reverse(taps[i].begin(), taps[i].end());
      origin = -origin;
      if (K % 2 == 0) origin -= 1;
    }
    PassDesc& d = ds[i];
    d = PassDesc{};
    d.outer = 1;
    for (int k = 0; k < axis; ++k) d.outer *= in->shape[k];
    d.L = in->shape[axis];
    d.inner = 1;
    for (int k = axis + 1; k < in->ndim; ++k) d.inner *= in->shape[k];
    d.axis = axis;
    d.K = K;
    d.anchor = K / 2 + origin;
    d.mode = p.mode;
    d.cval = p.cval;
    d.w64 = w64;
    d.cval_as_input = (p.flags & CIMX_F_CVAL_AS_INPUT) != 0;
    d.skip_zero = (p.flags & CIMX_F_SKIP_ZERO_TAPS) != 0;
    d.taps = taps[i].data();
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
