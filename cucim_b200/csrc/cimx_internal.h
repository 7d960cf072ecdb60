// cimx_internal.h — host-side interfaces between the C-ABI layer and the
// kernel families of libcimx.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/cimx.h"

namespace cimx {

// Taps travel to the kernels inside the launch parameters (no host->device
// copy per call) up to this many bytes; longer tap vectors are copied into
// scratch memory.
constexpr int kParamTapBytes = 4096;

// A single 1-D pass over the C-contiguous view (outer, L, inner) of the
// input, along the middle axis.
struct PassDesc {
  const void* in;
  void* out;
  int tin, tout;
  int64_t outer, L, inner;
  int axis;        // axis of the array the pass runs along
  int K;           // taps
  int anchor;      // tap k reads input coordinate l - anchor + k
  int mode;        // CIMX_MODE_*
  double cval;     // caller's fill value
  bool w64;        // weights type is float64
  bool cval_as_input;
  bool skip_zero;  // skip zero taps (only matters for non-finite inputs)
  bool no_alloc;   // the pass must not take scratch memory (cimx_separable_noalloc)
  bool ctaps;      // taps are K (re, im) pairs (CIMX_F_COMPLEX_TAPS)
  const double* taps;  // host taps, already flipped for convolution, not yet rounded
};

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// Argument checks shared by every entry point that takes a CimxPass list
// (cimx_api.cu): the boundary mode, and one pass resolved against the shape of
// `shape_of` into a PassDesc (taps copied into taps_store and flipped for
// convolution, origin checked, anchor computed). in/out/dtypes are left for
// the caller to fill.
int check_mode(int mode);
int make_pass(const CimxArray* shape_of, const CimxPass& p, std::vector<double>& taps_store,
              PassDesc& d);

// scratch memory through the installed allocator
void* scratch_alloc(size_t nbytes, cudaStream_t s);
void scratch_free(void* p, size_t nbytes, cudaStream_t s);

// The autotuner (cimx_tune.cu): the table key of a resolved pass list, and
// the library flags to run it with (the caller's, or the tuned schedule;
// with tuning on and an unseen key, `run(flags)` is timed for every
// candidate schedule first).
// Whether a call with these flags consults the tuning table at all (tuning
// on, or entries recorded and no schedule forced): cheap, so that untuned
// calls skip building the key.
bool tuning_needed(int lib_flags);
std::string tune_key(const CimxArray* in, const CimxArray* out, const PassDesc* ds,
                     int npasses, int lib_flags);
int tuned_flags(const std::string& key, int lib_flags, cudaStream_t st,
                const std::function<int(int)>& run);

// generic single pass (cimx_pass.cu)
int launch_generic_pass(const PassDesc& d, cudaStream_t stream);

// Passes over complex arrays or with complex taps (cimx_complex.cu): cuCIM's
// complex<float> / complex<double> arithmetic, one launch per pass through
// one scratch array of the output dtype. ds[i].in/out/tin/tout are set here.
// npasses == 0 copies `in` into `out` with a complex conversion.
int complex_separable(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
                      cudaStream_t st);

// elementwise helpers (cimx_elementwise.cu)
int launch_square_accumulate(void* acc, const void* term, int dt, int64_t n, bool first,
                             cudaStream_t stream);
int launch_sqrt_inplace(void* acc, int dt, int64_t n, cudaStream_t stream);

}  // namespace cimx
