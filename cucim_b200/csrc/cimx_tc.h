// cimx_tc.h — the split-precision tensor-core passes (cimx_tc.cu, cimx_tcs.cu).
#pragma once

#include "cimx_internal.h"

namespace cimx {

// Whether a resolved pass can run on the tensor-core kernel (float32 input
// and output, float32 weights, at most 385 taps).
bool tc_supports(const PassDesc& d);

// One pass on the tensor cores: BF16x3 split precision, float32 accumulation.
int launch_tc_pass(const PassDesc& d, cudaStream_t stream);

// The streaming TF32x3 tensor-core pass (cimx_tcs.cu): float32 input and
// output, float32 weights, at most about 450 taps.
bool tcs_supports(const PassDesc& d);
int launch_tcs_pass(const PassDesc& d, cudaStream_t stream);

}  // namespace cimx
