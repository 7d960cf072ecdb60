// cimx_tc.h — the split-precision tensor-core pass (cimx_tc.cu).
#pragma once

#include "cimx_internal.h"

namespace cimx {

// Whether a resolved pass can run on the tensor-core kernel (float32 input
// and output, float32 weights, at most 385 taps).
bool tc_supports(const PassDesc& d);

// One pass on the tensor cores: BF16x3 split precision, float32 accumulation.
int launch_tc_pass(const PassDesc& d, cudaStream_t stream);

}  // namespace cimx
