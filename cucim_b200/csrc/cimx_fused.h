// cimx_fused.h — entry into the fused multi-pass kernels (cimx_fused.cu).
#pragma once

#include "cimx_internal.h"

namespace cimx {

// Returned by try_fused when no fused kernel covers the pass list; the
// caller then runs the passes one launch at a time.
constexpr int CIMX_FUSED_DECLINED = 1;

// Runs the whole pass list `ds` (already resolved against the input shape)
// in fused launches when a fused kernel covers it. Returns CIMX_OK, a
// negative error, or CIMX_FUSED_DECLINED.
int try_fused(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
              cudaStream_t stream);

// elementwise copy with conversion (used when a filter has no passes)
int launch_copy_cast(const void* in, int tin, void* out, int tout, int64_t n,
                     cudaStream_t stream);

}  // namespace cimx
