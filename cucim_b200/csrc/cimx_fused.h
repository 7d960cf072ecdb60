// cimx_fused.h — entry into the fast kernels of the plain path
// (cimx_fast.cuh, instantiated per input dtype in cimx_fast_{f32,u16,u8}.cu)
// and the dispatcher that decides whether a pass list can use them
// (cimx_fused.cu).
#pragma once

#include "cimx_internal.h"

namespace cimx {

// Returned by try_fused when no fast kernel covers the pass list; the caller
// then runs the passes one launch at a time.
constexpr int CIMX_FUSED_DECLINED = 1;

constexpr int kSlabMaxK = 64;  // longest pass the slab kernel takes

// One pass of the slab kernel (float32 weights, already trimmed).
struct SlabPass {
  int K, K8, anchor, mode;
  double cval;
  int cval_as_input, dt, skip, pad;
  float w[kSlabMaxK];
};

struct SlabArgs {
  const void* in;
  void* out;
  long long B, Y, X;
  long long tiles_x, tiles_y;
  int has_y, has_x;
  int* status;  // device status word for bounded waits
  int no_rowstream;  // CIMX_L_NO_ROWSTREAM: always the slab kernel
  int span;          // slabs per CTA (float input with TMA); 0: about four
  SlabPass py, px;
};

// The three passes of a 3-D filter (z, y, x over the last three axes), for
// the single-launch volume kernel (cimx_vol.cuh).
struct VolArgs {
  const void* in;
  void* out;
  long long B, Z, Y, X;
  int zchunk;  // slices per CTA; 0: chosen from the grid size
  SlabPass pz, py, px;
};

// Runs the whole pass list `ds` (already resolved against the input shape)
// in fast launches when they cover it. Returns CIMX_OK, a negative error, or
// CIMX_FUSED_DECLINED (nothing was launched).
int try_fused(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
              int lib_flags, cudaStream_t stream);

// elementwise copy with conversion (used when a filter has no passes)
int launch_copy_cast(const void* in, int tin, void* out, int tout, int64_t n,
                     cudaStream_t stream);

// stream pass along a strided axis, by input dtype; K in {3,5,...,17} (odd)
int launch_stream_f32(const PassDesc& d, const float* w, int K, int anchor, bool interior_zero,
                      const void* in, int tout, void* out, cudaStream_t st);
int launch_stream_u16(const PassDesc& d, const float* w, int K, int anchor, bool interior_zero,
                      const void* in, int tout, void* out, cudaStream_t st);
int launch_stream_u8(const PassDesc& d, const float* w, int K, int anchor, bool interior_zero,
                     const void* in, int tout, void* out, cudaStream_t st);

// single-launch 3-D filter, by input dtype; equal K in {3, 5} on every axis
int launch_vol_f32(const VolArgs& v, int tout, cudaStream_t st);
int launch_vol_u16(const VolArgs& v, int tout, cudaStream_t st);
int launch_vol_u8(const VolArgs& v, int tout, cudaStream_t st);

// fused (y, x) slab launch, by input dtype
int launch_slab_f32(SlabArgs& a, int tout, cudaStream_t st);
int launch_slab_u16(SlabArgs& a, int tout, cudaStream_t st);
int launch_slab_u8(SlabArgs& a, int tout, cudaStream_t st);

}  // namespace cimx
