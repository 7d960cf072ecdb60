// cimx_fused.cu — decides whether a pass list runs on the fast kernels
// (cimx_fast.cuh, cimx_vol.cuh) and schedules them: a 3-D filter with short
// taps on all three axes is one launch of the volume kernel (k_vol);
// otherwise passes along leading axes are streamed one launch each
// (k_stream; the generic kernel for taps it does not cover), the passes
// along the last two axes run fused in one slab launch (k_slab or
// k_rowstream). Intermediates follow cuCIM's _run_1d_filters
// ping-pong: every pass writes the output dtype, the last launch writes the
// caller's output, one scratch buffer takes the others.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_fused.h"

namespace cimx {
namespace {

// (T, D) pairs with fast kernels; all of them use float32 weights.
bool fast_pair(int t, int d) {
  switch (t) {
    case DT_F32: return d == DT_F32;
    case DT_U16: return d == DT_F32 || d == DT_U16;
    case DT_U8: return d == DT_F32 || d == DT_U8 || d == DT_U16;
    default: return false;
  }
}

// tap counts of the stream kernel's instantiations: the gaussians of
// sigma 0.5 / 0.75 / 1 / 1.25 / 1.5 / 1.75 / 2 (truncate 4) and the short
// box and derivative filters. Longer passes run faster on the generic
// column kernel (measured along axis 0 of 256 x 512^2 float32: 19 / 25 taps
// 303 / 583 us on the stream kernel, 250 / 263 us on k_cols_pairs).
constexpr int kStreamMaxK = 17;
bool stream_supports(int K) {
  return K == 3 || K == 5 || K == 7 || K == 9 || K == 11 || K == 13 || K == 15 || K == 17;
}

struct Trimmed {
  int K = 0, anchor = 0;
  bool interior_zero = false;
  float w[kSlabMaxK];
};

// Taps rounded to float32; with the elementwise-kernel rule, zero taps at
// both ends are dropped (exact: they never enter the chain).
bool trim(const PassDesc& d, int max_k, Trimmed& t) {
  if (d.w64) return false;
  int lo = 0, hi = d.K;
  auto w = [&](int k) { return static_cast<float>(d.taps[k]); };
  if (d.skip_zero) {
    while (lo < hi && w(lo) == 0.f) ++lo;
    while (hi > lo && w(hi - 1) == 0.f) --hi;
  }
  t.K = hi - lo;
  if (t.K < 1 || t.K > max_k) return false;
  t.anchor = d.anchor - lo;
  t.interior_zero = false;
  for (int k = lo; k < hi; ++k) {
    t.w[k - lo] = w(k);
    if (d.skip_zero && w(k) == 0.f) t.interior_zero = true;
  }
  return true;
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

int launch_stream(const PassDesc& d, const Trimmed& t, int tin, const void* in, int tout,
                  void* out, cudaStream_t st) {
  switch (tin) {
    case DT_F32: return launch_stream_f32(d, t.w, t.K, t.anchor, t.interior_zero, in, tout, out, st);
    case DT_U16: return launch_stream_u16(d, t.w, t.K, t.anchor, t.interior_zero, in, tout, out, st);
    case DT_U8: return launch_stream_u8(d, t.w, t.K, t.anchor, t.interior_zero, in, tout, out, st);
    default: return CIMX_FUSED_DECLINED;
  }
}

int launch_slab(SlabArgs& a, int tin, int tout, cudaStream_t st) {
  switch (tin) {
    case DT_F32: return launch_slab_f32(a, tout, st);
    case DT_U16: return launch_slab_u16(a, tout, st);
    case DT_U8: return launch_slab_u8(a, tout, st);
    default: return CIMX_FUSED_DECLINED;
  }
}

void fill_slab_pass(SlabPass& s, const PassDesc& d, const Trimmed& t, int pass_in) {
  s.K = t.K;
  s.K8 = (t.K + 7) / 8 * 8;
  s.anchor = t.anchor;
  s.mode = d.mode;
  s.cval = d.cval;
  s.cval_as_input = d.cval_as_input ? 1 : 0;
  s.dt = pass_in;
  s.skip = (d.skip_zero && t.interior_zero) ? 1 : 0;
  s.pad = 0;
  std::fill(std::begin(s.w), std::end(s.w), 0.f);
  std::copy(t.w, t.w + t.K, s.w);
}

int launch_vol(const VolArgs& v, int tin, int tout, cudaStream_t st) {
  switch (tin) {
    case DT_F32: return launch_vol_f32(v, tout, st);
    case DT_U16: return launch_vol_u16(v, tout, st);
    case DT_U8: return launch_vol_u8(v, tout, st);
    default: return CIMX_FUSED_DECLINED;
  }
}

// z, y and x passes over the last three axes with the same short taps: one
// launch of the volume kernel, no intermediate volume
int try_vol(const CimxArray* in, const CimxArray* out, const PassDesc* ds, int zchunk,
            cudaStream_t st) {
  const int nd = in->ndim;
  const int D = out->dtype;
  if (!fast_pair(in->dtype, D)) return CIMX_FUSED_DECLINED;
  Trimmed t[3];
  for (int i = 0; i < 3; ++i)
    if (!trim(ds[i], 5, t[i])) return CIMX_FUSED_DECLINED;
  const int K = t[0].K;
  if ((K != 3 && K != 5) || t[1].K != K || t[2].K != K) return CIMX_FUSED_DECLINED;
  // the x chain takes its halo from the neighbouring lanes: centred taps,
  // and no wrap-around (whose halo lies at the far end of the row)
  if (t[2].anchor != K / 2 || ds[2].mode == CIMX_MODE_GRID_WRAP) return CIMX_FUSED_DECLINED;
  const long long X = in->shape[nd - 1], Y = in->shape[nd - 2], Z = in->shape[nd - 3];
  long long B = 1;
  for (int k = 0; k < nd - 3; ++k) B *= in->shape[k];
  if (X % 4 != 0 || X < 8 || Y < 1 || Z < 1 || B < 1) return CIMX_FUSED_DECLINED;
  if (Y * X >= (1LL << 31) || Z >= (1LL << 31)) return CIMX_FUSED_DECLINED;
  if (!aligned(in->data, 4 * dtype_size(in->dtype)) || !aligned(out->data, 4 * dtype_size(D)))
    return CIMX_FUSED_DECLINED;
  VolArgs v{};
  v.in = in->data;
  v.out = out->data;
  v.B = B;
  v.Z = Z;
  v.Y = Y;
  v.X = X;
  v.zchunk = zchunk;
  fill_slab_pass(v.pz, ds[0], t[0], in->dtype);
  fill_slab_pass(v.py, ds[1], t[1], D);
  fill_slab_pass(v.px, ds[2], t[2], D);
  return launch_vol(v, in->dtype, D, st);
}

}  // namespace

int try_fused(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
              int lib_flags, cudaStream_t st) {
  const int nd = in->ndim;
  const int D = out->dtype;
  if (npasses < 1 || nd < 1) return CIMX_FUSED_DECLINED;
  // passes in strictly ascending axis order, float32 weights
  int prev_axis = -1;
  for (int i = 0; i < npasses; ++i) {
    if (ds[i].axis <= prev_axis || ds[i].w64) return CIMX_FUSED_DECLINED;
    prev_axis = ds[i].axis;
  }

  if (nd >= 3 && npasses == 3 && ds[0].axis == nd - 3 && ds[1].axis == nd - 2 &&
      ds[2].axis == nd - 1 && !(lib_flags & CIMX_L_NO_VOLUME)) {
    static const int kChunks[4] = {0, 32, 64, 128};
    const int rc = try_vol(in, out, ds, kChunks[(lib_flags >> CIMX_L_ZCHUNK_SHIFT) & 3], st);
    if (rc != CIMX_FUSED_DECLINED) return rc;
  }

  // leading axes are streamed, the last two axes go to the slab kernel
  const int ylast = nd >= 2 ? nd - 2 : -1;
  std::vector<int> lead, tail;
  for (int i = 0; i < npasses; ++i) (ds[i].axis < ylast ? lead : tail).push_back(i);

  std::vector<Trimmed> tr(npasses);
  // a leading pass the stream kernel does not cover (longer taps, rows not
  // a multiple of 4) runs on the generic kernel: worthwhile while the last
  // two axes still take one slab launch
  std::vector<char> lead_generic(npasses, 0);
  for (size_t n = 0; n < lead.size(); ++n) {
    const int i = lead[n];
    const int tin = n == 0 ? in->dtype : D;
    const bool stream_ok = !(lib_flags & CIMX_L_NO_STREAM) && trim(ds[i], kStreamMaxK, tr[i]) &&
                           stream_supports(tr[i].K) && fast_pair(tin, D) &&
                           ds[i].inner % 4 == 0;
    if (!stream_ok) {
      if (tail.empty()) return CIMX_FUSED_DECLINED;
      lead_generic[i] = 1;
    }
  }
  const int tail_in = lead.empty() ? in->dtype : D;
  // a lone pass along the last axis over float32 data runs on the slab
  // kernel behind an identity y pass (one tap of 1: fma(v, 1, +0) = v, kept
  // as float32, exact). A -0 input becomes +0, which the x pass's chain from
  // +0 cannot tell apart. Measured on 16 x 2048 x 2048 with 9 taps: 148 us
  // against 266 us on the generic row kernel. For 8- and 16-bit input the
  // generic row kernel is the faster (uint16: 240 us against 316 us).
  const bool y_identity = !tail.empty() && nd >= 2 && ds[tail[0]].axis == nd - 1 &&
                          tail_in == DT_F32 && D == DT_F32;
  if (!tail.empty()) {
    // the slab kernel needs a pass along the second-to-last axis
    if (nd < 2 || (ds[tail[0]].axis != nd - 2 && !y_identity)) return CIMX_FUSED_DECLINED;
    if (!fast_pair(tail_in, D)) return CIMX_FUSED_DECLINED;
    for (int i : tail)
      if (!trim(ds[i], kSlabMaxK, tr[i])) return CIMX_FUSED_DECLINED;
  }
  const size_t vec_in = 4 * dtype_size(in->dtype), vec_out = 4 * dtype_size(D);
  if (!aligned(in->data, vec_in) || !aligned(out->data, vec_out)) return CIMX_FUSED_DECLINED;

  // ping-pong schedule: the last launch writes `out`
  const int nl = (int)lead.size() + (tail.empty() ? 0 : 1);
  int64_t n = 1;
  for (int k = 0; k < nd; ++k) n *= in->shape[k];
  const size_t tbytes = (size_t)n * dtype_size(D);
  void* temp = nullptr;
  if (nl >= 2) {
    temp = scratch_alloc(tbytes, st);
    if (!temp) return fail(CIMX_E_NOMEM, "scratch allocation for the ping-pong buffer failed");
  }
  auto dst_of = [&](int j) { return ((nl - 1 - j) % 2 == 0) ? out->data : temp; };

  int rc = CIMX_OK;
  const void* src = in->data;
  int tsrc = in->dtype;
  int j = 0;
  for (int i : lead) {
    void* dst = dst_of(j++);
    if (lead_generic[i]) {
      PassDesc d = ds[i];
      d.in = src;
      d.out = dst;
      d.tin = tsrc;
      d.tout = D;
      rc = launch_generic_pass(d, st);
    } else {
      rc = launch_stream(ds[i], tr[i], tsrc, src, D, dst, st);
    }
    if (rc != CIMX_OK) break;
    src = dst;
    tsrc = D;
  }
  if (rc == CIMX_OK && !tail.empty()) {
    SlabArgs a{};
    a.no_rowstream = (lib_flags & CIMX_L_NO_ROWSTREAM) ? 1 : 0;
    static const int kSpans[4] = {0, 1, 2, 8};
    a.span = kSpans[(lib_flags >> CIMX_L_SLAB_SPAN_SHIFT) & 3];
    a.in = src;
    a.out = dst_of(j++);
    a.X = in->shape[nd - 1];
    a.Y = nd >= 2 ? in->shape[nd - 2] : 1;
    a.B = (a.X * a.Y == 0) ? 0 : n / (a.X * a.Y);
    int pass_in = tsrc;
    if (y_identity) {
      a.py = SlabPass{};
      a.py.K = 1;
      a.py.K8 = 8;
      a.py.mode = CIMX_MODE_NEAREST;  // no halo: K = 1, anchor 0
      a.py.dt = pass_in;
      a.py.w[0] = 1.f;
      a.has_y = 1;
    }
    for (int i : tail) {
      const bool is_x = ds[i].axis == nd - 1;
      fill_slab_pass(is_x ? a.px : a.py, ds[i], tr[i], pass_in);
      (is_x ? a.has_x : a.has_y) = 1;
      pass_in = D;
    }
    rc = launch_slab(a, tsrc, D, st);
  }
  scratch_free(temp, tbytes, st);
  // every check that can decline ran before the first launch
  return rc == CIMX_FUSED_DECLINED ? fail(CIMX_E_INVALID, "fast kernel missing") : rc;
}

}  // namespace cimx
