// cimx_fused.cu — the fast kernels of the plain (exact float32) path.
//
// (a) k_stream: one pass along a strided axis of the view (outer, L, inner).
//     Each thread owns 4 consecutive inner positions (one 4-wide vector
//     load/store per row) and walks a chunk of L, keeping the last K rows in
//     registers as a ring indexed at compile time: every input row is read
//     once per chunk and every tap is a constant-bank FMA operand.
// (b) k_slab: the last two axes (y, x) of a (B, Y, X) view in one launch: a
//     halo'd tile is staged in shared memory, the y pass writes its result
//     (rounded through the output dtype, as the ping-pong of cuCIM's
//     _run_1d_filters does) to a second shared tile, and the x pass stores
//     the outputs, so the intermediate never travels to HBM.
//
// Both compute every output with the same fused multiply-add chain as the
// generic kernels (taps ascending, float32 FMA from +0, cast<D>()), so a pass
// list gives bit-identical results whichever kernels run it.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_fused.h"

namespace cimx {
namespace {

constexpr int P = 8;  // consecutive outputs per thread in the slab kernel
constexpr int kMaxSmem = 227 * 1024;

// ------------------------------------------------------------ vector I/O

template <class T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<uint16_t> { using type = ushort4; };
template <> struct Vec4<uint8_t> { using type = uchar4; };

template <class T>
__device__ __forceinline__ void load4(const T* p, float (&v)[4]) {
  const typename Vec4<T>::type q = *reinterpret_cast<const typename Vec4<T>::type*>(p);
  v[0] = static_cast<float>(q.x);
  v[1] = static_cast<float>(q.y);
  v[2] = static_cast<float>(q.z);
  v[3] = static_cast<float>(q.w);
}

template <class D>
__device__ __forceinline__ void store4(D* p, float a, float b, float c, float d) {
  typename Vec4<D>::type q;
  q.x = out_cast<D>(a);
  q.y = out_cast<D>(b);
  q.z = out_cast<D>(c);
  q.w = out_cast<D>(d);
  *reinterpret_cast<typename Vec4<D>::type*>(p) = q;
}

template <class T> constexpr int dt_code();
template <> constexpr int dt_code<float>() { return DT_F32; }
template <> constexpr int dt_code<uint16_t>() { return DT_U16; }
template <> constexpr int dt_code<uint8_t>() { return DT_U8; }

// ---------------------------------------------------------------- (a)

template <int K>
struct StreamArgs {
  const void* in;
  void* out;
  long long outer, L, inner;  // elements
  long long nchunks, chunk;
  int anchor, mode;
  double cval;
  int cval_as_input;
  unsigned long long active;  // bit k set: tap k takes part in the chain
  float w[K];
};

template <class T, class D, int K, bool MASK>
__global__ void __launch_bounds__(256) k_stream(const StreamArgs<K> a) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long i4n = a.inner >> 2;
  const long long i4 = tid % i4n;
  const long long rest = tid / i4n;
  const long long c = rest % a.nchunks;
  const long long o = rest / a.nchunks;
  if (o >= a.outer) return;
  const long long l0 = c * a.chunk;
  const long long l1 = min(l0 + a.chunk, a.L);
  const T* in = static_cast<const T*>(a.in) + (o * a.L) * a.inner + i4 * 4;
  D* out = static_cast<D*>(a.out) + (o * a.L) * a.inner + i4 * 4;
  const float cv = fill_value<float>(a.cval, a.cval_as_input, dt_code<T>());

  auto load_row = [&](float (&v)[4], long long coord) {
    long long m = coord;
    if (coord < 0 || coord >= a.L) m = map_coord(coord, a.L, a.mode);
    if (m < 0) {
      v[0] = v[1] = v[2] = v[3] = cv;
    } else {
      load4<T>(in + m * a.inner, v);
    }
  };

  float win[K][4];
#pragma unroll
  for (int k = 0; k < K - 1; ++k) load_row(win[k], l0 - a.anchor + k);

  for (long long l = l0; l < l1; l += K) {
#pragma unroll
    for (int s = 0; s < K; ++s) {
      if (l + s < l1) {
        load_row(win[(s + K - 1) % K], l + s - a.anchor + K - 1);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!MASK || ((a.active >> k) & 1ull)) {
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[v] = fmaf(win[(s + k) % K][v], a.w[k], acc[v]);
          }
        }
        store4<D>(out + (l + s) * a.inner, acc[0], acc[1], acc[2], acc[3]);
      }
    }
  }
}

// ---------------------------------------------------------------- (b)

constexpr int kSlabTY = 32;    // output rows per tile
constexpr int kSlabTX = 128;   // output columns per tile
constexpr int kSlabMaxK = 64;  // longest pass the slab kernel takes

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
  SlabPass py, px;
};

__host__ __device__ inline int pad8(int c) { return c + (c >> 3); }

template <bool SKIP, class At>
__device__ __forceinline__ void chain8(float (&acc)[P], const float* w, int K, int skip, At at) {
  float win[2 * P];
#pragma unroll
  for (int j = 0; j < P; ++j) win[j] = at(j);
  for (int k0 = 0; k0 < K; k0 += P) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P + j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const float t = w[k0 + j];
      if (k0 + j < K && (!SKIP || !skip || t != 0.f)) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fmaf(win[p + j], t, acc[p]);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) win[j] = win[P + j];
  }
}

// Shared layout: wy[64] wx[64] | s_in[RY][RXP] | s_mid[TY][RXP], with
// RX = TX + Kx8 staged columns stored at pad8(column) (one spare word every
// 8) so that lanes reading P-strided columns hit distinct banks.
__host__ __device__ inline int slab_rows(int Ky8) { return kSlabTY + Ky8; }
__host__ __device__ inline int slab_rxp(int Kx8) { return pad8(kSlabTX + Kx8) + 1; }
inline size_t slab_smem(int Ky8, int Kx8, bool has_y) {
  const size_t rxp = slab_rxp(Kx8);
  return sizeof(float) * (2 * kSlabMaxK + slab_rows(Ky8) * rxp + (has_y ? kSlabTY * rxp : 0));
}

template <class T, class D, bool SKIP>
__global__ void __launch_bounds__(256) k_slab(const SlabArgs a) {
  extern __shared__ __align__(16) float sm[];
  float* wy = sm;
  float* wx = sm + kSlabMaxK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < kSlabMaxK; k += blockDim.x) {
    wy[k] = (a.has_y && k < a.py.K) ? a.py.w[k] : 0.f;
    wx[k] = (a.has_x && k < a.px.K) ? a.px.w[k] : 0.f;
  }
  const int Ky8 = a.has_y ? a.py.K8 : 0;
  const int Kx8 = a.has_x ? a.px.K8 : 0;
  const int ay = a.has_y ? a.py.anchor : 0;
  const int ax = a.has_x ? a.px.anchor : 0;
  const int RY = slab_rows(Ky8);
  const int RX = kSlabTX + Kx8;
  const int RXP = slab_rxp(Kx8);
  float* s_in = sm + 2 * kSlabMaxK;
  float* s_mid = s_in + RY * RXP;

  long long bid = blockIdx.x;
  const long long tx = bid % a.tiles_x;
  bid /= a.tiles_x;
  const long long ty = bid % a.tiles_y;
  const long long b = bid / a.tiles_y;
  const long long y0 = ty * kSlabTY, x0 = tx * kSlabTX;
  const T* in = static_cast<const T*>(a.in) + b * a.Y * a.X;
  D* out = static_cast<D*>(a.out) + b * a.Y * a.X;
  const int my = a.has_y ? a.py.mode : CIMX_MODE_NEAREST;
  const int mx = a.has_x ? a.px.mode : CIMX_MODE_NEAREST;
  const float cy = a.has_y ? fill_value<float>(a.py.cval, a.py.cval_as_input, a.py.dt) : 0.f;
  const float cx = a.has_x ? fill_value<float>(a.px.cval, a.px.cval_as_input, a.px.dt) : 0.f;

  // 1. stage the halo'd input tile, boundary modes resolved here
  for (int r = warp; r < RY; r += 8) {
    const long long gy = y0 - ay + r;
    long long myy = gy;
    if (gy < 0 || gy >= a.Y) myy = map_coord(gy, a.Y, my);
    const T* row = in + myy * a.X;
    for (int c = lane; c < RX; c += 32) {
      const long long gx = x0 - ax + c;
      long long mxx = gx;
      if (gx < 0 || gx >= a.X) mxx = map_coord(gx, a.X, mx);
      float v;
      if (myy < 0) v = cy;
      else if (mxx < 0) v = a.has_y ? 0.f : cx;  // x-constant columns are filled after the y pass
      else v = static_cast<float>(row[mxx]);
      s_in[r * RXP + pad8(c)] = v;
    }
  }
  __syncthreads();

  if (a.has_y) {
    // 2. y pass over every staged column
    constexpr int groups = kSlabTY / P;
    for (int item = threadIdx.x; item < RX * groups; item += blockDim.x) {
      const int c = item % RX;
      const int rg = (item / RX) * P;
      const int pc = pad8(c);
      float acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = 0.f;
      chain8<SKIP>(acc, wy, a.py.K, a.py.skip, [&](int q) { return s_in[(rg + q) * RXP + pc]; });
      if (a.has_x) {
        const long long gx = x0 - ax + c;
        const bool xfill = mx == CIMX_MODE_CONSTANT && (gx < 0 || gx >= a.X);
#pragma unroll
        for (int p = 0; p < P; ++p)
          s_mid[(rg + p) * RXP + pc] = xfill ? cx : static_cast<float>(out_cast<D>(acc[p]));
      } else if (c < kSlabTX && x0 + c < a.X) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const long long yy = y0 + rg + p;
          if (yy < a.Y) out[yy * a.X + x0 + c] = out_cast<D>(acc[p]);
        }
      }
    }
    __syncthreads();
  }

  if (a.has_x) {
    // 3. x pass: P consecutive outputs of one row per thread
    constexpr int gpr = kSlabTX / P;
    const float* src = a.has_y ? s_mid : s_in;
    for (int item = threadIdx.x; item < kSlabTY * gpr; item += blockDim.x) {
      const int r = item / gpr;
      const int g = (item % gpr) * P;
      const long long yy = y0 + r;
      if (yy >= a.Y) continue;
      float acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = 0.f;
      const float* row = src + r * RXP;
      chain8<SKIP>(acc, wx, a.px.K, a.px.skip, [&](int q) { return row[pad8(g + q)]; });
      D* orow = out + yy * a.X + x0 + g;
      const long long left = a.X - (x0 + g);
      if (left >= P && ((reinterpret_cast<uintptr_t>(orow) & (sizeof(D) * 4 - 1)) == 0)) {
        store4<D>(orow, acc[0], acc[1], acc[2], acc[3]);
        store4<D>(orow + 4, acc[4], acc[5], acc[6], acc[7]);
      } else {
#pragma unroll
        for (int p = 0; p < P; ++p)
          if (p < left) orow[p] = out_cast<D>(acc[p]);
      }
    }
  }
}

// ----------------------------------------------------------- host side

// (T, D) pairs with fast kernels; all of them use float32 weights.
bool fast_pair(int t, int d) {
  const bool tin = t == DT_U8 || t == DT_U16 || t == DT_F32;
  const bool tout = d == DT_U8 || d == DT_U16 || d == DT_F32;
  return tin && tout && !(t == DT_F32 && d != DT_F32) && !(t == DT_U16 && d == DT_U8);
}

struct Trimmed {
  int K = 0, anchor = 0;
  bool interior_zero = false;
  float w[kSlabMaxK];
};

// Taps rounded to float32; with the elementwise-kernel rule, zero taps at
// both ends are dropped (exact: they never enter the chain).
bool trim(const PassDesc& d, int max_k, Trimmed& t) {
  if (d.w64 || d.K > 4096) return false;
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

// ---- (a) launchers

template <class T, class D, int K>
int launch_stream_k(const PassDesc& d, const Trimmed& t, int tin, const void* in, void* out,
                    cudaStream_t st) {
  StreamArgs<K> a{};
  a.in = in;
  a.out = out;
  a.outer = d.outer;
  a.L = d.L;
  a.inner = d.inner;
  a.anchor = t.anchor;
  a.mode = d.mode;
  a.cval = d.cval;
  a.cval_as_input = d.cval_as_input ? 1 : 0;
  a.active = 0;
  for (int k = 0; k < K; ++k) {
    a.w[k] = t.w[k];
    if (!(d.skip_zero && t.w[k] == 0.f)) a.active |= 1ull << k;
  }
  (void)tin;
  // chunk of L per thread: small enough to fill the GPU a few times over
  const long long lanes = d.outer * (d.inner / 4);
  long long chunk = 64;
  while (chunk > 8 && lanes * ((d.L + chunk - 1) / chunk) < 148LL * 2048 * 2) chunk /= 2;
  a.chunk = chunk;
  a.nchunks = (d.L + chunk - 1) / chunk;
  const long long threads = lanes * a.nchunks;
  const unsigned blocks = (unsigned)((threads + 255) / 256);
  if (t.interior_zero)
    k_stream<T, D, K, true><<<blocks, 256, 0, st>>>(a);
  else
    k_stream<T, D, K, false><<<blocks, 256, 0, st>>>(a);
  return cuda_fail(cudaGetLastError(), "stream pass launch");
}

template <class T, class D>
int launch_stream_td(const PassDesc& d, const Trimmed& t, int tin, const void* in, void* out,
                     cudaStream_t st) {
  switch (t.K) {
    case 3: return launch_stream_k<T, D, 3>(d, t, tin, in, out, st);
    case 5: return launch_stream_k<T, D, 5>(d, t, tin, in, out, st);
    case 7: return launch_stream_k<T, D, 7>(d, t, tin, in, out, st);
    case 9: return launch_stream_k<T, D, 9>(d, t, tin, in, out, st);
    case 13: return launch_stream_k<T, D, 13>(d, t, tin, in, out, st);
    case 17: return launch_stream_k<T, D, 17>(d, t, tin, in, out, st);
    default: return CIMX_FUSED_DECLINED;
  }
}

bool stream_supports(int K) {
  return K == 3 || K == 5 || K == 7 || K == 9 || K == 13 || K == 17;
}

int launch_stream(const PassDesc& d, const Trimmed& t, int tin, const void* in, int tout,
                  void* out, cudaStream_t st) {
#define CIMX_STREAM_CASE(TT, TD, CT, CD) \
  if (tin == TT && tout == TD) return launch_stream_td<CT, CD>(d, t, tin, in, out, st);
  CIMX_STREAM_CASE(DT_U16, DT_F32, uint16_t, float)
  CIMX_STREAM_CASE(DT_U16, DT_U16, uint16_t, uint16_t)
  CIMX_STREAM_CASE(DT_F32, DT_F32, float, float)
  CIMX_STREAM_CASE(DT_U8, DT_F32, uint8_t, float)
  CIMX_STREAM_CASE(DT_U8, DT_U8, uint8_t, uint8_t)
  CIMX_STREAM_CASE(DT_U8, DT_U16, uint8_t, uint16_t)
#undef CIMX_STREAM_CASE
  return CIMX_FUSED_DECLINED;
}

// ---- (b) launchers

void fill_slab_pass(SlabPass& s, const PassDesc& d, const Trimmed& t, int pass_in) {
  s.K = t.K;
  s.K8 = (t.K + P - 1) / P * P;
  s.anchor = t.anchor;
  s.mode = d.mode;
  s.cval = d.cval;
  s.cval_as_input = d.cval_as_input ? 1 : 0;
  s.dt = pass_in;
  s.skip = (d.skip_zero && t.interior_zero) ? 1 : 0;
  std::fill(std::begin(s.w), std::end(s.w), 0.f);
  std::copy(t.w, t.w + t.K, s.w);
}

template <class T, class D>
int launch_slab_td(SlabArgs& a, cudaStream_t st) {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_slab<T, D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_slab<T, D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
  });
  const size_t smem = slab_smem(a.has_y ? a.py.K8 : 0, a.has_x ? a.px.K8 : 0, a.has_y);
  a.tiles_x = (a.X + kSlabTX - 1) / kSlabTX;
  a.tiles_y = (a.Y + kSlabTY - 1) / kSlabTY;
  const long long blocks = a.B * a.tiles_x * a.tiles_y;
  if (blocks == 0) return CIMX_OK;
  const bool skip = (a.has_y && a.py.skip) || (a.has_x && a.px.skip);
  if (skip)
    k_slab<T, D, true><<<(unsigned)blocks, 256, smem, st>>>(a);
  else
    k_slab<T, D, false><<<(unsigned)blocks, 256, smem, st>>>(a);
  return cuda_fail(cudaGetLastError(), "slab launch");
}

int launch_slab(SlabArgs& a, int tin, int tout, cudaStream_t st) {
#define CIMX_SLAB_CASE(TT, TD, CT, CD) \
  if (tin == TT && tout == TD) return launch_slab_td<CT, CD>(a, st);
  CIMX_SLAB_CASE(DT_U16, DT_F32, uint16_t, float)
  CIMX_SLAB_CASE(DT_U16, DT_U16, uint16_t, uint16_t)
  CIMX_SLAB_CASE(DT_F32, DT_F32, float, float)
  CIMX_SLAB_CASE(DT_U8, DT_F32, uint8_t, float)
  CIMX_SLAB_CASE(DT_U8, DT_U8, uint8_t, uint8_t)
  CIMX_SLAB_CASE(DT_U8, DT_U16, uint8_t, uint16_t)
#undef CIMX_SLAB_CASE
  return CIMX_FUSED_DECLINED;
}

}  // namespace

int try_fused(const CimxArray* in, const CimxArray* out, PassDesc* ds, int npasses,
              cudaStream_t st) {
  const int nd = in->ndim;
  const int D = out->dtype;
  if (npasses < 1 || nd < 1) return CIMX_FUSED_DECLINED;
  // passes in strictly ascending axis order, float32 weights
  int prev_axis = -1;
  for (int i = 0; i < npasses; ++i) {
    if (ds[i].axis <= prev_axis || ds[i].w64) return CIMX_FUSED_DECLINED;
    prev_axis = ds[i].axis;
  }

  // split into leading passes (streamed) and the passes on the last two axes (slab)
  const int ylast = nd >= 2 ? nd - 2 : -1;
  std::vector<int> lead, tail;
  for (int i = 0; i < npasses; ++i) (ds[i].axis < ylast ? lead : tail).push_back(i);

  std::vector<Trimmed> tr(npasses);
  for (int n = 0; n < (int)lead.size(); ++n) {
    const int i = lead[n];
    const int tin = n == 0 ? in->dtype : D;
    if (!trim(ds[i], 17, tr[i]) || !stream_supports(tr[i].K)) return CIMX_FUSED_DECLINED;
    if (!fast_pair(tin, D) || ds[i].inner % 4 != 0) return CIMX_FUSED_DECLINED;
  }
  const int tail_in = lead.empty() ? in->dtype : D;
  if (!tail.empty()) {
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
    rc = launch_stream(ds[i], tr[i], tsrc, src, D, dst, st);
    if (rc != CIMX_OK) break;
    src = dst;
    tsrc = D;
  }
  if (rc == CIMX_OK && !tail.empty()) {
    SlabArgs a{};
    a.in = src;
    a.out = dst_of(j++);
    a.X = in->shape[nd - 1];
    a.Y = nd >= 2 ? in->shape[nd - 2] : 1;
    a.B = n / std::max<int64_t>(1, a.X * a.Y);
    if (a.X * a.Y == 0) a.B = 0;
    int pass_in = tsrc;
    for (int i : tail) {
      const bool is_x = ds[i].axis == nd - 1;
      SlabPass& sp = is_x ? a.px : a.py;
      fill_slab_pass(sp, ds[i], tr[i], pass_in);
      (is_x ? a.has_x : a.has_y) = 1;
      pass_in = D;
    }
    rc = launch_slab(a, tsrc, D, st);
  }
  scratch_free(temp, tbytes, st);
  // a decline after a partial run cannot happen: every check above ran first
  return rc;
}

}  // namespace cimx
