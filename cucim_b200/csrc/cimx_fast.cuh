// cimx_fast.cuh — kernel templates of the plain (exact float32) fast path.
//
// (a) k_stream: one pass along a strided axis of the view (outer, L, inner).
//     Each thread owns 4 consecutive inner positions (one 4-wide vector
//     load/store per row) and walks a chunk of L. The last K rows, plus PF
//     rows prefetched ahead, live in a register ring indexed at compile time:
//     every input row is read once per chunk, loads are issued PF rows before
//     they are used, and every tap is a constant-bank FMA operand.
// (b) k_slab: the last two axes (y, x) of a (B, Y, X) view in one launch. One
//     TMA bulk tensor copy brings the halo'd input tile into shared memory
//     (zero-filled outside the array); tiles touching the border get their
//     halo rewritten with the boundary mode's values. The y pass writes its
//     result, rounded through the output dtype as cuCIM's ping-pong does, to a
//     second shared tile and the x pass stores the outputs: the intermediate
//     never reaches HBM.
//
// Every output is the same fused multiply-add chain as in the generic
// kernels (taps ascending, float32 FMA from +0, cast<D>()), so a pass list
// gives bit-identical results whichever kernels run it.
#pragma once

#include <algorithm>
#include <cstring>
#include <mutex>

#include "cimx_common.cuh"
#include "cimx_fused.h"
#include "cimx_tma.cuh"

namespace cimx {
namespace fast {

constexpr int P = 8;  // consecutive outputs per thread in the slab kernel
constexpr int kMaxSmem = 227 * 1024;

// ------------------------------------------------------------ vector I/O

template <class T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<uint16_t> { using type = ushort4; };
template <> struct Vec4<uint8_t> { using type = uchar4; };

// Exact float value of an unsigned integer below 2^23 without the conversion
// unit: the integer placed in the mantissa of 2^23, minus 2^23.
template <class T>
__device__ __forceinline__ float exact_float(T v) {
  if constexpr (sizeof(T) == 4) {
    return static_cast<float>(v);
  } else {
    return __fsub_rn(__uint_as_float(0x4B000000u | static_cast<uint32_t>(v)), 8388608.0f);
  }
}

// cast<D>(a) of an intermediate that stays on chip, as the float the next
// pass reads (out_cast writes the narrowing conversion out explicitly, so
// widening its result again keeps the narrow value)
template <class D>
__device__ __forceinline__ float narrow_float(float a) {
  if constexpr (sizeof(D) == 4) return a;
  else return exact_float(out_cast<D>(a));
}

// cast<D>(a) as stored
template <class D>
__device__ __forceinline__ D narrow_cast(float a) {
  return out_cast<D>(a);
}

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
  q.x = narrow_cast<D>(a);
  q.y = narrow_cast<D>(b);
  q.z = narrow_cast<D>(c);
  q.w = narrow_cast<D>(d);
  *reinterpret_cast<typename Vec4<D>::type*>(p) = q;
}

template <class T> constexpr int dt_code();
template <> constexpr int dt_code<float>() { return DT_F32; }
template <> constexpr int dt_code<uint16_t>() { return DT_U16; }
template <> constexpr int dt_code<uint8_t>() { return DT_U8; }

// ------------------------------------------------------------- helpers

// Two independent IEEE float32 FMAs (round to nearest) in one instruction:
// d.x = fma(a.x, b.x, c.x), d.y = fma(a.y, b.y, c.y), bit-identical to fmaf.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{.reg .b64 ra, rb, rc, rd;\n"
      " mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n mov.b64 rc, {%6, %7};\n"
      " fma.rn.f32x2 rd, ra, rb, rc;\n"
      " mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <class T>
__device__ __forceinline__ void cp_async_vec4(T* dst, const T* src) {
  if constexpr (sizeof(T) == 4) cp_async16(dst, src);
  else if constexpr (sizeof(T) == 2) cp_async8(dst, src);
  else cp_async4(dst, src);
}


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

// rows in flight per thread: a multiple of K with at least 8 rows
template <int K> constexpr int stream_depth() { return K * ((8 + K - 1) / K); }
template <class T, int K> constexpr int stream_smem() {
  return stream_depth<K>() * 256 * 4 * (int)sizeof(T);
}

template <class T, class D, int K, bool MASK>
__global__ void __launch_bounds__(256) k_stream(const StreamArgs<K> a) {
  constexpr int DEPTH = stream_depth<K>();
  extern __shared__ __align__(16) unsigned char sm_stream[];
  // this thread's prefetch slots: slot d at pre + d * 256 * 4
  T* pre = reinterpret_cast<T*>(sm_stream) + threadIdx.x * 4;
  // grid = (inner/4 in blocks of 256, chunks of L, outer); outer beyond the
  // grid's z extent is visited by striding
  const long long i4 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i4 >= (a.inner >> 2)) return;  // no barrier in this kernel
  const long long l0 = (long long)blockIdx.y * a.chunk;
  for (long long o = blockIdx.z; o < a.outer; o += gridDim.z) {
  const long long l1 = min(l0 + a.chunk, a.L);
  const T* in = static_cast<const T*>(a.in) + (o * a.L) * a.inner + i4 * 4;
  D* out = static_cast<D*>(a.out) + (o * a.L) * a.inner + i4 * 4;
  const float cv = fill_value<float>(a.cval, a.cval_as_input, dt_code<T>());

  auto mapped = [&](long long coord) -> long long {
    return (coord < 0 || coord >= a.L) ? map_coord(coord, a.L, a.mode) : coord;
  };
  auto load_row = [&](float (&v)[4], long long coord) {
    const long long m = mapped(coord);
    if (m < 0) {
      v[0] = v[1] = v[2] = v[3] = cv;
    } else {
      load4<T>(in + m * a.inner, v);
    }
  };
  // input row consumed at step s (output l0 + s): the newest row of its window
  auto row_of_step = [&](long long s) { return l0 + s - a.anchor + K - 1; };
  auto issue = [&](int slot, long long s) {
    const long long m = mapped(row_of_step(s));
    if (m >= 0) cp_async_vec4<T>(pre + slot * 1024, in + m * a.inner);
    cp_commit();
  };

  // window ring: slot j holds input row (l0 - anchor + j) modulo K. Prefetch
  // slot d holds the row consumed at step d modulo DEPTH; the slot refilled at
  // step s is the one consumed at step s - 1, so no copy can land on a slot
  // whose shared load is still in flight.
  float win[K][4];
#pragma unroll
  for (int k = 0; k < K - 1; ++k) load_row(win[k], l0 - a.anchor + k);
#pragma unroll
  for (int d = 0; d < DEPTH - 1; ++d) issue(d, d);

  const long long n = l1 - l0;
  for (long long s0 = 0; s0 < n; s0 += DEPTH) {
#pragma unroll
    for (int u = 0; u < DEPTH; ++u) {
      const long long s = s0 + u;
      if (s < n) {
        issue((u + DEPTH - 1) % DEPTH, s + DEPTH - 1);
        cp_wait<DEPTH - 1>();
        float* v = win[(u + K - 1) % K];
        const long long m = mapped(row_of_step(s));
        if (m < 0) {
          v[0] = v[1] = v[2] = v[3] = cv;
        } else {
          const typename Vec4<T>::type q =
              *reinterpret_cast<const typename Vec4<T>::type*>(pre + u * 1024);
          v[0] = static_cast<float>(q.x);
          v[1] = static_cast<float>(q.y);
          v[2] = static_cast<float>(q.z);
          v[3] = static_cast<float>(q.w);
        }
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!MASK || ((a.active >> k) & 1ull)) {
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[e] = fmaf(win[(u + k) % K][e], a.w[k], acc[e]);
          }
        }
        store4<D>(out + (l0 + s) * a.inner, acc[0], acc[1], acc[2], acc[3]);
      }
    }
  }
  cp_wait<0>();
  }
}

template <class T, class D, int K>
int launch_stream_k(const PassDesc& d, const float* w, int anchor, bool interior_zero,
                    const void* in, void* out, cudaStream_t st) {
  StreamArgs<K> a{};
  a.in = in;
  a.out = out;
  a.outer = d.outer;
  a.L = d.L;
  a.inner = d.inner;
  a.anchor = anchor;
  a.mode = d.mode;
  a.cval = d.cval;
  a.cval_as_input = d.cval_as_input ? 1 : 0;
  a.active = 0;
  for (int k = 0; k < K; ++k) {
    a.w[k] = w[k];
    if (!(d.skip_zero && w[k] == 0.f)) a.active |= 1ull << k;
  }
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_stream<T, D, K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_stream<T, D, K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
  });
  // chunk of L per thread: small enough to fill the GPU a few times over
  const long long lanes = d.outer * (d.inner / 4);
  long long chunk = 64;
  while (chunk > 8 && lanes * ((d.L + chunk - 1) / chunk) < 148LL * 2048 * 2) chunk /= 2;
  a.chunk = chunk;
  a.nchunks = (d.L + chunk - 1) / chunk;
  if (a.nchunks > 65535) return CIMX_FUSED_DECLINED;
  const dim3 grid((unsigned)((d.inner / 4 + 255) / 256), (unsigned)a.nchunks,
                  (unsigned)std::min<long long>(d.outer, 65535));
  constexpr int smem = stream_smem<T, K>();
  if (interior_zero)
    k_stream<T, D, K, true><<<grid, 256, smem, st>>>(a);
  else
    k_stream<T, D, K, false><<<grid, 256, smem, st>>>(a);
  return cuda_fail(cudaGetLastError(), "stream pass launch");
}

template <class T, class D>
int launch_stream_td(const PassDesc& d, const float* w, int K, int anchor, bool interior_zero,
                     const void* in, void* out, cudaStream_t st) {
  switch (K) {
    case 3: return launch_stream_k<T, D, 3>(d, w, anchor, interior_zero, in, out, st);
    case 5: return launch_stream_k<T, D, 5>(d, w, anchor, interior_zero, in, out, st);
    case 7: return launch_stream_k<T, D, 7>(d, w, anchor, interior_zero, in, out, st);
    case 9: return launch_stream_k<T, D, 9>(d, w, anchor, interior_zero, in, out, st);
    case 11: return launch_stream_k<T, D, 11>(d, w, anchor, interior_zero, in, out, st);
    case 13: return launch_stream_k<T, D, 13>(d, w, anchor, interior_zero, in, out, st);
    case 15: return launch_stream_k<T, D, 15>(d, w, anchor, interior_zero, in, out, st);
    case 17: return launch_stream_k<T, D, 17>(d, w, anchor, interior_zero, in, out, st);
    default: return CIMX_FUSED_DECLINED;
  }
}

// ---------------------------------------------------------------- (b)

constexpr int kSlabTY = 32;    // output rows per tile
constexpr int kSlabTX = 128;   // output columns per tile

__host__ __device__ constexpr int pad8(int c) { return c + (c >> 3); }

// Compile-time tile geometry for taps bucket KB (both passes have K8 <= KB).
//
// Staged region: RY rows x RX columns starting at (y0 - ay, x0 - ax). Column
// pairs (2m, 2m+1) of the y pass are aligned in the buffer the y pass reads:
// the TMA tile (float input; its start column is 16-byte aligned, so the
// staged region starts at an offset `off` and pairs are taken from
// off - sh, sh = off & 1) or the converted tile s_in (other inputs, sh = 0).
// Shared memory:
//   mbarrier | y taps, x taps as (t, t) pairs |
//   float input: raw x 2 (BY x BX floats each; the next slab's tile loads
//                while this one is computed) | s_mid (TY/2 row pairs x RXQ float2)
//   other input: s_in (RY x RXS floats) | s_mid | raw (T; loads while the
//                passes run) for taps buckets up to 48, else
//                s_in | union { raw (T), s_mid }
template <class T, int KB>
struct Geom {
  static constexpr bool F32 = sizeof(T) == 4;
  static constexpr int RY = kSlabTY + KB;         // staged rows
  static constexpr int RX = kSlabTX + KB;         // staged columns (even)
  static constexpr int NPAIR = RX / 2 + 1;        // y-pass column pairs (one spare for sh)
  static constexpr int RXS = RX + 2;              // s_in row stride (floats)
  static constexpr int RXQ = pad8(RX + 2);        // s_mid row-pair stride (float2)
  static constexpr int VE = 16 / (int)sizeof(T);  // elements per 16 bytes
  static constexpr int BX = (RX + VE + VE - 1) / VE * VE;  // TMA box width >= RX + off + 1
  static constexpr int BY = RY;                   // TMA box height
  static constexpr int RAW = BX * BY * (int)sizeof(T);
  static constexpr int MID = (kSlabTY / 2) * RXQ * 8;
  static constexpr int OFF_W = 128;
  static constexpr int RAWP = (RAW + 127) / 128 * 128;
  // one TMA buffer: measured faster than two (two cost resident CTAs per SM;
  // with two, the 17-tap gaussian of the 512 x 1024 x 1024 stack took
  // 3.0 ms instead of 2.2 ms)
  static constexpr int NBUF = 1;
  static constexpr int OFF_A = OFF_W + 2 * KB * 8;  // raw (f32) or s_in
  static constexpr int SZ_A = F32 ? NBUF * RAWP : RY * RXS * 4;
  static constexpr int OFF_B = (OFF_A + SZ_A + 127) / 128 * 128;  // s_mid (f32) or union
  // threads: enough for every y-pass item (NPAIR column pairs x TY/P row
  // groups) in one round; the x pass has TY/2 x TX/P = 256 items
  static constexpr int NT = ((NPAIR * (kSlabTY / P) + 31) / 32) * 32;
  static constexpr int NW = NT / 32;
  // resident CTAs per SM asked of the compiler (registers per thread):
  // three up to 320 threads (64 registers), two beyond (three would leave
  // 56 registers and spill)
  static constexpr int MINB = NT <= 320 ? 3 : 2;
  // other inputs: the raw tile gets a buffer of its own (after s_mid) where
  // that keeps MINB CTAs per SM by shared memory (taps buckets up to 48), so
  // that the next slab's tile loads while this one is computed; else it
  // shares its buffer with s_mid
  static constexpr int SMEM_U = OFF_B + (RAW > MID ? RAW : MID);
  static constexpr int OFF_R = (OFF_B + MID + 127) / 128 * 128;
  static constexpr int SMEM_S = OFF_R + RAWP;
  static constexpr int fit(int s) { return (228 * 1024) / (s + 1024); }
  static constexpr bool SEP = !F32 && fit(SMEM_S) >= (fit(SMEM_U) < MINB ? fit(SMEM_U) : MINB);
  static constexpr int SMEM = F32 ? OFF_B + MID : (SEP ? SMEM_S : SMEM_U);
};

__device__ __forceinline__ long long floor_div(long long a, long long b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// Two float32 lanes in one 64-bit register (x in the low half).
using f2 = unsigned long long;

__device__ __forceinline__ f2 pack2(float x, float y) {
  return (static_cast<f2>(__float_as_uint(y)) << 32) | __float_as_uint(x);
}
__device__ __forceinline__ float lo2(f2 v) { return __uint_as_float(static_cast<unsigned>(v)); }
__device__ __forceinline__ float hi2(f2 v) {
  return __uint_as_float(static_cast<unsigned>(v >> 32));
}

// d = fma(a, b, c) on both lanes, each an IEEE float32 FMA rounded to nearest
// (bit-identical to fmaf on each lane).
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// One fused multiply-add chain per lane for P outputs: acc[p] += x[p+k] w[k],
// k ascending. `at(qb, j)` returns the staged input pair at window offset
// qb + j, where qb is a multiple of P and j < P is a compile-time constant
// (so the accessor computes its address once per chunk); w2 holds (t, t)
// pairs. Full chunks of P taps run without guards, two chunks per iteration
// so the window halves swap roles without register moves.
template <class At>
__device__ __forceinline__ void chain2(f2 (&acc)[P], const f2* w2, int K, int skip, At at) {
  f2 win[2 * P];
#pragma unroll
  for (int j = 0; j < P; ++j) win[j] = at(0, j);
  int k0 = 0;
  if (!skip) {
    for (; k0 + 2 * P <= K; k0 += 2 * P) {
#pragma unroll
      for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P, j);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const f2 t = w2[k0 + j];
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma2(win[p + j], t, acc[p]);
      }
#pragma unroll
      for (int j = 0; j < P; ++j) win[j] = at(k0 + 2 * P, j);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const f2 t = w2[k0 + P + j];
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma2(win[(P + p + j) % (2 * P)], t, acc[p]);
      }
    }
    if (k0 + P <= K) {
#pragma unroll
      for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P, j);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const f2 t = w2[k0 + j];
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma2(win[p + j], t, acc[p]);
      }
#pragma unroll
      for (int j = 0; j < P; ++j) win[j] = win[P + j];
      k0 += P;
    }
  }
  if (!skip && k0 < K) {
    // last partial chunk: r = K - k0 taps, unrolled per r without guards
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P, j);
    const int r = K - k0;
#define CIMX_TAIL(R)                                                         \
  case R:                                                                    \
    _Pragma("unroll") for (int j = 0; j < R; ++j) {                          \
      const f2 t = w2[k0 + j];                                               \
      _Pragma("unroll") for (int p = 0; p < P; ++p) acc[p] = fma2(win[p + j], t, acc[p]); \
    }                                                                        \
    break;
    switch (r) {
      CIMX_TAIL(1) CIMX_TAIL(2) CIMX_TAIL(3) CIMX_TAIL(4) CIMX_TAIL(5) CIMX_TAIL(6)
      CIMX_TAIL(7)
      default: break;
    }
#undef CIMX_TAIL
    return;
  }
  // every chunk with guards when zero taps must be skipped
  for (; k0 < K; k0 += P) {
#pragma unroll
    for (int j = 0; j < P; ++j) win[P + j] = at(k0 + P, j);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const f2 t = w2[k0 + j];
      if (k0 + j < K && (!skip || lo2(t) != 0.f)) {
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = fma2(win[p + j], t, acc[p]);
      }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) win[j] = win[P + j];
  }
}

// Value of the staged element (gy, gx) of the slab, boundary modes applied.
template <class T>
__device__ __forceinline__ float staged_value(const T* in, long long gy, long long gx,
                                              const SlabArgs& a, int my, int mx, float cy) {
  long long yy = gy, xx = gx;
  if (gy < 0 || gy >= a.Y) yy = map_coord_near(gy, a.Y, my);
  if (gx < 0 || gx >= a.X) xx = map_coord_near(gx, a.X, mx);
  if (yy < 0) return cy;
  if (xx < 0) return 0.f;  // x-constant columns are replaced after the y pass
  return static_cast<float>(in[yy * a.X + xx]);
}

template <class T, class D, int KB, bool TMA>
__global__ void __launch_bounds__(Geom<T, KB>::NT, Geom<T, KB>::MINB) k_slab(const __grid_constant__ CUtensorMap map,
                                               const SlabArgs a) {
  using G = Geom<T, KB>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // bar[0], bar[1]: one per raw buffer
  f2* wy = reinterpret_cast<f2*>(smem + G::OFF_W);
  f2* wx = wy + KB;
  T* raw0 = reinterpret_cast<T*>(smem + (G::F32 ? G::OFF_A : (G::SEP ? G::OFF_R : G::OFF_B)));
  float* s_in = reinterpret_cast<float*>(smem + G::OFF_A);  // non-float inputs only
  f2* s_mid = reinterpret_cast<f2*>(smem + G::OFF_B);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  if (TMA && threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_fence_init();
  }
  for (int k = threadIdx.x; k < KB; k += blockDim.x) {
    const float ty_ = k < a.py.K ? a.py.w[k] : 0.f;
    const float tx_ = (a.has_x && k < a.px.K) ? a.px.w[k] : 0.f;
    wy[k] = pack2(ty_, ty_);
    wx[k] = pack2(tx_, tx_);
  }
  __syncthreads();

  const int ay = a.py.anchor;
  const int ax = a.has_x ? a.px.anchor : 0;
  const int my = a.py.mode;
  const int mx = a.has_x ? a.px.mode : CIMX_MODE_NEAREST;
  const float cy = fill_value<float>(a.py.cval, a.py.cval_as_input, a.py.dt);
  const float cx = a.has_x ? fill_value<float>(a.px.cval, a.px.cval_as_input, a.px.dt) : 0.f;
  // grid = (tiles_x, tiles_y, slabs); slabs beyond the grid's z extent are
  // visited by striding, the mbarrier phase flipping once per slab
  const long long y0 = (long long)blockIdx.y * kSlabTY, x0 = (long long)blockIdx.x * kSlabTX;
  const long long ys = y0 - ay, xst = x0 - ax;
  const long long xs = floor_div(xst, G::VE) * G::VE;  // 16-byte aligned TMA start column
  const int off = static_cast<int>(xst - xs);
  // staged columns [cl, cr) and rows [rl, rr) lie inside the array
  auto clampi = [](long long v, long long lo, long long hi) {
    return static_cast<int>(v < lo ? lo : (v > hi ? hi : v));
  };
  const int cl = clampi(-xst, 0, G::RX);
  const int cr = clampi(a.X - xst, cl, G::RX);
  const int rl = clampi(-ys, 0, G::RY);
  const int rr = clampi(a.Y - ys, rl, G::RY);
  // other inputs with a raw buffer of their own: the y pass reads element
  // pairs of the raw tile and the conversion to s_in is skipped, for every
  // tile whose staged elements outside the array can be patched in place
  // with elements of the array: all of them but those with rows outside
  // under a constant y mode (whose fill value need not fit in T); x-constant
  // columns are replaced after the y pass (the same for every thread of the
  // CTA)
  const bool direct = !G::F32 && G::SEP && TMA &&
                      ((rl == 0 && rr == G::RY) || my != CIMX_MODE_CONSTANT);
  // float input, or a direct tile: pairs are read from the TMA tile starting
  // at column off - sh (an even column)
  const int sh = ((TMA && G::F32) || direct) ? (off & 1) : 0;
  // float input: two TMA buffers; the copy for the next slab is issued before
  // the current slab is computed. Other inputs: one buffer.
  constexpr int NBUF = G::NBUF;
  auto issue = [&](long long bb, int k) {
    fence_proxy_async_smem();  // earlier reads of this buffer came first
    mbar_expect_tx(bar + k, G::RAW);
    tma_load_3d(reinterpret_cast<unsigned char*>(raw0) + k * G::RAWP, &map, bar + k,
                static_cast<int>(xs), static_cast<int>(ys), static_cast<int>(bb));
  };
  // float input, one buffer: the y pass is the last reader of the raw tile
  // (the x pass reads s_mid), so the next slab's tile is issued right after
  // it and lands while the x pass runs. The same holds for other inputs with
  // a raw buffer of their own (the conversion to s_in, or on a direct tile
  // the y pass, is the last reader).
  constexpr bool kEarly = (G::F32 || G::SEP) && NBUF == 1;
  if (TMA && (NBUF == 2 || kEarly) && threadIdx.x == 0 && blockIdx.z < a.B) issue(blockIdx.z, 0);
  long long it = 0;
  for (long long b = blockIdx.z; b < a.B; b += gridDim.z, ++it) {
  const T* in = static_cast<const T*>(a.in) + b * a.Y * a.X;
  D* out = static_cast<D*>(a.out) + b * a.Y * a.X;
  const int kb = static_cast<int>(it % NBUF);
  T* raw = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(raw0) + kb * G::RAWP);

  // 1. stage the tile
  if (TMA) {
    // thread 0 prefetches the next slab's tile (double buffering, float input)
    // and waits (bounded) for this one; the others wait at the barrier, where
    // they issue no instructions
    int ok = 1;
    if (threadIdx.x == 0) {
      if (NBUF == 2 && b + gridDim.z < a.B) issue(b + gridDim.z, 1 - kb);
      if (NBUF == 1 && !kEarly) issue(b, 0);
      const uint32_t parity = static_cast<uint32_t>((it / NBUF) & 1);
      ok = mbar_wait(bar + kb, parity, a.status) ? 1 : 0;
    }
    if (!__syncthreads_and(ok)) return;
  }
  if ((G::F32 && TMA) || direct) {
    // the y pass reads the raw tile: rewrite only the staged elements that
    // lie outside the array with their boundary-mode values, as elements of T
    // (the same test for every thread of the CTA, so the barrier inside holds)
    if (!(rl == 0 && rr == G::RY && cl == 0 && cr == G::RX)) {
      T* rawf = raw;
      // Only the staged elements outside the array are visited, spread over
      // every thread of the CTA.
      // 1. rows inside the array: a column outside takes the value of the
      //    column it maps to, read from the staged tile when that column is
      //    staged (always, for overhangs shorter than the row), else from HBM;
      //    x-constant columns hold 0 until the y pass replaces them
      const int nleft = cl, nout = cl + (G::RX - cr);
      const int n1 = (rr - rl) * nout;
      for (int t = threadIdx.x; t < n1; t += G::NT) {
        const int r = rl + t / nout, j = t % nout;
        const int c = j < nleft ? j : cr + (j - nleft);
        T* row = rawf + r * G::BX + off;
        const long long xm = map_coord_near(xst + c, a.X, mx);
        T v = T(0);
        if (xm >= 0) {
          const long long sc = xm - xst;
          if (sc >= cl && sc < cr) {
            v = row[sc];
          } else {
            v = in[(ys + r) * a.X + xm];
          }
        }
        row[c] = v;
      }
      __syncthreads();
      // 2. rows outside the array: the fill value (constant mode), or a copy
      //    of the (now complete) staged row they map to, else from HBM
      const int nrow_out = G::RY - (rr - rl);
      const int n2 = nrow_out * G::RX;
      for (int t = threadIdx.x; t < n2; t += G::NT) {
        const int q = t / G::RX, c = t % G::RX;
        const int r = q < rl ? q : rr + (q - rl);
        T* row = rawf + r * G::BX + off;
        const long long ym = map_coord_near(ys + r, a.Y, my);
        const long long sr = ym - ys;
        T v;
        if (ym < 0) {
          // float input only: a direct tile has no y-constant rows outside
          if constexpr (G::F32) v = cy;
          else v = T(0);
        } else if (sr >= rl && sr < rr) {
          v = rawf[sr * G::BX + off + c];
        } else {
          // an element of the array (exact in float), or 0 in an x-constant column
          v = static_cast<T>(staged_value<T>(in, ys + r, xst + c, a, my, mx, cy));
        }
        row[c] = v;
      }
    }
  } else {
    // convert to float into the staging buffer at column c (pairs aligned)
    float* dst = G::F32 ? reinterpret_cast<float*>(raw) : s_in;
    const int stride = G::F32 ? G::BX : G::RXS;
    for (int r = warp; r < G::RY; r += G::NW) {
      const bool row_in = r >= rl && r < rr;
      for (int c = lane; c < G::RX; c += 32) {
        float v;
        if (TMA && row_in && c >= cl && c < cr) v = static_cast<float>(raw[r * G::BX + off + c]);
        else v = staged_value<T>(in, ys + r, xst + c, a, my, mx, cy);
        dst[r * stride + c] = v;
      }
    }
  }
  __syncthreads();

  // 2. y pass: one column pair x P rows per item, written to s_mid as row
  //    pairs (rounded through D); column index e = staged column + sh
  {
    const float* src = G::F32 ? reinterpret_cast<const float*>(raw) : s_in;
    const int stride = G::F32 ? G::BX : G::RXS;
    const int soff = (G::F32 && TMA) ? off - sh : 0;
    const int npair = (G::RX + sh + 1) / 2;
    constexpr int groups = kSlabTY / P;
    for (int item = threadIdx.x; item < G::NPAIR * groups; item += blockDim.x) {
      const int m = item % G::NPAIR;
      const int rg = (item / G::NPAIR) * P;
      if (m >= npair) continue;
      const int e = 2 * m;
      f2 acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = 0ull;
      if constexpr (!G::F32 && G::SEP && TMA) {
        if (direct) {
          // the pair (e - sh, e - sh + 1) of staged columns, one aligned
          // 2-element load from the raw tile, widened exactly
          using Pair = typename std::conditional<sizeof(T) == 2, uint32_t, uint16_t>::type;
          constexpr int kBits = 8 * static_cast<int>(sizeof(T));
          const Pair* colr = reinterpret_cast<const Pair*>(raw + rg * G::BX + off - sh + e);
          chain2(acc, wy, a.py.K, a.py.skip, [&](int qb, int j) {
            const uint32_t w = colr[(qb + j) * (G::BX / 2)];
            return pack2(exact_float<T>(static_cast<T>(w & ((1u << kBits) - 1))),
                         exact_float<T>(static_cast<T>(w >> kBits)));
          });
        }
      }
      if (!direct) {
        const f2* col = reinterpret_cast<const f2*>(src + rg * stride + soff + e);
        chain2(acc, wy, a.py.K, a.py.skip,
               [&](int qb, int j) { return col[(qb + j) * (stride / 2)]; });
      }
      const long long gx = xst + e - sh;
      if (a.has_x) {
        const bool f0 = mx == CIMX_MODE_CONSTANT && (gx < 0 || gx >= a.X);
        const bool f1 = mx == CIMX_MODE_CONSTANT && (gx + 1 < 0 || gx + 1 >= a.X);
        f2* d0 = s_mid + (rg / 2) * G::RXQ + pad8(e);
        f2* d1 = s_mid + (rg / 2) * G::RXQ + pad8(e + 1);
#pragma unroll
        for (int p = 0; p < P; p += 2) {
          const float a0 = f0 ? cx : narrow_float<D>(lo2(acc[p]));
          const float b0 = f0 ? cx : narrow_float<D>(lo2(acc[p + 1]));
          const float a1 = f1 ? cx : narrow_float<D>(hi2(acc[p]));
          const float b1 = f1 ? cx : narrow_float<D>(hi2(acc[p + 1]));
          d0[(p / 2) * G::RXQ] = pack2(a0, b0);
          d1[(p / 2) * G::RXQ] = pack2(a1, b1);
        }
      } else {
        // y only: store straight to the output
        const long long c0 = e - sh;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const long long yy = y0 + rg + p;
          if (yy >= a.Y) continue;
          if (c0 >= 0 && c0 < kSlabTX && x0 + c0 < a.X)
            out[yy * a.X + x0 + c0] = narrow_cast<D>(lo2(acc[p]));
          if (c0 + 1 >= 0 && c0 + 1 < kSlabTX && x0 + c0 + 1 < a.X)
            out[yy * a.X + x0 + c0 + 1] = narrow_cast<D>(hi2(acc[p]));
        }
      }
    }
  }

  if (a.has_x) {
    __syncthreads();
    // every read of the raw tile is done: its next slab may land now
    if (TMA && kEarly && threadIdx.x == 0 && b + gridDim.z < a.B) issue(b + gridDim.z, 0);
    // 3. x pass: one row pair x P consecutive outputs per item; output column
    //    g + q reads s_mid column g + q + sh, and since g is a multiple of 8,
    //    pad8(g + q + sh) = pad8(g) + pad8(q + sh)
    constexpr int gpr = kSlabTX / P;
    for (int item = threadIdx.x; item < (kSlabTY / 2) * gpr; item += blockDim.x) {
      const int rp = item / gpr;
      const int g = (item % gpr) * P;
      f2 acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = 0ull;
      const f2* row = s_mid + rp * G::RXQ + pad8(g);
      if (sh)
        chain2(acc, wx, a.px.K, a.px.skip,
               [&](int qb, int j) { return row[pad8(qb) + (j + 1) + ((j + 1) >> 3)]; });
      else
        chain2(acc, wx, a.px.K, a.px.skip, [&](int qb, int j) { return row[pad8(qb) + j]; });
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long yy = y0 + 2 * rp + h;
        if (yy >= a.Y) continue;
        D* orow = out + yy * a.X + x0 + g;
        const long long left = a.X - (x0 + g);
        float v[P];
#pragma unroll
        for (int p = 0; p < P; ++p) v[p] = h ? hi2(acc[p]) : lo2(acc[p]);
        if (left >= P && ((reinterpret_cast<uintptr_t>(orow) & (sizeof(D) * 4 - 1)) == 0)) {
          store4<D>(orow, v[0], v[1], v[2], v[3]);
          store4<D>(orow + 4, v[4], v[5], v[6], v[7]);
        } else {
#pragma unroll
          for (int p = 0; p < P; ++p)
            if (p < left) orow[p] = narrow_cast<D>(v[p]);
        }
      }
    }
  }
  // shared buffers are reused by the next slab. With a raw buffer of its own
  // (float input, or SEP), TMA and an x pass, the barrier after the next
  // slab's tile wait already orders this slab's x pass (the last reader of
  // s_mid) before the next y pass, and this slab's y pass (the last reader of
  // s_in) before the next conversion: no barrier here
  if (!(TMA && kEarly && a.has_x)) __syncthreads();
  if (TMA && kEarly && !a.has_x && threadIdx.x == 0 && b + gridDim.z < a.B)
    issue(b + gridDim.z, 0);
  }
}

template <class T, class D, int KB>
int launch_slab_kb(SlabArgs& a, cudaStream_t st) {
  using G = Geom<T, KB>;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_slab<T, D, KB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
    cudaFuncSetAttribute(k_slab<T, D, KB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
  });
  a.tiles_x = (a.X + kSlabTX - 1) / kSlabTX;
  a.tiles_y = (a.Y + kSlabTY - 1) / kSlabTY;
  const long long blocks = a.B * a.tiles_x * a.tiles_y;
  if (blocks == 0) return CIMX_OK;
  a.status = device_status_word();
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const bool tma = make_tensor_map_3d(&map, a.in, dt_code<T>(), a.X, a.Y, a.B, G::BX, G::BY);
  // without TMA a float tile is staged by plain loads into the raw buffer
  if (a.tiles_y > 65535) return CIMX_FUSED_DECLINED;
  // enough CTAs to fill the GPU several times over; each walks a stride of
  // slabs so that it can load the next slab's tile while computing the
  // current one (float input, or other inputs with a raw buffer of their
  // own: about four slabs per CTA, at least ~12 CTAs per SM)
  const long long per_slab = a.tiles_x * a.tiles_y;
  constexpr bool kWalk = G::F32 || G::SEP;
  long long zs;
  if (G::NBUF == 2)
    zs = std::max<long long>(
        1, std::min<long long>({a.B, 65535LL, (148LL * 8 + per_slab - 1) / per_slab}));
  else if (kWalk && tma && a.span > 0)  // a tuned or forced span (any span is exact)
    zs = std::max<long long>(1, std::min<long long>({a.B, 65535LL, (a.B + a.span - 1) / a.span}));
  else if (kWalk && tma)
    zs = std::max<long long>(1, std::min<long long>({a.B, 65535LL,
                                                     std::max<long long>((a.B + 3) / 4,
                                                     (148LL * 12 + per_slab - 1) / per_slab)}));
  else
    zs = std::min<long long>(a.B, 65535LL);
  const dim3 grid((unsigned)a.tiles_x, (unsigned)a.tiles_y, (unsigned)zs);
  if (tma)
    k_slab<T, D, KB, true><<<grid, G::NT, G::SMEM, st>>>(map, a);
  else
    k_slab<T, D, KB, false><<<grid, G::NT, G::SMEM, st>>>(map, a);
  return cuda_fail(cudaGetLastError(), "slab launch");
}


// ---------------------------------------------------------------- (c)
// Row streaming: the fused (y, x) passes of a slab when the rows are short
// enough for one CTA (X % 4 == 0, X / 4 threads: X <= 4096, or 2048 for
// K >= 9) and both passes
// have the same compile-time length K in {3, 5} (zero taps skipped when the
// pass says so).
// A CTA walks a chunk of rows of one slab: every thread prefetches its 4
// columns of the row DEPTH steps ahead with cp.async (no boundary columns:
// every load is an aligned vector inside the row), keeps K rows in a
// register ring, runs the y chain, and writes the row — rounded through D —
// to one of two shared row buffers; after one barrier it runs the x chain
// for its 4 outputs from the buffer. Each buffer has K - 1 halo slots on
// both sides holding the intermediate at the mapped column (written each row
// by the thread that owns that column, from a bit mask computed once) or the
// x fill value in constant mode: that is how cuCIM's second pass sees the
// first pass's output beyond the row ends. The arithmetic, tap order and
// rounding are those of k_slab.

template <int K>
struct RowArgs {
  const void* in;
  void* out;
  long long B, Y, X;
  long long chunk;
  int ay, ax, my, mx;
  double cval_y, cval_x;  // fill values, rounded in the kernel as k_slab rounds them
  int cin_y, cin_x, dt_y, dt_x;
  uint32_t act_y, act_x;  // bit k: tap k takes part in the chain (zero taps skipped)
  float wy[K], wx[K];
};

template <int K> constexpr int row_depth() { return K * ((8 + K - 1) / K); }
// threads per CTA at most (one per 4 columns): long rings need more registers
template <int K> constexpr int row_max_threads() { return K >= 9 ? 512 : 1024; }

// row buffer (floats): RP halo slots, 4 * nthreads columns, RP halo slots, 4
// spare; RP = K - 1 rounded up to 4 keeps every float4 of the row 16-byte
// aligned. The prefetch region before the buffers is rounded up to 16 bytes.
template <int K> constexpr int row_pad() { return (K - 1 + 3) / 4 * 4; }
template <int K> constexpr int row_buf(int nthreads) { return 4 * nthreads + 2 * row_pad<K>() + 4; }
template <class T, int K>
constexpr size_t row_pre_bytes(int nthreads) {
  return ((size_t)row_depth<K>() * nthreads * 4 * sizeof(T) + 15) / 16 * 16;
}
template <class T, int K>
constexpr size_t row_smem(int nthreads) {
  return row_pre_bytes<T, K>(nthreads) + 2 * (size_t)row_buf<K>(nthreads) * 4;
}

template <class T, class D, int K>
__global__ void __launch_bounds__(row_max_threads<K>()) k_rowstream(const RowArgs<K> a) {
  constexpr int DEPTH = row_depth<K>();
  extern __shared__ __align__(16) unsigned char sm_rows[];
  const int NT = blockDim.x;
  const int t = threadIdx.x;
  T* pre = reinterpret_cast<T*>(sm_rows) + t * 4;  // prefetch slot d at pre + d * NT * 4
  // row buffers; column c of buffer j at R0 + j * RS + c (RP halo slots before)
  float* R0 = reinterpret_cast<float*>(sm_rows + row_pre_bytes<T, K>(NT)) + row_pad<K>();
  const int RS = row_buf<K>(NT);
  const long long X = a.X, Y = a.Y;
  const float cy = fill_value<float>(a.cval_y, a.cin_y, a.dt_y);
  const float cx = fill_value<float>(a.cval_x, a.cin_x, a.dt_x);
  const long long c0 = 4LL * t;  // this thread's first column
  const long long l0 = (long long)blockIdx.x * a.chunk;
  const long long l1 = min(l0 + a.chunk, Y);
  const long long n = l1 - l0;
  // halo slots: h = -ax .. -1 (bits 0 .. ax-1) and X .. X + K - 2 - ax (bits
  // ax ..); this thread fills the slots whose mapped column is one of its own
  const int nleft = a.ax, nhalo = K - 1;
  auto halo_col = [&](int i) { return i < nleft ? i - nleft : static_cast<int>(X) + (i - nleft); };
  uint32_t own = 0;
  for (int i = 0; i < nhalo; ++i) {
    const int m = map_coord32(halo_col(i), static_cast<int>(X), a.mx);
    if (m >= 0 && m >= c0 && m < c0 + 4) own |= 1u << i;
  }
  if (a.mx == CIMX_MODE_CONSTANT) {
    // constant mode: the halo holds the fill value for good
    for (int i = t; i < 2 * nhalo; i += NT)
      R0[(i / nhalo) * RS + halo_col(i % nhalo)] = cx;
  }

  for (long long b = blockIdx.y; b < a.B; b += gridDim.y) {
    const T* in = static_cast<const T*>(a.in) + b * Y * X + c0;
    D* out = static_cast<D*>(a.out) + b * Y * X + c0;
    auto mapped = [&](long long r) -> long long {
      return (r < 0 || r >= Y) ? map_coord(r, Y, a.my) : r;
    };
    auto load_row = [&](float (&v)[4], long long r) {
      const long long m = mapped(r);
      if (m < 0) v[0] = v[1] = v[2] = v[3] = cy;
      else load4<T>(in + m * X, v);
    };
    auto row_of_step = [&](long long s) { return l0 + s - a.ay + K - 1; };
    auto issue = [&](int slot, long long s) {
      const long long m = mapped(row_of_step(s));
      if (m >= 0) cp_async_vec4<T>(pre + (size_t)slot * NT * 4, in + m * X);
      cp_commit();
    };
    float win[K][4];
#pragma unroll
    for (int k = 0; k < K - 1; ++k) load_row(win[k], l0 - a.ay + k);
#pragma unroll
    for (int d = 0; d < DEPTH - 1; ++d) issue(d, d);

    // x chain of row r (its y row is complete in buffer r & 1), stored
    const bool x_aligned = (a.ax & 3) == 0;
    auto x_row = [&](long long r) {
      const float* R = R0 + (r & 1) * RS + (c0 - a.ax);
      float rv[(K + 3 + 3) / 4 * 4];
      if (x_aligned) {
#pragma unroll
        for (int q = 0; q < (K + 3 + 3) / 4; ++q) {
          const float4 f = *reinterpret_cast<const float4*>(R + 4 * q);
          rv[4 * q] = f.x;
          rv[4 * q + 1] = f.y;
          rv[4 * q + 2] = f.z;
          rv[4 * q + 3] = f.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < K + 3; ++j) rv[j] = R[j];
      }
      float xo[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < K; ++k)
        if ((a.act_x >> k) & 1u)
#pragma unroll
          for (int e = 0; e < 4; ++e) xo[e] = fmaf(rv[e + k], a.wx[k], xo[e]);
      store4<D>(out + (l0 + r) * X, xo[0], xo[1], xo[2], xo[3]);
    };

    // step s: the y chain of row s into buffer s & 1, then the x chain of
    // row s - 1 (independent work the compiler interleaves), then one
    // barrier. A buffer is rewritten two steps after it was read, and every
    // thread has passed the barrier in between.
    for (long long s0 = 0; s0 < n; s0 += DEPTH) {
#pragma unroll
      for (int u = 0; u < DEPTH; ++u) {
        const long long s = s0 + u;
        if (s < n) {  // the same for every thread of the CTA
          issue((u + DEPTH - 1) % DEPTH, s + DEPTH - 1);
          cp_wait<DEPTH - 1>();
          float* v = win[(u + K - 1) % K];
          const long long m = mapped(row_of_step(s));
          if (m < 0) {
            v[0] = v[1] = v[2] = v[3] = cy;
          } else {
            const typename Vec4<T>::type q =
                *reinterpret_cast<const typename Vec4<T>::type*>(pre + (size_t)u * NT * 4);
            v[0] = exact_float(q.x);
            v[1] = exact_float(q.y);
            v[2] = exact_float(q.z);
            v[3] = exact_float(q.w);
          }
          // y chain, rounded through D into this step's row buffer
          float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int k = 0; k < K; ++k)
            if ((a.act_y >> k) & 1u)
#pragma unroll
              for (int e = 0; e < 4; ++e) acc[e] = fmaf(win[(u + k) % K][e], a.wy[k], acc[e]);
          float* R = R0 + (s & 1) * RS;
          float iv[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) iv[e] = narrow_float<D>(acc[e]);
          *reinterpret_cast<float4*>(R + c0) = make_float4(iv[0], iv[1], iv[2], iv[3]);
          for (uint32_t bits = own; bits; bits &= bits - 1) {
            const int i = __ffs(bits) - 1;
            const int h = halo_col(i);
            const int e = map_coord32(h, static_cast<int>(X), a.mx) - static_cast<int>(c0);
            R[h] = e == 0 ? iv[0] : e == 1 ? iv[1] : e == 2 ? iv[2] : iv[3];
          }
          if (s > 0) x_row(s - 1);
          __syncthreads();
        }
      }
    }
    if (n > 0) x_row(n - 1);
    cp_wait<0>();
    __syncthreads();  // the row buffers are reused by the next slab
  }
}

template <class T, class D, int K>
int launch_rowstream_k(const SlabArgs& s, cudaStream_t st) {
  RowArgs<K> a{};
  a.in = s.in;
  a.out = s.out;
  a.B = s.B;
  a.Y = s.Y;
  a.X = s.X;
  a.ay = s.py.anchor;
  a.ax = s.px.anchor;
  a.my = s.py.mode;
  a.mx = s.px.mode;
  a.cval_y = s.py.cval;
  a.cval_x = s.px.cval;
  a.cin_y = s.py.cval_as_input;
  a.cin_x = s.px.cval_as_input;
  a.dt_y = s.py.dt;
  a.dt_x = s.px.dt;
  a.act_y = a.act_x = 0;
  for (int k = 0; k < K; ++k) {
    a.wy[k] = s.py.w[k];
    a.wx[k] = s.px.w[k];
    // with skipping, a zero tap leaves the chain (k_slab's chain2 does the same)
    if (!(s.py.skip && s.py.w[k] == 0.f)) a.act_y |= 1u << k;
    if (!(s.px.skip && s.px.w[k] == 0.f)) a.act_x |= 1u << k;
  }
  const int nt = static_cast<int>(s.X / 4);
  const size_t smem = row_smem<T, K>(nt);
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_rowstream<T, D, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kMaxSmem);
  });
  // rows per CTA: enough CTAs to fill the GPU a few times over
  long long chunk = 128;
  while (chunk > 16 && s.B * ((s.Y + chunk - 1) / chunk) < 148LL * 4) chunk /= 2;
  a.chunk = chunk;
  const long long nchunks = (s.Y + chunk - 1) / chunk;
  if (nchunks > 0x7fffffffLL) return CIMX_FUSED_DECLINED;
  const dim3 grid((unsigned)nchunks, (unsigned)std::min<long long>(s.B, 65535));
  k_rowstream<T, D, K><<<grid, nt, smem, st>>>(a);
  return cuda_fail(cudaGetLastError(), "row stream launch");
}

template <class T, class D>
bool rowstream_fits(const SlabArgs& s) {
  if (s.no_rowstream || !s.has_x || !s.has_y || s.py.K != s.px.K) return false;
  if (s.X % 4 != 0 || s.X < 4 || s.Y < 1) return false;
  // measured on a 512 x 1024 x 1024 float32 stack: 4.0 / 3.1 TB/s for 3 / 5
  // taps, faster than the slab kernel; 9 and 17 taps run at 1.7 / 0.94 TB/s,
  // below the slab's 2.4 / 1.9 (16 warps per SM cannot hide the dependent
  // chains between row barriers)
  const int K = s.py.K;
  if (K != 3 && K != 5) return false;
  if (s.X / 4 > (K >= 9 ? row_max_threads<9>() : row_max_threads<3>())) return false;
  const size_t smem = K == 3 ? row_smem<T, 3>(s.X / 4)
                      : K == 5 ? row_smem<T, 5>(s.X / 4)
                      : K == 9 ? row_smem<T, 9>(s.X / 4) : row_smem<T, 17>(s.X / 4);
  return smem <= (size_t)kMaxSmem;
}

template <class T, class D>
int launch_rowstream_td(const SlabArgs& s, cudaStream_t st) {
  switch (s.py.K) {
    case 3: return launch_rowstream_k<T, D, 3>(s, st);
    case 5: return launch_rowstream_k<T, D, 5>(s, st);
    case 9: return launch_rowstream_k<T, D, 9>(s, st);
    default: return launch_rowstream_k<T, D, 17>(s, st);
  }
}

template <class T, class D>
int launch_slab_td(SlabArgs& a, cudaStream_t st) {
  if (!a.has_y) return CIMX_FUSED_DECLINED;
  if (rowstream_fits<T, D>(a)) return launch_rowstream_td<T, D>(a, st);
  const int k8 = std::max(a.py.K8, a.has_x ? a.px.K8 : 0);
  if (k8 <= 8) return launch_slab_kb<T, D, 8>(a, st);
  if (k8 <= 16) return launch_slab_kb<T, D, 16>(a, st);
  if (k8 <= 24) return launch_slab_kb<T, D, 24>(a, st);
  if (k8 <= 32) return launch_slab_kb<T, D, 32>(a, st);
  if (k8 <= 40) return launch_slab_kb<T, D, 40>(a, st);
  if (k8 <= 48) return launch_slab_kb<T, D, 48>(a, st);
  return launch_slab_kb<T, D, 64>(a, st);
}

}  // namespace fast
}  // namespace cimx
