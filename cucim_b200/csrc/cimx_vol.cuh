// cimx_vol.cuh — the three passes of a 3-D filter (z, then y, then x, the
// order of cuCIM's _run_1d_filters, _vendored/_ndimage_filters_core.py:124-163)
// in one launch, for short taps (K in {3, 5} on every axis). Each voxel is
// read once and each output written once; the two intermediate volumes of
// the pass-by-pass schedule never reach HBM.
//
// A CTA owns an output tile of 16 M - (K - 1) rows x 120 columns and walks a
// chunk of z. Its input region is 16 M rows x 128 columns: warp w holds region
// rows w, w + 16, .. (M of them), one 4-column group per lane, 4 halo
// columns on each side. Per z step:
//   * every thread cp.async-prefetches its own groups of a future slice into
//     its own shared-memory slots (PF slices ahead, no barrier needed);
//   * the z chain runs in registers: each thread keeps the last K values of
//     its groups (a ring indexed at compile time, as f32x2 pairs), rounds the
//     chain's result through the output dtype and stores it to the plane
//     buffer P;
//   * one step later, warp w takes tile rows M*w .. M*w + M - 1: the y chain
//     from P into registers (rounded through the output dtype), then the x
//     chain with the neighbouring lanes' columns fetched by shuffles; lanes
//     1..30 store 120 output columns, lanes 0 and 31 are halo.
// P is double-buffered, so one barrier per z step orders its writes and
// reads. Boundary modes: z and y read mapped slices / rows at the address
// level; x halo columns outside the array get the z result of the column
// they map to, written by the lane that computed it (wrap-around in x reads
// columns from the far side of the array and is left to the pass-by-pass
// schedule). Constant mode fills the plane (y) or the y result (x) with the
// pass's fill value, as the separate passes would read it.
//
// Every output is the FMA chain of the separate passes (taps ascending,
// float32 fma from +0, zero taps skipped where the pass skips them, each
// intermediate rounded through the output dtype), so the result is
// bit-identical to running the three passes one launch each.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "cimx_common.cuh"
#include "cimx_fast.cuh"
#include "cimx_fused.h"

namespace cimx {
namespace vol {

// 16 warps per SM; region rows per warp: 4 for 3 taps, 3 for 5 taps (the
// ring of five slices needs the registers). 3 taps: two CTAs of 8 warps per
// SM (their barriers are independent; sobel on the 512 x 1024 x 1024 uint16
// stack 0.922 against 0.957 ms with one CTA of 16); 5 taps: one CTA of 16
// (the uniform filter 1.341 against 1.408 ms with two of 8). 24 or 32 warps
// with fewer rows each ran slower (register spills, more halo rows).
constexpr int kNW3 = 8;
constexpr int kNW5 = 16;
constexpr int kM3 = 4;
constexpr int kM5 = 3;
constexpr int kRX = 128;             // region columns (4 per lane)
constexpr int kHX = 4;               // halo columns on each side (one lane)
constexpr int kTX = kRX - 2 * kHX;   // output columns per tile

template <int K>
struct VolKArgs {
  const void* in;
  void* out;
  long long B;
  int Z, Y, X;
  int tiles_x, zchunk;
  int az, ay;
  int mz, my, mx;
  double cval_z, cval_y, cval_x;
  int cin_z, cin_y, cin_x, dt_z, dt_y, dt_x;
  uint32_t act_z, act_y, act_x;
  float wx[K];
  unsigned long long wz2[K], wy2[K];  // z and y taps, duplicated into both f32x2 lanes
};

// NW warps per CTA. Region rows are one per (warp, group): M * NW; a tile
// stores the M * NW - (K - 1) rows whose y windows lie inside the region.
template <int K, int M, int NW> constexpr int vol_ry() { return M * NW; }
template <int K, int M, int NW> constexpr int vol_out_rows() { return M * NW - (K - 1); }
// plane rows allocated: the y chains of the last warp read K - 1 rows past
// the region (never written; they only feed rows that are not stored)
template <int K, int M, int NW> constexpr int vol_plane_rows() { return M * NW + K - 1; }
template <class T> constexpr int vol_pf() { return sizeof(T) == 4 ? 3 : 5; }
template <class T, int K, int M, int NW>
constexpr size_t vol_pre_bytes() {
  return (size_t)(vol_pf<T>() + 1) * M * NW * kRX * sizeof(T);
}
template <class T, int K, int M, int NW>
constexpr size_t vol_smem() {
  return vol_pre_bytes<T, K, M, NW>() + 2 * (size_t)vol_plane_rows<K, M, NW>() * kRX * sizeof(float);
}

using fast::f2;
using fast::fma2;
using fast::hi2;
using fast::lo2;
using fast::pack2;

// four elements of T from this thread's prefetch slot, as two f32x2 pairs
template <class T>
__device__ __forceinline__ void slot_to_pairs(const T* p, f2 (&v)[2]) {
  const typename fast::Vec4<T>::type q = *reinterpret_cast<const typename fast::Vec4<T>::type*>(p);
  v[0] = pack2(fast::exact_float(q.x), fast::exact_float(q.y));
  v[1] = pack2(fast::exact_float(q.z), fast::exact_float(q.w));
}

// cast<D>() of a chain result. TRUNC: the result is known (bounded on the
// host) to lie in [0, max(D) + 1), where cast<D>() is truncation toward zero:
// adding 2^23 rounded toward zero leaves the integer in the low mantissa bits.
template <class D, bool TRUNC>
__device__ __forceinline__ float vol_narrow(float a) {
  if constexpr (sizeof(D) == 4) return a;
  else if constexpr (TRUNC) return __fsub_rn(__fadd_rz(a, 8388608.0f), 8388608.0f);
  else return fast::narrow_float<D>(a);
}

template <class D, bool TRUNC>
__device__ __forceinline__ D vol_store_cast(float a) {
  if constexpr (sizeof(D) < 4 && TRUNC)
    return static_cast<D>(__float_as_uint(__fadd_rz(a, 8388608.0f)) & (sizeof(D) == 2 ? 0xFFFFu : 0xFFu));
  else return out_cast<D>(a);
}

template <class D, bool TRUNC>
__device__ __forceinline__ void vol_store4(D* p, float a, float b, float c, float d) {
  typename fast::Vec4<D>::type q;
  q.x = vol_store_cast<D, TRUNC>(a);
  q.y = vol_store_cast<D, TRUNC>(b);
  q.z = vol_store_cast<D, TRUNC>(c);
  q.w = vol_store_cast<D, TRUNC>(d);
  *reinterpret_cast<typename fast::Vec4<D>::type*>(p) = q;
}

__device__ __forceinline__ float pick4(const float (&v)[4], int e) {
  return e == 0 ? v[0] : e == 1 ? v[1] : e == 2 ? v[2] : v[3];
}

// MASK: zero taps that the pass skips are tested for (float input, where a
// skipped tap keeps inf and nan out of the chain). Without it every tap takes
// part: for finite inputs a zero tap leaves an FMA chain from +0 unchanged.
template <class T, class D, int K, int M, int NW, bool MASK, bool TRUNC>
__global__ void __launch_bounds__(32 * NW, NW <= 8 ? 2 : 1) k_vol(const VolKArgs<K> a) {
  constexpr int RY = vol_ry<K, M, NW>();
  constexpr int TYO = vol_out_rows<K, M, NW>();
  constexpr int RXH = K / 2;  // x halo used by the x chain (symmetric taps)
  static_assert(RXH <= kHX, "x halo wider than one lane");
  constexpr int PF = vol_pf<T>();
  constexpr int DEPTH = PF + 1;
  constexpr int SLOT = M * NW * kRX;             // elements of T per prefetch slot
  constexpr int PS = vol_plane_rows<K, M, NW>() * kRX;  // floats per plane buffer
  extern __shared__ __align__(16) unsigned char sm_vol[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // this thread's prefetch position of group i: pre + slot * SLOT + i * NW * kRX
  T* const pre = reinterpret_cast<T*>(sm_vol) + w * kRX + 4 * lane;
  float* const P0 = reinterpret_cast<float*>(sm_vol + vol_pre_bytes<T, K, M, NW>());

  const int Z = a.Z, Y = a.Y, X = a.X;
  const long long YX = (long long)Y * X;
  const int bx = blockIdx.x % a.tiles_x, by = blockIdx.x / a.tiles_x;
  const int x0 = bx * kTX, y0 = by * TYO;
  const int z0 = blockIdx.y * a.zchunk;
  const int n = min(a.zchunk, Z - z0);
  const float cz = fill_value<float>(a.cval_z, a.cin_z, a.dt_z);
  const float cy = fill_value<float>(a.cval_y, a.cin_y, a.dt_y);
  const float cx = fill_value<float>(a.cval_x, a.cin_x, a.dt_x);

  // this lane's columns gx .. gx + 3 (X is a multiple of 4: all in or all out)
  const int gx = x0 - kHX + 4 * lane;
  const bool col_in = gx >= 0 && gx + 4 <= X;
  const bool xfill = a.mx == CIMX_MODE_CONSTANT && !col_in;
  // x halo columns outside the array hold the z result of the column they
  // map to (non-constant modes, no wrap-around), written by the lane that
  // computed it: at most two per lane, as (region column, element)
  int hc0 = -1, he0 = 0, hc1 = -1, he1 = 0;
  if (col_in && a.mx != CIMX_MODE_CONSTANT) {
    for (int i = 0; i < 2 * RXH; ++i) {
      const int h = i < RXH ? i - RXH : X + (i - RXH);
      const int rc = h - (x0 - kHX);
      const int m = map_coord32(h, X, a.mx);
      if (rc >= 0 && rc < kRX && m >= gx && m < gx + 4) {
        if (hc0 < 0) {
          hc0 = rc;
          he0 = m - gx;
        } else {
          hc1 = rc;
          he1 = m - gx;
        }
      }
    }
  }
  // rows of this thread's groups: group i is region row w + NW * i
  int roff[M];         // mapped row * X + gx (read only by lanes inside the array)
  uint32_t rfill = 0;  // bit i: constant mode, row outside the array
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int gy = y0 - a.ay + w + NW * i;
    const int my = (gy >= 0 && gy < Y) ? gy : map_coord32(gy, Y, a.my);
    roff[i] = my * X + gx;
    if (my < 0) rfill |= 1u << i;
  }
  // output rows of this warp's y chains: tile rows M * w + t
  const bool store_lane = lane >= 1 && lane <= 30 && gx < X;
  int nstore = 0;  // rows t < nstore are stored
  if (store_lane) nstore = max(0, min(M, min(TYO - M * w, Y - y0 - M * w)));

  for (long long b = blockIdx.z; b < a.B; b += gridDim.z) {
    const T* inb = static_cast<const T*>(a.in) + b * Z * YX;
    D* orow = static_cast<D*>(a.out) + b * Z * YX + (long long)z0 * YX +
              (long long)(y0 + M * w) * X + gx;
    auto slice_of = [&](int j) {
      const int gz = z0 - a.az + j;
      return (gz >= 0 && gz < Z) ? gz : map_coord32(gz, Z, a.mz);
    };
    const int NIN = n + K - 1;  // input slices of this chunk
    int slot_w = 0;             // prefetch slot the next issue fills
    auto issue = [&](int j) {
      if (j < NIN && col_in) {
        const int mz = slice_of(j);
        if (mz >= 0) {
          const T* src = inb + (long long)mz * YX;
          T* dst = pre + slot_w * SLOT;
#pragma unroll
          for (int i = 0; i < M; ++i)
            if (!((rfill >> i) & 1u)) fast::cp_async_vec4<T>(dst + i * NW * kRX, src + roff[i]);
        }
      }
      fast::cp_commit();
      slot_w = slot_w == DEPTH - 1 ? 0 : slot_w + 1;
    };
#pragma unroll
    for (int j = 0; j < PF; ++j) issue(j);
    int slot_r = 0;  // prefetch slot of the slice consumed next

    f2 win[M][K][2];
    // iteration j: slice j enters the ring; the z chain of output step
    // j - K + 1 goes to P; the y and x chains of output step j - K are stored
    for (int j0 = 0; j0 <= NIN; j0 += K) {
#pragma unroll
      for (int u = 0; u < K; ++u) {
        const int j = j0 + u;
        if (j <= NIN) {  // the same for every thread of the CTA
          issue(j + PF);
          fast::cp_wait<PF>();
          if (j < NIN) {
            const int mz = slice_of(j);
            const T* slot = pre + slot_r * SLOT;
            slot_r = slot_r == DEPTH - 1 ? 0 : slot_r + 1;
#pragma unroll
            for (int i = 0; i < M; ++i) {
              f2 (&v)[2] = win[i][u];
              if (mz < 0) {
                v[0] = v[1] = pack2(cz, cz);
              } else if (col_in && !((rfill >> i) & 1u)) {
                slot_to_pairs<T>(slot + i * NW * kRX, v);
              } else {
                v[0] = v[1] = 0ull;
              }
            }
            if (j >= K - 1) {
              float* P = P0 + ((j - K + 1) & 1) * PS + w * kRX + 4 * lane;
#pragma unroll
              for (int i = 0; i < M; ++i) {
                float* pr = P + i * NW * kRX;
                if ((rfill >> i) & 1u) {
                  *reinterpret_cast<float4*>(pr) = make_float4(cy, cy, cy, cy);
                } else if (col_in) {
                  f2 acc[2] = {0ull, 0ull};
#pragma unroll
                  for (int k = 0; k < K; ++k)
                    if (!MASK || ((a.act_z >> k) & 1u)) {
                      acc[0] = fma2(win[i][(u + 1 + k) % K][0], a.wz2[k], acc[0]);
                      acc[1] = fma2(win[i][(u + 1 + k) % K][1], a.wz2[k], acc[1]);
                    }
                  float o[4] = {vol_narrow<D, TRUNC>(lo2(acc[0])), vol_narrow<D, TRUNC>(hi2(acc[0])),
                                vol_narrow<D, TRUNC>(lo2(acc[1])), vol_narrow<D, TRUNC>(hi2(acc[1]))};
                  if (hc0 >= 0) {
                    pr[hc0 - 4 * lane] = pick4(o, he0);
                    if (hc1 >= 0) pr[hc1 - 4 * lane] = pick4(o, he1);
                  }
                  *reinterpret_cast<float4*>(pr) = make_float4(o[0], o[1], o[2], o[3]);
                }
                // halo lanes: their columns come from their owners
              }
            }
          }
          if (j >= K) {
            const int s = j - K;  // output step of the y and x chains
            const float* P = P0 + (s & 1) * PS + (M * w) * kRX + 4 * lane;
            f2 q[M][2];
#pragma unroll
            for (int t = 0; t < M; ++t) q[t][0] = q[t][1] = 0ull;
#pragma unroll
            for (int rr = 0; rr < M + K - 1; ++rr) {
              const ulonglong2 p = *reinterpret_cast<const ulonglong2*>(P + rr * kRX);
#pragma unroll
              for (int t = 0; t < M; ++t) {
                const int k = rr - t;
                if (k >= 0 && k < K && (!MASK || ((a.act_y >> k) & 1u))) {
                  q[t][0] = fma2(p.x, a.wy2[k], q[t][0]);
                  q[t][1] = fma2(p.y, a.wy2[k], q[t][1]);
                }
              }
            }
            D* o = orow + (long long)s * YX;
#pragma unroll
            for (int t = 0; t < M; ++t) {
              float xw[4 + 2 * RXH];
              xw[RXH + 0] = xfill ? cx : vol_narrow<D, TRUNC>(lo2(q[t][0]));
              xw[RXH + 1] = xfill ? cx : vol_narrow<D, TRUNC>(hi2(q[t][0]));
              xw[RXH + 2] = xfill ? cx : vol_narrow<D, TRUNC>(lo2(q[t][1]));
              xw[RXH + 3] = xfill ? cx : vol_narrow<D, TRUNC>(hi2(q[t][1]));
#pragma unroll
              for (int c = 0; c < RXH; ++c) {
                xw[c] = __shfl_up_sync(0xffffffffu, xw[4 + c], 1);
                xw[RXH + 4 + c] = __shfl_down_sync(0xffffffffu, xw[RXH + c], 1);
              }
              float xo[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
              for (int k = 0; k < K; ++k)
                if (!MASK || ((a.act_x >> k) & 1u))
#pragma unroll
                  for (int e = 0; e < 4; ++e) xo[e] = fmaf(xw[e + k], a.wx[k], xo[e]);
              if (t < nstore) vol_store4<D, TRUNC>(o + (long long)t * X, xo[0], xo[1], xo[2], xo[3]);
            }
          }
          __syncthreads();
        }
      }
    }
    fast::cp_wait<0>();
  }
}

inline unsigned long long two_lanes(float w) {
  uint32_t b;
  std::memcpy(&b, &w, 4);
  return (static_cast<unsigned long long>(b) << 32) | b;
}

template <class T, class D, int K, int M, int NW, bool MASK, bool TRUNC>
int launch_vol_km(const VolArgs& v, cudaStream_t st) {
  VolKArgs<K> a{};
  a.in = v.in;
  a.out = v.out;
  a.B = v.B;
  a.Z = static_cast<int>(v.Z);
  a.Y = static_cast<int>(v.Y);
  a.X = static_cast<int>(v.X);
  a.az = v.pz.anchor;
  a.ay = v.py.anchor;
  a.mz = v.pz.mode;
  a.my = v.py.mode;
  a.mx = v.px.mode;
  a.cval_z = v.pz.cval;
  a.cval_y = v.py.cval;
  a.cval_x = v.px.cval;
  a.cin_z = v.pz.cval_as_input;
  a.cin_y = v.py.cval_as_input;
  a.cin_x = v.px.cval_as_input;
  a.dt_z = v.pz.dt;
  a.dt_y = v.py.dt;
  a.dt_x = v.px.dt;
  a.act_z = a.act_y = a.act_x = 0;
  for (int k = 0; k < K; ++k) {
    a.wz2[k] = two_lanes(v.pz.w[k]);
    a.wy2[k] = two_lanes(v.py.w[k]);
    a.wx[k] = v.px.w[k];
    if (!(v.pz.skip && v.pz.w[k] == 0.f)) a.act_z |= 1u << k;
    if (!(v.py.skip && v.py.w[k] == 0.f)) a.act_y |= 1u << k;
    if (!(v.px.skip && v.px.w[k] == 0.f)) a.act_x |= 1u << k;
  }
  constexpr int TY = vol_out_rows<K, M, NW>();
  a.tiles_x = static_cast<int>((v.X + kTX - 1) / kTX);
  const long long tiles = (long long)a.tiles_x * ((v.Y + TY - 1) / TY);
  // z chunk: long enough that the K - 1 extra slices stay a small share,
  // short enough for a few waves of CTAs (one or two per SM). Measured on the
  // 512 x 1024 x 1024 uint16 stack: 3 taps ran 2.3 % faster with 32-slice
  // chunks (12 waves) than with 64; 5 taps showed no such gain.
  const long long waves = K == 3 ? 12 : 6;
  int zc = 128;
  while (zc > 16 && tiles * ((v.Z + zc - 1) / zc) * v.B < 148LL * waves) zc /= 2;
  if (v.zchunk > 0) zc = v.zchunk;  // a tuned or forced chunk (any chunk is exact)
  a.zchunk = zc;
  const long long nzc = (v.Z + zc - 1) / zc;
  if (tiles > 0x7fffffffLL || nzc > 65535) return CIMX_FUSED_DECLINED;
  constexpr size_t smem = vol_smem<T, K, M, NW>();
  static_assert(smem <= (size_t)fast::kMaxSmem, "volume kernel shared memory");
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(k_vol<T, D, K, M, NW, MASK, TRUNC>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (attr != cudaSuccess) return cuda_fail(attr, "volume kernel shared memory attribute");
  const dim3 grid((unsigned)tiles, (unsigned)nzc, (unsigned)std::min<long long>(v.B, 65535));
  k_vol<T, D, K, M, NW, MASK, TRUNC><<<grid, 32 * NW, smem, st>>>(a);
  return cuda_fail(cudaGetLastError(), "volume kernel launch");
}

// Integer input and integer output: when every tap is non-negative, every
// fill value lies in [0, max(D)] and the largest input times the taps'
// sums stays below max(D) + 1 after each pass, every chain result lies in
// [0, max(D) + 1) and cast<D>() is plain truncation (the TRUNC kernels).
template <class T, class D>
bool trunc_bounded(const VolArgs& v) {
  const double dmax = sizeof(D) == 2 ? 65535.0 : 255.0;
  const double tmax = sizeof(T) == 2 ? 65535.0 : 255.0;
  const SlabPass* ps[3] = {&v.pz, &v.py, &v.px};
  double bound = tmax;
  for (const SlabPass* p : ps) {
    if (p->mode == CIMX_MODE_CONSTANT && !(p->cval >= 0.0 && p->cval <= std::min(tmax, dmax)))
      return false;
    double sum = 0.0;
    for (int k = 0; k < p->K; ++k) {
      if (!(p->w[k] >= 0.f)) return false;
      sum += p->w[k];
    }
    // a float32 FMA chain of K non-negative terms exceeds the exact sum by
    // at most K * 2^-24 of it (below 1e-6 for K <= 16); truncation only
    // lowers the next pass's input
    bound *= sum * (1.0 + 1e-6);
    if (!(bound < dmax + 1.0)) return false;
  }
  return true;
}

// Skipped zero taps only change a chain whose input is inf or nan. Integer
// input is finite, and so is every intermediate while the taps cannot
// overflow float32 (bounded here on the host) and the fill values are
// finite: those launches run without the tests. Float input keeps them when
// any pass skips a tap.
template <class T, class D>
int launch_vol_td(const VolArgs& v, cudaStream_t st) {
  const int K = v.pz.K;
  bool mask = v.pz.skip || v.py.skip || v.px.skip;
  auto nonfinite_fill = [](const SlabPass& p) {
    return p.mode == CIMX_MODE_CONSTANT && !std::isfinite(p.cval);
  };
  if (mask && sizeof(T) < 4) {
    if (nonfinite_fill(v.pz) || nonfinite_fill(v.py) || nonfinite_fill(v.px))
      return CIMX_FUSED_DECLINED;
    double sz = 0, sy = 0;
    for (int k = 0; k < K; ++k) {
      sz += std::fabs((double)v.pz.w[k]);
      sy += std::fabs((double)v.py.w[k]);
    }
    // |z result| <= 65535 sz, |y result| <= 65535 sz sy (before rounding)
    if (65536.0 * sz * std::max(1.0, sy) >= 1e37) return CIMX_FUSED_DECLINED;
    mask = false;
  }
  if constexpr (sizeof(T) == 4) {
    if (mask) {
      if (K == 3) return launch_vol_km<T, D, 3, kM3, kNW3, true, false>(v, st);
      if (K == 5) return launch_vol_km<T, D, 5, kM5, kNW5, true, false>(v, st);
      return CIMX_FUSED_DECLINED;
    }
  }
  if constexpr (sizeof(T) < 4 && sizeof(D) < 4) {
    if (trunc_bounded<T, D>(v)) {
      if (K == 3) return launch_vol_km<T, D, 3, kM3, kNW3, false, true>(v, st);
      if (K == 5) return launch_vol_km<T, D, 5, kM5, kNW5, false, true>(v, st);
      return CIMX_FUSED_DECLINED;
    }
  }
  if (K == 3) return launch_vol_km<T, D, 3, kM3, kNW3, false, false>(v, st);
  if (K == 5) return launch_vol_km<T, D, 5, kM5, kNW5, false, false>(v, st);
  return CIMX_FUSED_DECLINED;
}

}  // namespace vol
}  // namespace cimx
