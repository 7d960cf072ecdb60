// cimx_batch.cu — many uneven tiles in one persistent launch: for every
// uint8 RGB tile, rgb2gray, then a gaussian (its own sigma, mode 'nearest'),
// then the sobel gradient magnitude (mode 'reflect'), float32 out — the
// pipeline of skimage.color.rgb2gray -> skimage.filters.gaussian ->
// skimage.filters.sobel (color/colorconv.py:1038-1095,
// _shared/filters.py:21-166, filters/edges.py:148-306), computed with exactly
// the arithmetic of the per-tile path of this library:
//   gray  = (float)(0.2125 r + 0.7154 g + 0.0721 b) in float64, r = (float)u8 * (float)(1/255);
//   T     = gaussian along y of gray (float32 FMA chain, taps ascending, from +0),
//   S     = gaussian along x of T, both with 'nearest' borders;
//   d0    = smooth along x of (edge along y of S), d1 = smooth along y of (edge along x of S),
//           edge taps [-a, 0, a] (a = 1/sqrt(2) in float32), smooth [1/4, 1/2, 1/4],
//           'reflect' borders, float32 intermediates;
//   out   = sqrt(d0*d0 + d1*d1), each product and the sum rounded to float32.
//
// Work: the tiles' 64 x 64 output blocks form one flat list (each tile knows
// the index of its first block); CTAs walk the list with a grid stride. A
// block stages its gray halo region (64 + 2 + 2r)^2 in shared memory, runs
// the y pass into a second buffer, then the x pass, the two edge passes and
// the two smoothing passes in the space the gray region left. The launch
// reads only device memory that the caller prepared, so it can be captured
// in a CUDA graph and replayed.
#include <algorithm>
#include <mutex>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

constexpr int kBT = 64;          // output block side
constexpr int kBThreads = 256;
constexpr int kBMaxTaps = 129;   // radius <= 64
static_assert(sizeof(CimxBatchTile) == 56, "CimxBatchTile layout is part of the ABI");

struct BatchArgs {
  const CimxBatchTile* tiles;
  int ntiles;
  long long nblocks;
  const float* taps;
  int max_r;
  float edge[3], smooth[3];
};

__device__ __forceinline__ int nearest_idx(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

__device__ __forceinline__ float luma_u8(const uint8_t* p) {
  const float s = static_cast<float>(1.0 / 255.0);
  const float r = __fmul_rn(static_cast<float>(p[0]), s);
  const float g = __fmul_rn(static_cast<float>(p[1]), s);
  const float b = __fmul_rn(static_cast<float>(p[2]), s);
  float y = 0.2125 * r + 0.7154 * g + 0.0721 * b;
  return y;
}

constexpr int kBR = 8;  // outputs per thread in the Gaussian passes
constexpr int kBG = (kBT + 2 + kBR - 1) / kBR;  // 8-output groups over 66 rows or columns

// acc[p] = the fused multiply-add chain over taps k = 0 .. K-1 of
// x(p + k) * w[k], for kBR consecutive outputs p: the taps ascending from
// +0 exactly as the one-output loop, with the inputs of a chunk of kBR taps
// held in registers (each loaded once for the kBR outputs). `at(i)` may be
// asked for up to 2 kBR - 1 inputs beyond the last one used.
template <class At>
__device__ __forceinline__ void chain_r(float (&acc)[kBR], const float* w, int K, At at) {
  float win[2 * kBR];
#pragma unroll
  for (int j = 0; j < kBR; ++j) win[j] = at(j);
  int k0 = 0;
  for (; k0 + kBR <= K; k0 += kBR) {
#pragma unroll
    for (int j = 0; j < kBR; ++j) win[kBR + j] = at(k0 + kBR + j);
#pragma unroll
    for (int j = 0; j < kBR; ++j) {
      const float t = w[k0 + j];
#pragma unroll
      for (int p = 0; p < kBR; ++p) acc[p] = fmaf(win[p + j], t, acc[p]);
    }
#pragma unroll
    for (int j = 0; j < kBR; ++j) win[j] = win[kBR + j];
  }
  if (k0 < K) {
#pragma unroll
    for (int j = 0; j < kBR; ++j) win[kBR + j] = at(k0 + kBR + j);
#pragma unroll
    for (int j = 0; j < kBR; ++j) {
      if (k0 + j < K) {
        const float t = w[k0 + j];
#pragma unroll
        for (int p = 0; p < kBR; ++p) acc[p] = fmaf(win[p + j], t, acc[p]);
      }
    }
  }
}

__global__ void __launch_bounds__(kBThreads, 2) k_batch_gray_gauss_sobel(const BatchArgs a) {
  extern __shared__ float smf[];
  __shared__ int s_tile;
  __shared__ float s_w[kBMaxTaps];                 // this tile's taps
  __shared__ int s_ci[kBT + 2], s_cj[kBT + 2];     // source row / column of each T row, S column
  __shared__ int s_yc[kBG], s_xc[kBG];             // group of 8 with consecutive sources
  const int tid = threadIdx.x;
  // strides sized for the batch's largest radius; odd, so that lanes on
  // consecutive rows read different banks
  const int gcs = kBT + 3 + 2 * a.max_r;  // row stride of the gray region and of T
  float* G = smf;                          // (64 + 2 + 2r) rows x gcs
  float* T = smf + gcs * gcs;              // 66 rows x gcs
  // overlays of G once T exists: S (66 x 66), E0 (64 x 66), E1 (66 x 64)
  float* S = smf;
  float* E0 = S + (kBT + 2) * (kBT + 2);
  float* E1 = E0 + kBT * (kBT + 2);

  for (long long g = blockIdx.x; g < a.nblocks; g += gridDim.x) {
    if (tid == 0) {
      int lo = 0, hi = a.ntiles - 1;  // last tile whose first block <= g
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.tiles[mid].first_block <= g) lo = mid;
        else hi = mid - 1;
      }
      s_tile = lo;
    }
    __syncthreads();
    const CimxBatchTile t = a.tiles[s_tile];
    const int H = t.height, W = t.width;
    // row pitches: a tile may be a region of a larger slide (0 = packed)
    const long long in_pitch = t.rgb_pitch > 0 ? t.rgb_pitch : 3LL * W;
    const long long out_pitch = t.out_pitch > 0 ? t.out_pitch : W;
    const int nbx = (W + kBT - 1) / kBT;
    const long long j = g - t.first_block;
    // a block index outside the tile (inconsistent table) is skipped; the
    // test is uniform across the CTA, so every barrier below is still met
    const bool valid = j >= 0 && j < static_cast<long long>(nbx) * ((H + kBT - 1) / kBT) &&
                       t.ntaps >= 1 && t.ntaps / 2 <= a.max_r;
    if (!valid) {
      __syncthreads();
      continue;
    }
    const int y0 = static_cast<int>(j / nbx) * kBT, x0 = static_cast<int>(j % nbx) * kBT;
    const int K = t.ntaps, r = K / 2;
    const float* w = a.taps + t.taps_offset;
    const int GR = kBT + 2 + 2 * r, GC = kBT + 2 + 2 * r;

    // 0. the tile's taps, and the source row / column (in the gray region)
    //    of every smoothed row / column the edge passes read: 'reflect'
    //    around the tile, kept inside the region
    for (int k = tid; k < K; k += kBThreads) s_w[k] = w[k];
    for (int i = tid; i < kBT + 2; i += kBThreads) {
      int ci = map_coord32(y0 - 1 + i, H, CIMX_MODE_REFLECT) - (y0 - 1 - r);
      s_ci[i] = ci < r ? r : (ci > GR - 1 - r ? GR - 1 - r : ci);
      int cj = map_coord32(x0 - 1 + i, W, CIMX_MODE_REFLECT) - (x0 - 1 - r);
      s_cj[i] = cj < r ? r : (cj > GC - 1 - r ? GC - 1 - r : cj);
    }
    __syncthreads();
    if (tid < 2 * kBG) {
      const int q = tid % kBG, i0 = q * kBR;
      const int* src = tid < kBG ? s_ci : s_cj;
      int ok = i0 + kBR <= kBT + 2;
      for (int p = 1; ok && p < kBR; ++p) ok = src[i0 + p] == src[i0] + p;
      (tid < kBG ? s_yc : s_xc)[q] = ok;
    }

    // 1. gray region: rows y0-1-r .., columns x0-1-r .., 'nearest' borders
    for (int idx = tid; idx < GR * GC; idx += kBThreads) {
      const int gr = idx / GC, c = idx - gr * GC;
      const int gy = nearest_idx(y0 - 1 - r + gr, H), gx = nearest_idx(x0 - 1 - r + c, W);
      G[gr * gcs + c] = luma_u8(t.rgb + static_cast<long long>(gy) * in_pitch + gx * 3LL);
    }
    __syncthreads();

    // 2. gaussian along y: T row tr is the smoothed row refl(y0 - 1 + tr);
    //    rows outside the tile only feed outputs that are not stored. A
    //    thread takes 8 consecutive T rows of one column; where their source
    //    rows are not consecutive (tile borders) it runs them one by one.
    for (int idx = tid; idx < kBG * GC; idx += kBThreads) {
      const int q = idx / GC, c = idx - q * GC;
      const int tr0 = q * kBR, nr = min(kBR, kBT + 2 - tr0);
      if (s_yc[q]) {
        float acc[kBR];
#pragma unroll
        for (int p = 0; p < kBR; ++p) acc[p] = 0.f;
        const float* col = G + (s_ci[tr0] - r) * gcs + c;
        chain_r(acc, s_w, K, [&](int i) { return col[i * gcs]; });
#pragma unroll
        for (int p = 0; p < kBR; ++p) T[(tr0 + p) * gcs + c] = acc[p];
      } else {
        for (int p = 0; p < nr; ++p) {
          const float* col = G + (s_ci[tr0 + p] - r) * gcs + c;
          float acc = 0.f;
          for (int k = 0; k < K; ++k) acc = fmaf(col[k * gcs], s_w[k], acc);
          T[(tr0 + p) * gcs + c] = acc;
        }
      }
    }
    __syncthreads();

    // 3. gaussian along x: S(sr, sc) is the smoothed value at
    //    (refl(y0 - 1 + sr), refl(x0 - 1 + sc)); a thread takes 8
    //    consecutive columns of one row (lanes on consecutive rows)
    for (int idx = tid; idx < kBG * (kBT + 2); idx += kBThreads) {
      const int q = idx / (kBT + 2), sr = idx - q * (kBT + 2);
      const int sc0 = q * kBR, nc = min(kBR, kBT + 2 - sc0);
      if (s_xc[q]) {
        float acc[kBR];
#pragma unroll
        for (int p = 0; p < kBR; ++p) acc[p] = 0.f;
        const float* row = T + sr * gcs + (s_cj[sc0] - r);
        chain_r(acc, s_w, K, [&](int i) { return row[i]; });
#pragma unroll
        for (int p = 0; p < kBR; ++p) S[sr * (kBT + 2) + sc0 + p] = acc[p];
      } else {
        for (int p = 0; p < nc; ++p) {
          const float* row = T + sr * gcs + (s_cj[sc0 + p] - r);
          float acc = 0.f;
          for (int k = 0; k < K; ++k) acc = fmaf(row[k], s_w[k], acc);
          S[sr * (kBT + 2) + sc0 + p] = acc;
        }
      }
    }
    __syncthreads();

    // 4. edge passes: E0 along y (64 x 66), E1 along x (66 x 64)
    for (int idx = tid; idx < kBT * (kBT + 2); idx += kBThreads) {
      const int y = idx / (kBT + 2), sc = idx - y * (kBT + 2);
      float acc = 0.f;
      acc = fmaf(S[y * (kBT + 2) + sc], a.edge[0], acc);
      acc = fmaf(S[(y + 1) * (kBT + 2) + sc], a.edge[1], acc);
      acc = fmaf(S[(y + 2) * (kBT + 2) + sc], a.edge[2], acc);
      E0[idx] = acc;
    }
    for (int idx = tid; idx < (kBT + 2) * kBT; idx += kBThreads) {
      const int sr = idx / kBT, x = idx - sr * kBT;
      const float* row = S + sr * (kBT + 2) + x;
      float acc = 0.f;
      acc = fmaf(row[0], a.edge[0], acc);
      acc = fmaf(row[1], a.edge[1], acc);
      acc = fmaf(row[2], a.edge[2], acc);
      E1[idx] = acc;
    }
    __syncthreads();

    // 5. smoothing passes and the magnitude
    for (int idx = tid; idx < kBT * kBT; idx += kBThreads) {
      const int y = idx / kBT, x = idx - y * kBT;
      if (y0 + y >= H || x0 + x >= W) continue;
      const float* e0 = E0 + y * (kBT + 2) + x;
      float d0 = 0.f;
      d0 = fmaf(e0[0], a.smooth[0], d0);
      d0 = fmaf(e0[1], a.smooth[1], d0);
      d0 = fmaf(e0[2], a.smooth[2], d0);
      const float* e1 = E1 + y * kBT + x;
      float d1 = 0.f;
      d1 = fmaf(e1[0], a.smooth[0], d1);
      d1 = fmaf(e1[kBT], a.smooth[1], d1);
      d1 = fmaf(e1[2 * kBT], a.smooth[2], d1);
      const float m = __fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1));
      t.out[static_cast<long long>(y0 + y) * out_pitch + x0 + x] = sqrtf(m);
    }
    __syncthreads();  // shared buffers are reused by the next block
  }
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" int cimx_batch_gray_gauss_sobel(const CimxBatchTile* tiles, int ntiles,
                                           long long nblocks, const float* taps, int max_taps,
                                           const float* edge_taps, const float* smooth_taps,
                                           void* stream) {
  if (ntiles < 0 || nblocks < 0) return fail(CIMX_E_INVALID, "batch: negative counts");
  if (ntiles == 0 || nblocks == 0) return CIMX_OK;
  if (!tiles || !taps || !edge_taps || !smooth_taps)
    return fail(CIMX_E_INVALID, "batch: NULL argument");
  if (max_taps < 1 || max_taps > kBMaxTaps || max_taps % 2 == 0)
    return fail(CIMX_E_INVALID, "batch: max_taps must be odd and at most 129");
  BatchArgs a{};
  a.tiles = tiles;
  a.ntiles = ntiles;
  a.nblocks = nblocks;
  a.taps = taps;
  a.max_r = max_taps / 2;
  for (int k = 0; k < 3; ++k) {
    a.edge[k] = edge_taps[k];
    a.smooth[k] = smooth_taps[k];
  }
  // gray region + T, or S + E0 + E1 (which overlay the gray region and
  // spill into T for small radii), whichever is larger
  const int gcs = kBT + 3 + 2 * a.max_r;
  // the register-blocked chains read up to 2 * 8 - 1 inputs past the last
  // one they use: slack after T for its last row
  const size_t region = static_cast<size_t>(gcs) * gcs + static_cast<size_t>(kBT + 2) * gcs + 64;
  const size_t overlay = static_cast<size_t>(kBT + 2) * (kBT + 2) + 2 * kBT * (kBT + 2);
  const size_t smem = sizeof(float) * std::max(region, overlay);
  // the kernel also holds about 1.2 KB of static shared memory (taps and
  // the row / column tables); the sum stays under the 227 KB per CTA
  constexpr int kDynLimit = 225 * 1024;
  if (smem > static_cast<size_t>(kDynLimit)) return fail(CIMX_E_INVALID, "batch: taps too long");
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [] {
    attr_err = cudaFuncSetAttribute(k_batch_gray_gauss_sobel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, kDynLimit);
  });
  if (attr_err != cudaSuccess) return cuda_fail(attr_err, "batch: shared memory attribute");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long grid = std::min<long long>(nblocks, 2LL * sms);
  k_batch_gray_gauss_sobel<<<(unsigned)grid, kBThreads, smem, static_cast<cudaStream_t>(stream)>>>(a);
  return cuda_fail(cudaGetLastError(), "batch launch");
}
