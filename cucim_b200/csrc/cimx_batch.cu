// cimx_batch.cu — many uneven tiles in one persistent launch: for every
// uint8 RGB tile, rgb2gray, then a gaussian (its own sigma, mode 'nearest'),
// then the sobel gradient magnitude (mode 'reflect'), float32 out — the
// pipeline of skimage.color.rgb2gray -> skimage.filters.gaussian ->
// skimage.filters.sobel (color/colorconv.py:1038-1095,
// _shared/filters.py:21-166, filters/edges.py:148-306), computed with exactly
// the arithmetic of the per-tile path of this library:
//   gray  = (float)(0.0721 b + (0.2125 r + 0.7154 g)) in float64 fused multiply-adds,
//           r = (float)u8 * (float)(1/255) (a 256-entry table of the float64 values);
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

// The float64 value of one channel: (double)((float)u * (float)(1/255)).
__device__ __forceinline__ double channel_f64(int u) {
  return static_cast<double>(__fmul_rn(static_cast<float>(u), static_cast<float>(1.0 / 255.0)));
}

// gray = (float)(0.2125 r + 0.7154 g + 0.0721 b) with the float64
// operations in the order the per-tile rgb2gray kernel contracts them:
// 0.0721 b + (0.2125 r + 0.7154 g), each sum a fused multiply-add.
__device__ __forceinline__ float luma_f64(double r, double g, double b) {
  return __double2float_rn(__fma_rn(0.0721, b, __fma_rn(0.2125, r, __dmul_rn(0.7154, g))));
}

constexpr int kSS = kBT + 3;  // row stride of S: odd, for the column-wise writes of the x pass
constexpr int kGB = 4;  // 4-pixel groups whose words a thread loads at once (gray step)
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
  __shared__ CimxBatchTile s_t;                    // this block's tile
  __shared__ float s_w[kBMaxTaps];                 // this tile's taps
  __shared__ int s_ci[kBT + 2], s_cj[kBT + 2];     // source row / column of each T row, S column
  __shared__ int s_yc[kBG], s_xc[kBG];             // group of 8 with consecutive sources
  __shared__ double s_ch[256];                     // channel_f64 of every byte value
  const int tid = threadIdx.x;
  for (int u = tid; u < 256; u += kBThreads) s_ch[u] = channel_f64(u);
  // strides sized for the batch's largest radius; odd, so that lanes on
  // consecutive rows read different banks
  const int gcs = kBT + 3 + 2 * a.max_r;  // row stride of the gray region and of T
  float* G = smf;                          // (64 + 2 + 2r) rows x gcs
  float* T = smf + gcs * gcs;              // 66 rows x gcs
  // overlays of G once T exists: S (66 x 66, row stride kSS), E0 (64 x 66),
  // E1 (66 x 64)
  float* S = smf;
  float* E0 = S + (kBT + 2) * kSS;
  float* E1 = E0 + kBT * (kBT + 2);

  for (long long g = blockIdx.x; g < a.nblocks; g += gridDim.x) {
    if (tid < 32) {
      // the last tile whose first block <= g, found by the first warp: each
      // round probes 32 evenly spaced tiles of (lo, hi] and keeps the span
      // between the last probe <= g and the next one (three rounds for
      // 4096 tiles)
      int lo = 0, hi = a.ntiles - 1;
      while (hi > lo) {
        const int step = (hi - lo + 31) / 32;
        const int cand = lo + 1 + tid * step;
        const bool le = cand <= hi && a.tiles[cand].first_block <= g;
        const int nle = __popc(__ballot_sync(0xffffffffu, le));
        if (nle == 0) {
          hi = lo;
        } else {
          lo += 1 + (nle - 1) * step;
          hi = min(hi, lo + step - 1);
        }
      }
      if (tid == 0) s_t = a.tiles[lo];
    }
    __syncthreads();
    const CimxBatchTile& t = s_t;
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

    // 1. gray region: rows y0-1-r .., columns x0-1-r .., 'nearest' borders.
    //    A thread takes groups of 4 consecutive pixels of a row: where they
    //    lie inside the row, their 12 bytes come from three or four aligned
    //    32-bit words (each word holds at least one of the 12 bytes, so it
    //    lies in the tile's allocation); at the tile's borders pixel by
    //    pixel. The words of kGB groups are loaded before any is used.
    {
      const int GC4 = (GC + 3) >> 2, ng = GR * GC4;
      const int xb = x0 - 1 - r;  // source column of region column 0
      for (int i0 = tid; i0 < ng; i0 += kGB * kBThreads) {
        uint32_t wv[kGB][4];
        unsigned shv[kGB];
        bool fast[kGB];
#pragma unroll
        for (int u = 0; u < kGB; ++u) {
          const int idx = i0 + u * kBThreads;
          const int gr = idx / GC4, c0 = (idx - gr * GC4) * 4;
          const int xs = xb + c0;
          fast[u] = idx < ng && xs >= 0 && xs + 3 < W && c0 + 3 < GC;
          shv[u] = 0;
          wv[u][0] = wv[u][1] = wv[u][2] = wv[u][3] = 0u;
          if (fast[u]) {
            const uint8_t* px = t.rgb + static_cast<long long>(nearest_idx(y0 - 1 - r + gr, H)) * in_pitch + 3LL * xs;
            const uintptr_t pa = reinterpret_cast<uintptr_t>(px);
            const uint32_t* wp = reinterpret_cast<const uint32_t*>(pa & ~static_cast<uintptr_t>(3));
            shv[u] = static_cast<unsigned>(pa & 3) * 8u;
            wv[u][0] = __ldg(wp);
            wv[u][1] = __ldg(wp + 1);
            wv[u][2] = __ldg(wp + 2);
            if (shv[u]) wv[u][3] = __ldg(wp + 3);
          }
        }
#pragma unroll
        for (int u = 0; u < kGB; ++u) {
          const int idx = i0 + u * kBThreads;
          if (idx >= ng) break;
          const int gr = idx / GC4, c0 = (idx - gr * GC4) * 4;
          float* dst = G + gr * gcs + c0;
          if (fast[u]) {
            const unsigned sh = shv[u];
            const uint32_t v0 = __funnelshift_r(wv[u][0], wv[u][1], sh);
            const uint32_t v1 = __funnelshift_r(wv[u][1], wv[u][2], sh);
            const uint32_t v2 = __funnelshift_r(wv[u][2], wv[u][3], sh);
            dst[0] = luma_f64(s_ch[v0 & 255u], s_ch[(v0 >> 8) & 255u], s_ch[(v0 >> 16) & 255u]);
            dst[1] = luma_f64(s_ch[v0 >> 24], s_ch[v1 & 255u], s_ch[(v1 >> 8) & 255u]);
            dst[2] = luma_f64(s_ch[(v1 >> 16) & 255u], s_ch[v1 >> 24], s_ch[v2 & 255u]);
            dst[3] = luma_f64(s_ch[(v2 >> 8) & 255u], s_ch[(v2 >> 16) & 255u], s_ch[v2 >> 24]);
          } else {
            const uint8_t* row = t.rgb + static_cast<long long>(nearest_idx(y0 - 1 - r + gr, H)) * in_pitch;
            const int xs = xb + c0;
            for (int p = 0; p < 4 && c0 + p < GC; ++p) {
              const uint8_t* px = row + 3LL * nearest_idx(xs + p, W);
              dst[p] = luma_f64(s_ch[px[0]], s_ch[px[1]], s_ch[px[2]]);
            }
          }
        }
      }
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
        for (int p = 0; p < kBR; ++p) S[sr * kSS + sc0 + p] = acc[p];
      } else {
        for (int p = 0; p < nc; ++p) {
          const float* row = T + sr * gcs + (s_cj[sc0 + p] - r);
          float acc = 0.f;
          for (int k = 0; k < K; ++k) acc = fmaf(row[k], s_w[k], acc);
          S[sr * kSS + sc0 + p] = acc;
        }
      }
    }
    __syncthreads();

    // 4. edge passes: E0 along y (64 x 66), E1 along x (66 x 64)
    for (int idx = tid; idx < kBT * (kBT + 2); idx += kBThreads) {
      const int y = idx / (kBT + 2), sc = idx - y * (kBT + 2);
      float acc = 0.f;
      acc = fmaf(S[y * kSS + sc], a.edge[0], acc);
      acc = fmaf(S[(y + 1) * kSS + sc], a.edge[1], acc);
      acc = fmaf(S[(y + 2) * kSS + sc], a.edge[2], acc);
      E0[idx] = acc;
    }
    for (int idx = tid; idx < (kBT + 2) * kBT; idx += kBThreads) {
      const int sr = idx / kBT, x = idx - sr * kBT;
      const float* row = S + sr * kSS + x;
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
  const size_t overlay = static_cast<size_t>(kBT + 2) * kSS + 2 * kBT * (kBT + 2);
  const size_t smem = sizeof(float) * std::max(region, overlay);
  // the kernel also holds about 3.2 KB of static shared memory (taps, the
  // row / column tables, the channel table); the sum stays under the 227 KB
  // per CTA
  constexpr int kDynLimit = 223 * 1024;
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
