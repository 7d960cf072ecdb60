// cimx_batch.cu — many uneven tiles in one persistent launch: for every
// uint8 RGB tile, rgb2gray, then a gaussian (its own sigma, mode 'nearest'),
// then the sobel gradient magnitude (mode 'reflect'), float32 out — the
// pipeline of skimage.color.rgb2gray -> skimage.filters.gaussian ->
// skimage.filters.sobel (color/colorconv.py:1038-1095,
// _shared/filters.py:21-166, filters/edges.py:148-306), computed with exactly
// the arithmetic of the per-tile path of this library:
//   gray  = (float)(0.0721 b + (0.2125 r + 0.7154 g)) in float64 fused multiply-adds,
//           r = (float)u8 * (float)(1/255) widened to float64;
//   T     = gaussian along y of gray (float32 FMA chain, taps ascending, from +0),
//   S     = gaussian along x of T, both with 'nearest' borders;
//   d0    = smooth along x of (edge along y of S), d1 = smooth along y of (edge along x of S),
//           edge taps [-a, 0, a] (a = 1/sqrt(2) in float32), smooth [1/4, 1/2, 1/4],
//           'reflect' borders, float32 intermediates;
//   out   = sqrt(d0*d0 + d1*d1), each product and the sum rounded to float32.
//
// Work: the tiles' 64 x 64 output blocks form one flat list (each tile knows
// the index of its first block); CTAs (three per SM up to a radius of about
// 38) walk the list with a grid stride. A block computes its gray halo
// region ((64 + 2 + 2r) rows) in strips of 28 columns through two
// shared-memory buffers, the next strip's loads in flight during the current
// strip's y pass into T; then the x pass into S (over the strip buffers),
// and the edge, smoothing and magnitude steps per 4 outputs in registers.
// The launch reads only device memory that the caller prepared, so it can
// be captured in a CUDA graph and replayed.
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

// The float64 value of one channel, (double)((float)u * (float)(1/255)),
// computed without a table (a table's random reads conflicted on the
// shared-memory banks): float(u) exactly, the float32 product, then the
// float widened by rebiasing its exponent (the value is 0 or normal)
__device__ __forceinline__ double chan(uint32_t u) {
  const float f = __fmul_rn(__fsub_rn(__uint_as_float(0x4B000000u | u), 8388608.0f),
                            static_cast<float>(1.0 / 255.0));
  const unsigned long long b = __float_as_uint(f);
  return __longlong_as_double(
      b ? static_cast<long long>((b << 29) + (static_cast<unsigned long long>(1023 - 127) << 52))
        : 0ll);
}

// gray = (float)(0.2125 r + 0.7154 g + 0.0721 b) with the float64
// operations in the order the per-tile rgb2gray kernel contracts them:
// 0.0721 b + (0.2125 r + 0.7154 g), each sum a fused multiply-add.
__device__ __forceinline__ float luma_f64(double r, double g, double b) {
  return __double2float_rn(__fma_rn(0.0721, b, __fma_rn(0.2125, r, __dmul_rn(0.7154, g))));
}

constexpr int kSS = kBT + 3;  // row stride of S: odd, for the column-wise writes of the x pass
constexpr int kGB = 4;  // 4-pixel groups whose words a thread loads at once (gray step)
constexpr int kCW = 28;  // gray-region columns per strip: 9 x 28 y-pass items fill 256 threads once
constexpr int kCG = kCW / 4;  // 4-pixel groups per strip row
constexpr int kSlack = 16;    // spare strip rows: the chains may read 2 x 8 - 1 rows past the last
constexpr int kBR = 8;  // outputs per thread in the Gaussian passes
constexpr int kBG = (kBT + 2 + kBR - 1) / kBR;  // 8-output groups over 66 rows or columns

// Shared-memory areas for the batch's largest radius (floats). A: two gray
// strips of (64 + 2 + 2 max_r + kSlack) rows x kCW, or S (66 x kSS). B: T
// (66 rows x the odd stride 64 + 3 + 2 max_r, 64 spare floats for the x
// chains' reads past the last row).
__host__ __device__ inline int batch_area_a(int max_r) {
  const int strips = 2 * (kBT + 2 + 2 * max_r + kSlack) * kCW;
  return strips > (kBT + 2) * kSS ? strips : (kBT + 2) * kSS;
}
__host__ __device__ inline int batch_area_b(int max_r) {
  return (kBT + 2) * (kBT + 3 + 2 * max_r) + 64;
}

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

__global__ void __launch_bounds__(kBThreads, 3) k_batch_gray_gauss_sobel(const BatchArgs a) {
  extern __shared__ float smf[];
  __shared__ CimxBatchTile s_t;                    // this block's tile
  __shared__ float s_w[kBMaxTaps];                 // this tile's taps
  __shared__ int s_ci[kBT + 2], s_cj[kBT + 2];     // source row / column of each T row, S column
  __shared__ int s_yc[kBG], s_xc[kBG];             // group of 8 with consecutive sources
  const int tid = threadIdx.x;
  // sizes for the batch's largest radius. Area A: two strip buffers of the
  // gray region (kCW columns, kSlack spare rows for the register-blocked
  // chains' reads past the last row), later S. Area B: T (odd row stride,
  // so that lanes on consecutive rows read different banks).
  const int gcs = kBT + 3 + 2 * a.max_r;
  const int gsr = kBT + 2 + 2 * a.max_r + kSlack;
  float* const Gb0 = smf;
  float* const Gb1 = smf + gsr * kCW;
  float* const T = smf + batch_area_a(a.max_r);
  float* const S = smf;

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

    // 1-2. the gray region (rows y0-1-r .., columns x0-1-r .., 'nearest'
    //    borders) and the gaussian along y, in strips of kCW region columns
    //    through two buffers: while the y pass runs on strip s, the words of
    //    strip s + 1 are in flight. Gray: a thread takes groups of 4
    //    consecutive pixels of a row; where they lie inside the row, their
    //    12 bytes come from three or four aligned 32-bit words (each word
    //    holds at least one of the 12 bytes, so it lies in the tile's
    //    allocation), at the tile's borders pixel by pixel. The y pass: T
    //    row tr is the smoothed row refl(y0 - 1 + tr) (rows outside the tile
    //    only feed outputs that are not stored); a thread takes 8
    //    consecutive T rows of one column, one by one where their source
    //    rows are not consecutive (tile borders).
    const int ng = GR * kCG;       // 4-pixel groups of one strip
    const int xb = x0 - 1 - r;     // source column of region column 0
    const int nstrips = (GC + kCW - 1) / kCW;
    uint32_t wv[kGB][4];
    unsigned shv[kGB];
    bool fast[kGB];
    auto gray_load = [&](int st, int i0) {
#pragma unroll
      for (int u = 0; u < kGB; ++u) {
        const int idx = i0 + u * kBThreads;
        const int gr = idx / kCG, c0 = st * kCW + (idx - gr * kCG) * 4;
        const int xs = xb + c0;
        fast[u] = idx < ng && c0 + 3 < GC && xs >= 0 && xs + 3 < W;
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
    };
    auto gray_store = [&](int st, int i0) {
      float* Gs = (st & 1) ? Gb1 : Gb0;
#pragma unroll
      for (int u = 0; u < kGB; ++u) {
        const int idx = i0 + u * kBThreads;
        if (idx >= ng) break;
        const int gr = idx / kCG, cl = (idx - gr * kCG) * 4, c0 = st * kCW + cl;
        if (c0 >= GC) continue;
        float* dst = Gs + gr * kCW + cl;
        if (fast[u]) {
          const unsigned sh = shv[u];
          const uint32_t v0 = __funnelshift_r(wv[u][0], wv[u][1], sh);
          const uint32_t v1 = __funnelshift_r(wv[u][1], wv[u][2], sh);
          const uint32_t v2 = __funnelshift_r(wv[u][2], wv[u][3], sh);
          // one 16-byte store: strip rows are 28 floats and groups start at
          // multiples of 4, so dst is 16-byte aligned
          *reinterpret_cast<float4*>(dst) = make_float4(
              luma_f64(chan(v0 & 255u), chan((v0 >> 8) & 255u), chan((v0 >> 16) & 255u)),
              luma_f64(chan(v0 >> 24), chan(v1 & 255u), chan((v1 >> 8) & 255u)),
              luma_f64(chan((v1 >> 16) & 255u), chan(v1 >> 24), chan(v2 & 255u)),
              luma_f64(chan((v2 >> 8) & 255u), chan((v2 >> 16) & 255u), chan(v2 >> 24)));
        } else {
          const uint8_t* row = t.rgb + static_cast<long long>(nearest_idx(y0 - 1 - r + gr, H)) * in_pitch;
          const int xs = xb + c0;
          for (int p = 0; p < 4 && c0 + p < GC; ++p) {
            const uint8_t* px = row + 3LL * nearest_idx(xs + p, W);
            dst[p] = luma_f64(chan(px[0]), chan(px[1]), chan(px[2]));
          }
        }
      }
    };
    auto ypass = [&](int st) {
      const float* Gs = (st & 1) ? Gb1 : Gb0;
      for (int idx = tid; idx < kBG * kCW; idx += kBThreads) {
        const int q = idx / kCW, cl = idx - q * kCW, c = st * kCW + cl;
        if (c >= GC) continue;
        const int tr0 = q * kBR, nr = min(kBR, kBT + 2 - tr0);
        if (s_yc[q]) {
          float acc[kBR];
#pragma unroll
          for (int p = 0; p < kBR; ++p) acc[p] = 0.f;
          const float* col = Gs + (s_ci[tr0] - r) * kCW + cl;
          chain_r(acc, s_w, K, [&](int i) { return col[i * kCW]; });
#pragma unroll
          for (int p = 0; p < kBR; ++p) T[(tr0 + p) * gcs + c] = acc[p];
        } else {
          for (int p = 0; p < nr; ++p) {
            const float* col = Gs + (s_ci[tr0 + p] - r) * kCW + cl;
            float acc = 0.f;
            for (int k = 0; k < K; ++k) acc = fmaf(col[k * kCW], s_w[k], acc);
            T[(tr0 + p) * gcs + c] = acc;
          }
        }
      }
    };
    for (int i0 = tid; i0 < ng; i0 += kGB * kBThreads) {
      gray_load(0, i0);
      gray_store(0, i0);
    }
    __syncthreads();
    for (int st = 0; st < nstrips; ++st) {
      const bool next = st + 1 < nstrips;  // the same for every thread
      if (next) gray_load(st + 1, tid);
      ypass(st);
      if (next) {
        gray_store(st + 1, tid);
        for (int i0 = tid + kGB * kBThreads; i0 < ng; i0 += kGB * kBThreads) {
          gray_load(st + 1, i0);
          gray_store(st + 1, i0);
        }
      }
      __syncthreads();
    }

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

    // 4-5. edge passes (E0 along y, E1 along x), smoothing passes and the
    //    magnitude, per 4 consecutive outputs of a row: every E0 and E1
    //    value they read comes from the 3 x 6 window of S at (y, x), kept in
    //    registers; each value is the same chain as a separate pass over a
    //    stored E0 / E1 would compute. Lanes take consecutive rows (S's odd
    //    row stride: conflict-free).
    for (int it = tid; it < kBT * (kBT / 4); it += kBThreads) {
      const int y = it % kBT, x = (it / kBT) * 4;
      if (y0 + y >= H || x0 + x >= W) continue;
      float sw[3][6];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 6; ++c) sw[i][c] = S[(y + i) * kSS + x + c];
      float e0[6], e1[3][4];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        float acc = 0.f;
        acc = fmaf(sw[0][c], a.edge[0], acc);
        acc = fmaf(sw[1][c], a.edge[1], acc);
        acc = fmaf(sw[2][c], a.edge[2], acc);
        e0[c] = acc;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float acc = 0.f;
          acc = fmaf(sw[i][c], a.edge[0], acc);
          acc = fmaf(sw[i][c + 1], a.edge[1], acc);
          acc = fmaf(sw[i][c + 2], a.edge[2], acc);
          e1[i][c] = acc;
        }
      float* orow = t.out + static_cast<long long>(y0 + y) * out_pitch + x0 + x;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float d0 = 0.f;
        d0 = fmaf(e0[c], a.smooth[0], d0);
        d0 = fmaf(e0[c + 1], a.smooth[1], d0);
        d0 = fmaf(e0[c + 2], a.smooth[2], d0);
        float d1 = 0.f;
        d1 = fmaf(e1[0][c], a.smooth[0], d1);
        d1 = fmaf(e1[1][c], a.smooth[1], d1);
        d1 = fmaf(e1[2][c], a.smooth[2], d1);
        const float m = __fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1));
        if (x0 + x + c < W) orow[c] = sqrtf(m);
      }
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
  const size_t smem = sizeof(float) * (static_cast<size_t>(batch_area_a(a.max_r)) +
                                       static_cast<size_t>(batch_area_b(a.max_r)));
  // the kernel also holds about 1.2 KB of static shared memory (taps, the
  // row / column tables); the sum stays under the 227 KB per CTA
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
  // resident CTAs per SM: three while the shared memory allows (largest
  // radius up to about 38), two beyond; the grid walks the block list with
  // a stride
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_gray_gauss_sobel, kBThreads,
                                                    smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const long long grid = std::min<long long>(nblocks, static_cast<long long>(per_sm) * sms);
  k_batch_gray_gauss_sobel<<<(unsigned)grid, kBThreads, smem, static_cast<cudaStream_t>(stream)>>>(a);
  return cuda_fail(cudaGetLastError(), "batch launch");
}
