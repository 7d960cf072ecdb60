// cimx_slabw.cuh — the (y, x) passes of float32 slabs on a persistent,
// warp-specialised kernel (k_slabw).
//
// k_slab (cimx_fast.cuh) stages one tile per CTA and separates its phases
// (tile load, border patch, y pass, x pass) with CTA-wide barriers; with 2-3
// CTAs per SM the FMA pipe stays about a fifth busy (barrier stalls ~1/3 of
// the samples). Here one CTA per SM walks a list of 64 x 128 output tiles:
//   - a producer warp issues each tile's TMA load into a ring of two input
//     stages (full / empty mbarriers), up to two tiles ahead;
//   - eight consumer warps each own 8 output rows of the tile: a warp patches
//     the border halo of the rows it reads itself (values from outside its
//     rows come from HBM, as in k_slab's fallback), runs the y pass for its
//     rows over all staged columns into its private rows of the intermediate,
//     releases the stage, and runs the x pass from its own intermediate rows.
//     The hand-off between the passes is a __syncwarp: no CTA-wide barrier
//     in the steady state, and every wait is a bounded mbarrier wait.
// The arithmetic is k_slab's: the same k-ascending FMA chains (chain2, f32x2
// pairs), the intermediate rounded through the output type, the same
// boundary values, so the results are bit-identical.
#pragma once

#include "cimx_fast.cuh"

namespace cimx {
namespace fast {

constexpr int kWTY = 64;   // output rows per tile: 8 consumer warps x P rows
constexpr int kWTX = 128;  // output columns per tile
constexpr int kWCW = 8;    // consumer warps
constexpr int kWNS = 2;    // input stages
constexpr int kWThreads = 32 * (kWCW + 1);
constexpr int kWMaxKB = 48;  // longest pass (taps rounded up to 8) it takes
static_assert(kWTY == kWCW * P, "each consumer warp owns P output rows");

template <int KB>
struct GeomW {
  static constexpr int RY = kWTY + KB;            // staged rows
  static constexpr int RX = kWTX + KB;            // staged columns
  static constexpr int NPAIR = RX / 2 + 1;        // y-pass column pairs (one spare for sh)
  static constexpr int RXQ = pad8(RX + 2);        // intermediate row-pair stride (float2)
  static constexpr int BX = (RX + 4 + 3) / 4 * 4;  // TMA box width >= RX + off + 1
  static constexpr int BY = RY;
  static constexpr int RAW = BX * BY * 4;          // bytes of one stage
  static constexpr int RAWP = (RAW + 127) / 128 * 128;
  static constexpr int MIDW = (P / 2) * RXQ;       // float2 per consumer warp
  static constexpr int OFF_W = 128;                // after the mbarriers and the abort flag
  static constexpr int OFF_RAW = (OFF_W + 2 * KB * 8 + 127) / 128 * 128;
  static constexpr int OFF_MID = OFF_RAW + kWNS * RAWP;
  static constexpr int SMEM = OFF_MID + kWCW * MIDW * 8;
  static_assert(SMEM <= kMaxSmem, "k_slabw shared memory");
  static_assert(BX <= 256 && BY <= 256, "TMA box extents");
};

struct TileW {
  long long b, y0, x0, ys, xst, xs;
  int off;
};

__device__ __forceinline__ TileW tile_w(const SlabArgs& a, long long t) {
  TileW w;
  const long long per_slab = a.tiles_x * a.tiles_y;
  w.b = t / per_slab;
  const long long r = t - w.b * per_slab;
  w.y0 = (r / a.tiles_x) * kWTY;
  w.x0 = (r % a.tiles_x) * kWTX;
  w.ys = w.y0 - a.py.anchor;
  w.xst = w.x0 - a.px.anchor;
  w.xs = floor_div(w.xst, 4) * 4;  // 16-byte aligned TMA start column
  w.off = static_cast<int>(w.xst - w.xs);
  return w;
}

template <int KB>
__global__ void __launch_bounds__(kWThreads, 1)
    k_slabw(const __grid_constant__ CUtensorMap map, const SlabArgs a) {
  using G = GeomW<KB>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kWNS;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kWNS);
  f2* wy = reinterpret_cast<f2*>(smem + G::OFF_W);
  f2* wx = wy + KB;
  float* raw0 = reinterpret_cast<float*>(smem + G::OFF_RAW);
  f2* mid0 = reinterpret_cast<f2*>(smem + G::OFF_MID);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (tid == 0) {
    for (int s = 0; s < kWNS; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, kWCW);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  for (int k = tid; k < KB; k += blockDim.x) {
    const float ty_ = k < a.py.K ? a.py.w[k] : 0.f;
    const float tx_ = k < a.px.K ? a.px.w[k] : 0.f;
    wy[k] = pack2(ty_, ty_);
    wx[k] = pack2(tx_, tx_);
  }
  __syncthreads();  // the only CTA-wide barrier
  const long long ntiles = a.B * a.tiles_x * a.tiles_y;

  if (warp == kWCW) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      long long it = 0;
      for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        if (*abort_flag) break;
        const int s = static_cast<int>(it % kWNS);
        if (it >= kWNS &&
            !mbar_wait(empty + s, static_cast<uint32_t>(((it / kWNS) - 1) & 1), a.status)) {
          *abort_flag = 1;
          break;
        }
        const TileW w = tile_w(a, t);
        fence_proxy_async_smem();
        mbar_expect_tx(full + s, G::RAW);
        tma_load_3d(raw0 + s * (G::RAWP / 4), &map, full + s, static_cast<int>(w.xs),
                    static_cast<int>(w.ys), static_cast<int>(w.b));
      }
      // copies still in flight (consumers that gave up no longer wait for
      // them) land before the CTA leaves: the last kWNS issued stages
      for (long long j = it > kWNS ? it - kWNS : 0; j < it; ++j)
        mbar_wait(full + j % kWNS, static_cast<uint32_t>((j / kWNS) & 1), nullptr);
    }
    return;
  }

  // ----------------------------------------------------------- consumers
  const int my = a.py.mode, mx = a.px.mode;
  const float cy = fill_value<float>(a.py.cval, a.py.cval_as_input, a.py.dt);
  const float cx = fill_value<float>(a.px.cval, a.px.cval_as_input, a.px.dt);
  const int rg = warp * P;  // this warp's output rows in the tile
  f2* mid = mid0 + warp * G::MIDW;
  auto clampi = [](long long v, long long lo, long long hi) {
    return static_cast<int>(v < lo ? lo : (v > hi ? hi : v));
  };
  long long it = 0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = static_cast<int>(it % kWNS);
    const bool ok = mbar_wait(full + s, static_cast<uint32_t>((it / kWNS) & 1), a.status);
    if (!__all_sync(0xffffffffu, ok) || *abort_flag) {
      if (lane == 0) *abort_flag = 1;
      break;
    }
    const TileW w = tile_w(a, t);
    const float* in = static_cast<const float*>(a.in) + w.b * a.Y * a.X;
    float* out = static_cast<float*>(a.out) + w.b * a.Y * a.X;
    float* raw = raw0 + s * (G::RAWP / 4);
    const int off = w.off;
    const int sh = off & 1;
    // staged columns [cl, cr) and rows [rl, rr) lie inside the array
    const int cl = clampi(-w.xst, 0, G::RX);
    const int cr = clampi(a.X - w.xst, cl, G::RX);
    const int rl = clampi(-w.ys, 0, G::RY);
    const int rr = clampi(a.Y - w.ys, rl, G::RY);

    // 1. border halo of the rows this warp's y chains read
    if (!(rl == 0 && rr == G::RY && cl == 0 && cr == G::RX)) {
      const int r_lo = rg, r_hi = min(G::RY, rg + P + a.py.K - 1);
      // 1a. rows inside the array: columns outside take the value of the
      //     column they map to (staged, or from HBM); x-constant columns 0
      const int ra = max(r_lo, rl), rb = min(r_hi, rr);
      const int nleft = cl, nout = cl + (G::RX - cr);
      for (int q = lane; q < (rb - ra) * nout; q += 32) {
        const int r = ra + q / nout, j = q % nout;
        const int c = j < nleft ? j : cr + (j - nleft);
        float* row = raw + r * G::BX + off;
        const long long xm = map_coord_near(w.xst + c, a.X, mx);
        float v = 0.f;
        if (xm >= 0) {
          const long long sc = xm - w.xst;
          v = (sc >= cl && sc < cr) ? row[sc] : in[(w.ys + r) * a.X + xm];
        }
        row[c] = v;
      }
      __syncwarp();
      // 1b. rows outside the array: the fill value (constant mode), or the
      //     row they map to (this warp's patched copy when it holds it, else
      //     from HBM)
      for (int r = r_lo; r < r_hi; ++r) {
        if (r >= rl && r < rr) continue;
        const long long ym = map_coord_near(w.ys + r, a.Y, my);
        const long long sr = ym - w.ys;
        float* row = raw + r * G::BX + off;
        for (int c = lane; c < G::RX; c += 32) {
          float v;
          if (ym < 0) v = cy;
          else if (sr >= ra && sr < rb) v = raw[sr * G::BX + off + c];
          else v = staged_value<float>(in, w.ys + r, w.xst + c, a, my, mx, cy);
          row[c] = v;
        }
      }
      __syncwarp();
    }

    // 2. y pass: this warp's P rows, one column pair per item, into its
    //    intermediate rows (as row pairs, rounded through the output type)
    {
      const int soff = off - sh;
      const int npair = (G::RX + sh + 1) / 2;
      for (int m = lane; m < npair; m += 32) {
        const int e = 2 * m;
        f2 acc[P];
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = 0ull;
        const f2* col = reinterpret_cast<const f2*>(raw + rg * G::BX + soff + e);
        chain2(acc, wy, a.py.K, a.py.skip,
               [&](int qb, int j) { return col[(qb + j) * (G::BX / 2)]; });
        const long long gx = w.xst + e - sh;
        const bool f0 = mx == CIMX_MODE_CONSTANT && (gx < 0 || gx >= a.X);
        const bool f1 = mx == CIMX_MODE_CONSTANT && (gx + 1 < 0 || gx + 1 >= a.X);
        f2* d0 = mid + pad8(e);
        f2* d1 = mid + pad8(e + 1);
#pragma unroll
        for (int p = 0; p < P; p += 2) {
          const float a0 = f0 ? cx : lo2(acc[p]);
          const float b0 = f0 ? cx : lo2(acc[p + 1]);
          const float a1 = f1 ? cx : hi2(acc[p]);
          const float b1 = f1 ? cx : hi2(acc[p + 1]);
          d0[(p / 2) * G::RXQ] = pack2(a0, b0);
          d1[(p / 2) * G::RXQ] = pack2(a1, b1);
        }
      }
    }
    // the stage is free once every warp's y pass is done with it; this
    // warp's patch writes are ordered before the next TMA write into it
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive1(empty + s);

    // 3. x pass: this warp's row pairs x 8 consecutive outputs per item
    constexpr int gpr = kWTX / P;
    for (int item = lane; item < (P / 2) * gpr; item += 32) {
      const int rp = item / gpr;
      const int g = (item % gpr) * P;
      f2 acc[P];
#pragma unroll
      for (int p = 0; p < P; ++p) acc[p] = 0ull;
      const f2* row = mid + rp * G::RXQ + pad8(g);
      if (sh)
        chain2(acc, wx, a.px.K, a.px.skip,
               [&](int qb, int j) { return row[pad8(qb) + (j + 1) + ((j + 1) >> 3)]; });
      else
        chain2(acc, wx, a.px.K, a.px.skip, [&](int qb, int j) { return row[pad8(qb) + j]; });
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long yy = w.y0 + rg + 2 * rp + h;
        if (yy >= a.Y) continue;
        float* orow = out + yy * a.X + w.x0 + g;
        const long long left = a.X - (w.x0 + g);
        float v[P];
#pragma unroll
        for (int p = 0; p < P; ++p) v[p] = h ? hi2(acc[p]) : lo2(acc[p]);
        if (left >= P && ((reinterpret_cast<uintptr_t>(orow) & 15) == 0)) {
          store4<float>(orow, v[0], v[1], v[2], v[3]);
          store4<float>(orow + 4, v[4], v[5], v[6], v[7]);
        } else {
#pragma unroll
          for (int p = 0; p < P; ++p)
            if (p < left) orow[p] = v[p];
        }
      }
    }
    __syncwarp();  // the intermediate rows are rewritten by the next tile
  }
}

template <int KB>
int launch_slabw_kb(SlabArgs& a, cudaStream_t st) {
  using G = GeomW<KB>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(k_slabw<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                G::SMEM);
  });
  if (attr != cudaSuccess) return CIMX_FUSED_DECLINED;
  a.tiles_x = (a.X + kWTX - 1) / kWTX;
  a.tiles_y = (a.Y + kWTY - 1) / kWTY;
  const long long ntiles = a.B * a.tiles_x * a.tiles_y;
  if (ntiles == 0) return CIMX_OK;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if (!make_tensor_map_3d(&map, a.in, DT_F32, a.X, a.Y, a.B, G::BX, G::BY))
    return CIMX_FUSED_DECLINED;  // not TMA-eligible: the one-tile kernel stages by plain loads
  if (a.B >= (1LL << 31) || a.Y >= (1LL << 31) || a.X >= (1LL << 31)) return CIMX_FUSED_DECLINED;
  a.status = device_status_word();
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long grid = std::min<long long>(ntiles, sms);
  k_slabw<KB><<<(unsigned)grid, kWThreads, G::SMEM, st>>>(map, a);
  return cuda_fail(cudaGetLastError(), "slab launch");
}

// float32 -> float32 (y, x) passes with up to kWMaxKB taps each (after
// rounding up to 8); CIMX_FUSED_DECLINED when the kernel does not apply
inline int launch_slabw(SlabArgs& a, cudaStream_t st) {
  if (a.no_slabw || !a.has_y || !a.has_x) return CIMX_FUSED_DECLINED;
  const int k8 = std::max(a.py.K8, a.px.K8);
  if (k8 <= 8) return launch_slabw_kb<8>(a, st);
  if (k8 <= 16) return launch_slabw_kb<16>(a, st);
  if (k8 <= 24) return launch_slabw_kb<24>(a, st);
  if (k8 <= 32) return launch_slabw_kb<32>(a, st);
  if (k8 <= 40) return launch_slabw_kb<40>(a, st);
  if (k8 <= kWMaxKB) return launch_slabw_kb<48>(a, st);
  return CIMX_FUSED_DECLINED;
}

}  // namespace fast
}  // namespace cimx
