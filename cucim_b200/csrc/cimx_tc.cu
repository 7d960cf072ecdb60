// cimx_tc.cu — the split-precision tensor-core path for long 1-D passes
// (float32 in, float32 out), on sm_100a's tcgen05 MMA with TMEM accumulators.
//
// A pass y[l] = sum_k w[k] x[l - anchor + k] over a tile of 128 consecutive
// outputs l0..l0+127 and 64 independent lines is the matrix product
//   D[m][n] = sum_j T[m][j] X[j][n],   T[m][j] = w[j - m] (0 <= j - m < K),
// with X[j][n] = input at coordinate l0 - anchor + j of line n. j runs over
// S = ceil((128 + K - 1) / 16) slices of 16. The banded Toeplitz operand of
// slice s is T[m][16s + c] = w[16s + c - m]; all slices are windows of one
// tall band B[r][c] = w[c + R0 - r] (R0 = 16 (S - 1)), slice s starting at
// row R0 - 16s, so the band costs (16 S + 112) x 16 elements of shared memory.
//
// Precision: every operand is split into bfloat16 hi + lo (x = hi + lo up to
// 2^-17 |x|) and D accumulates hi*hi + hi*lo + lo*hi in float32 (BF16x3).
// The result is not bit-identical to cuCIM's float32 chain; its error against
// float64 is measured and reported by the tests and the bench.
//
// Operand layouts (no swizzle, "interleaved" canonical UMMA layouts; a core
// matrix is 8 rows x 16 bytes stored as 128 contiguous bytes):
//   band (A, K-major):           (r/8)*256 + (c/8)*128 + (r%8)*16 + (c%8)*2
//                                 LBO = 128 (next 8 c), SBO = 256 (next 8 r)
//   tile, strided axis (B, MN-major, line n contiguous in memory):
//                                 (n/8)*256S + (j/8)*128 + (j%8)*16 + (n%8)*2
//                                 LBO = 128 (next 8 j), SBO = 256 S (next 8 n)
//   tile, contiguous axis (B, K-major, coordinate j contiguous in memory):
//                                 (j/8)*1024 + n*16 + (j%8)*2
//                                 LBO = 1024 (next 8 j), SBO = 128 (next 8 n)
// One thread issues the 3 S MMAs (128 x 64 x 16 each), commits them to an
// mbarrier and waits (bounded); four warps then read the 128 x 64 float32
// accumulator from TMEM and store it.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"
#include "cimx_tc.h"
#include "cimx_tma.cuh"

namespace cimx {
namespace {

constexpr int kTcM = 128;       // outputs per tile (MMA M)
constexpr int kTcN = 64;        // lines per tile (MMA N)
constexpr int kTcMaxS = 32;     // slices: K <= 16 * 32 - 127 = 385
constexpr int kTcThreads = 128;
constexpr int kTcMaxTaps = kTcMaxS * 16 - kTcM + 1;

struct TcArgs {
  const float* in;
  float* out;
  long long outer, L, inner;  // strided: view (outer, L, inner); contiguous: rows = outer, L = X
  int K, S, anchor, mode;
  float cval;
  int* status;
  float w[kTcMaxTaps];
};

// ---------------------------------------------------------------- PTX

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // start address, leading / stride byte offsets (all >> 4), version 1,
  // base offset 0, no swizzle
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D f32, A and B bf16, M = 128, N = 64
__host__ __device__ constexpr uint32_t idesc_bf16(bool b_mn_major) {
  return (1u << 4)                          // D format: f32
         | (1u << 7)                        // A format: bf16
         | (1u << 10)                       // B format: bf16
         | (0u << 15)                       // A K-major
         | ((b_mn_major ? 1u : 0u) << 16)   // B major
         | ((uint32_t)(kTcN >> 3) << 17)    // N
         | ((uint32_t)(kTcM >> 4) << 24);   // M
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------- helpers

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// 8 floats -> 16 bytes of bf16 hi at dh and 16 bytes of bf16 lo at dl
__device__ __forceinline__ void put8(unsigned char* dh, unsigned char* dl, const float (&v)[8]) {
  __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) split_bf16(v[i], h[i], l[i]);
  *reinterpret_cast<uint4*>(dh) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(dl) = *reinterpret_cast<const uint4*>(l);
}

struct TcSmem {
  int S, RT;
  uint32_t band_bytes, tile_bytes;
  uint32_t off_bh, off_bl, off_th, off_tl, total;
};

__host__ __device__ inline TcSmem tc_layout(int S) {
  TcSmem L;
  L.S = S;
  L.RT = 16 * (S - 1) + kTcM;
  L.band_bytes = (uint32_t)L.RT * 32;
  L.tile_bytes = (uint32_t)(16 * S) * kTcN * 2;
  L.off_bh = 128;  // mbarrier and TMEM address slot first
  L.off_bl = L.off_bh + (L.band_bytes + 127) / 128 * 128;
  L.off_th = L.off_bl + (L.band_bytes + 127) / 128 * 128;
  L.off_tl = L.off_th + (L.tile_bytes + 127) / 128 * 128;
  L.total = L.off_tl + L.tile_bytes;
  return L;
}

// CONTIG = false: pass along the middle axis of (outer, L, inner); a tile is
// 128 outputs along L x 64 consecutive inner positions.
// CONTIG = true: pass along the last axis of (outer rows, L); a tile is 128
// outputs along the row x 64 consecutive rows.
template <bool CONTIG>
__global__ void __launch_bounds__(kTcThreads) k_tc_pass(const TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const TcSmem G = tc_layout(a.S);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 64);
  unsigned char* band_h = sm + G.off_bh;
  unsigned char* band_l = sm + G.off_bl;
  unsigned char* tile_h = sm + G.off_th;
  unsigned char* tile_l = sm + G.off_tl;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const long long l0 = (long long)blockIdx.x * kTcM;  // first output along the pass axis
  const long long n0 = (long long)blockIdx.y * kTcN;  // first line
  const long long o = blockIdx.z;                     // outer index (strided form)
  const long long nlines = CONTIG ? a.outer : a.inner;

  // TMEM: 64 float32 columns x 128 lanes, allocated by warp 0
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tslot)),
                 "r"(kTcN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }

  // band: B[r][c] = w[c + R0 - r] split into hi / lo (zero outside the taps)
  const int R0 = 16 * (a.S - 1);
  for (int idx = tid; idx < G.RT * 2; idx += kTcThreads) {
    const int r = idx >> 1, cc = idx & 1;  // 8-column chunk cc of row r
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int k = cc * 8 + e + R0 - r;
      v[e] = (k >= 0 && k < a.K) ? a.w[k] : 0.f;
    }
    const uint32_t off = (r >> 3) * 256 + cc * 128 + (r & 7) * 16;
    put8(band_h + off, band_l + off, v);
  }

  // input tile: 16 S coordinates x 64 lines, boundary modes applied
  const int J = 16 * a.S;
  if (!CONTIG) {
    // line n = inner position n0 + n, contiguous in memory: one thread loads
    // 8 lines of one coordinate j
    const float* base = a.in + o * a.L * a.inner;
    for (int idx = tid; idx < J * (kTcN / 8); idx += kTcThreads) {
      const int j = idx % J, g = idx / J;
      const long long c = l0 - a.anchor + j;
      const long long m = (c >= 0 && c < a.L) ? c : map_coord(c, a.L, a.mode);
      float v[8];
      const long long i = n0 + 8 * g;
      if (m < 0) {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = a.cval;
      } else {
        const float* src = base + m * a.inner + i;
        if (i + 8 <= a.inner && (a.inner & 3) == 0) {
          const float4 p = *reinterpret_cast<const float4*>(src);
          const float4 q = *reinterpret_cast<const float4*>(src + 4);
          v[0] = p.x; v[1] = p.y; v[2] = p.z; v[3] = p.w;
          v[4] = q.x; v[5] = q.y; v[6] = q.z; v[7] = q.w;
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) v[e] = (i + e < a.inner) ? src[e] : 0.f;
        }
      }
      const uint32_t off = g * (256u * a.S) + (j >> 3) * 128 + (j & 7) * 16;
      put8(tile_h + off, tile_l + off, v);
    }
  } else {
    // line n = row n0 + n; coordinates along the row: one thread loads 8
    // consecutive coordinates of one row
    for (int idx = tid; idx < (J / 8) * kTcN; idx += kTcThreads) {
      const int n = idx % kTcN, cc = idx / kTcN;
      const long long row = n0 + n;
      float v[8];
      if (row < nlines) {
        const float* src = a.in + row * a.L;
        const long long c0 = l0 - a.anchor + 8 * cc;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const long long c = c0 + e;
          const long long m = (c >= 0 && c < a.L) ? c : map_coord(c, a.L, a.mode);
          v[e] = m < 0 ? a.cval : src[m];
        }
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = 0.f;
      }
      const uint32_t off = cc * 1024 + n * 16;
      put8(tile_h + off, tile_l + off, v);
    }
  }

  // make the generic-proxy writes visible to the tensor core, then issue
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  int ok = 1;
  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(!CONTIG);
    const uint32_t bh = smem_addr(band_h), bl = smem_addr(band_l);
    const uint32_t th = smem_addr(tile_h), tl = smem_addr(tile_l);
    const uint32_t tile_lbo = CONTIG ? 1024u : 128u;
    const uint32_t tile_sbo = CONTIG ? 128u : 256u * a.S;
    for (int s = 0; s < a.S; ++s) {
      const uint32_t aoff = (uint32_t)((R0 - 16 * s) >> 3) * 256;
      const uint32_t boff = CONTIG ? (uint32_t)s * 2048 : (uint32_t)s * 256;
      const uint64_t ah = smem_desc(bh + aoff, 128, 256), al = smem_desc(bl + aoff, 128, 256);
      const uint64_t xh = smem_desc(th + boff, tile_lbo, tile_sbo);
      const uint64_t xl = smem_desc(tl + boff, tile_lbo, tile_sbo);
      tc_mma(tmem, ah, xh, idesc, s > 0 ? 1u : 0u);  // hi * hi
      tc_mma(tmem, ah, xl, idesc, 1u);               // hi * lo
      tc_mma(tmem, al, xh, idesc, 1u);               // lo * hi
    }
    tc_commit(bar);
    ok = mbar_wait(bar, 0, a.status) ? 1 : 0;
  }
  ok = __syncthreads_and(ok);
  tc_fence_after();

  if (ok) {
    // warp w owns TMEM lanes 32w..32w+31 = outputs l0 + 32w + lane
    const long long l = l0 + 32 * warp + lane;
    const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int q = 0; q < kTcN / 16; ++q) {
      float v[16];
      tmem_ld16(trow + 16 * q, v);
      if (l < a.L) {
        if (!CONTIG) {
          float* dst = a.out + (o * a.L + l) * a.inner + n0 + 16 * q;
          const long long left = a.inner - (n0 + 16 * q);
          if (left >= 16 && (a.inner & 3) == 0) {
#pragma unroll
            for (int e = 0; e < 16; e += 4)
              *reinterpret_cast<float4*>(dst + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (e < left) dst[e] = v[e];
          }
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const long long row = n0 + 16 * q + e;
            if (row < nlines) a.out[row * a.L + l] = v[e];
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcN)
                 : "memory");
}

}  // namespace

bool tc_supports(const PassDesc& d) {
  if (d.w64 || d.tin != DT_F32 || d.tout != DT_F32) return false;
  if (d.K < 1 || d.K > kTcMaxTaps) return false;
  return true;
}

int launch_tc_pass(const PassDesc& d, cudaStream_t st) {
  if (!tc_supports(d)) return fail(CIMX_E_INVALID, "tensor-core pass: unsupported pass");
  TcArgs a{};
  a.in = static_cast<const float*>(d.in);
  a.out = static_cast<float*>(d.out);
  a.K = d.K;
  a.S = (kTcM + d.K - 1 + 15) / 16;
  a.anchor = d.anchor;
  a.mode = d.mode;
  // fill value of constant mode: float32 input, so both of cuCIM's rules agree
  a.cval = static_cast<float>(d.cval);
  a.status = device_status_word();
  for (int k = 0; k < d.K; ++k) a.w[k] = static_cast<float>(d.taps[k]);
  const bool contig = d.inner == 1;
  const TcSmem L = tc_layout(a.S);
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_tc_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    cudaFuncSetAttribute(k_tc_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  });
  if (L.total > 227u * 1024u) return fail(CIMX_E_INVALID, "tensor-core pass: tile too large");
  const long long tiles_l = (d.L + kTcM - 1) / kTcM;
  if (contig) {
    a.outer = d.outer;
    a.L = d.L;
    a.inner = 1;
    const long long tiles_n = (d.outer + kTcN - 1) / kTcN;
    if (tiles_n > 65535 || tiles_l > 0x7fffffff) return fail(CIMX_E_INVALID, "tensor-core pass: grid");
    if (tiles_l * tiles_n == 0) return CIMX_OK;
    k_tc_pass<true><<<dim3((unsigned)tiles_l, (unsigned)tiles_n, 1), kTcThreads, L.total, st>>>(a);
  } else {
    a.outer = d.outer;
    a.L = d.L;
    a.inner = d.inner;
    const long long tiles_n = (d.inner + kTcN - 1) / kTcN;
    if (tiles_n > 65535 || d.outer > 65535) return fail(CIMX_E_INVALID, "tensor-core pass: grid");
    if (tiles_l * tiles_n * d.outer == 0) return CIMX_OK;
    k_tc_pass<false><<<dim3((unsigned)tiles_l, (unsigned)tiles_n, (unsigned)d.outer), kTcThreads,
                       L.total, st>>>(a);
  }
  return cuda_fail(cudaGetLastError(), "tensor-core pass launch");
}

}  // namespace cimx
