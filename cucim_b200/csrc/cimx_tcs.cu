// cimx_tcs.cu — the streaming TF32x3 tensor-core pass for long float32 1-D
// filters on sm_100a: persistent, warp-specialised CTAs fed by TMA, with
// tcgen05 MMAs accumulating in tensor memory (TMEM).
//
// Arithmetic. A pass y[l] = sum_k w[k] x[l - anchor + k] over a block of BO
// consecutive outputs is the product of a banded Toeplitz matrix
// T[p][j] = w[j - p] with the block's input window (j = 0 .. BO + K - 2).
// j is cut into slices of 8 coordinates (one tf32 MMA step); every slice of
// T is a window of one tall band Bd[r][c] = w[c + R0 - r] (R0 = 8 (SB - 1),
// SB slices per block), slice t starting at row R0 - 8t, so the band is
// built once per CTA. Operands are split into tf32 pieces, x = hi + lo with
// hi = x rounded to tf32 (cvt.rna) and lo = x - hi (exact in float32); the
// MMAs accumulate hi*hi + hi*lo + lo*hi in float32 (TF32x3). The dropped
// lo*lo term and the tf32 reading of lo leave a relative error per product
// of about 2^-21. The tensor core rounds its float32 accumulator toward zero
// as it aligns each product to the accumulator, a bias toward zero that
// grows with the number of products summed into one accumulator at full
// magnitude; hi*hi therefore accumulates alone, spread over NHH accumulators
// (slice tt into accumulator tt mod NHH: 1 up to 64 taps, 2 up to 160, else
// 3), and the two small cross terms go to one more accumulator; the epilogue
// adds them with round-to-nearest. The result is not bit-identical to cuCIM's float32
// chain.
//
// Streaming. A CTA owns a contiguous range of the flattened (strip, block)
// sequence, where a strip is NL neighbouring lines and a block 128 outputs
// along them, and walks it in runs along each strip: the input window of a
// run is staged once, slice after slice, and every staged slice feeds each
// of the (at most ceil(SB / 16)) blocks whose window covers it, each block
// accumulating in its own TMEM slot (2 NL columns: hi*hi, cross terms). A
// block whose last slice has been multiplied is committed to the epilogue
// while later blocks accumulate. D[output][line] = T * X: the band is the A
// operand (M = 128 outputs), the data the B operand (N = NL lines).
//
// Layout in shared memory. TMA loads raw float32 input tiles with the
// 128-byte swizzle. Every data operand is K-major with that swizzle (rows =
// lines, 128 bytes = the 32 coordinates of one stage per row, SBO 1024);
// tcgen05 kind::tf32 reads MN-major operands as zeros on this part, so the
// coordinate axis must be the contiguous one:
//   pass along the last axis ("contiguous"): box {32 coordinates, NL rows}
//     is already that layout; converters round it to tf32 in place (hi) and
//     write lo at the same offsets of a second buffer;
//   pass along another axis ("strided"): NL/32 boxes {32 lines, 32
//     coordinates} arrive line-contiguous; converters transpose 4 x 4
//     blocks into separate hi and lo tiles.
// Coordinates outside the axis are patched with the boundary mode first.
// The band is K-major without swizzle:
//   (r/8)*256 + (c/4)*128 + (r%8)*16 + (c%4)*4, LBO 128, SBO 256.
//
// Roles (448 threads): warps 0-3 epilogue (TMEM -> registers -> global),
// warp 4 TMEM allocation and the single MMA-issuing thread, warp 5 the TMA
// thread, warps 6-13 converters. Every wait is bounded by a 2 s deadline on
// %globaltimer; a timeout records CIMX_E_TIMEOUT in the device status word,
// raises a CTA-wide abort flag and every role leaves its loop.
#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "cimx_common.cuh"
#include "cimx_internal.h"
#include "cimx_tc.h"
#include "cimx_tma.cuh"

namespace cimx {
namespace {

constexpr int kChunk = 32;          // coordinates per pipeline stage
constexpr int kSlicesPerChunk = 4;  // tf32 MMA steps of 8 coordinates
constexpr int kBPS = 16;            // slices per block step (128 outputs)
constexpr int kMaxStages = 8;
constexpr int kMaxSlots = 8;
// warps 0-3 epilogue, 4-6 MMA issue (one thread each, on three different SM
// sub-partitions), 7 TMA, 8-15 converters
constexpr int kMmaWarp = 4, kIssuers = 3, kTmaWarp = 7, kConvWarp0 = 8, kConvWarps = 8;
constexpr int kThreads = 32 * (kConvWarp0 + kConvWarps);  // 512
constexpr int kConvThreads = 32 * kConvWarps;
constexpr int kTcsMaxTaps = 452;  // taps after the alignment shift
constexpr uint64_t kTcsWaitNs = 2000000000ull;

struct TcsArgs {
  const float* in;
  float* out;
  long long rows;  // contiguous: number of lines; strided: outer extent
  long long L, inner;
  long long nblk;          // output blocks per line
  long long total;         // strips * nblk
  long long strips_per_o;  // strided: strips per outer index
  int K, anchor, mode;     // taps and anchor after the alignment shift
  int SB, BO, NL, NB, NACC, NST;  // BO = 128 outputs per block; NB = TMEM columns per slot
  int NHH;                        // hi*hi accumulators per block (1-3, by slice tt mod NHH)
  int use_tma, vec_out;
  uint32_t off_band_lo, off_stage0, stage_bytes, raw_bytes;
  uint32_t off_hi;  // offset of the hi tile in a stage (0: in place over the raw tile)
  float cval;
  int* status;
  float w[kTcsMaxTaps];
};

// ---------------------------------------------------------------- PTX

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait (`limit_ns` of %globaltimer); false on timeout (recorded) or
// when another role aborted.
__device__ __noinline__ bool wait_bar(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                      int* status, uint64_t limit_ns = kTcsWaitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (gtimer() - t0 > limit_ns) {
        if (abort_flag) *abort_flag = 1;
        if (status) atomicExch(status, -6 /* CIMX_E_TIMEOUT */);
        return false;
      }
    }
  }
}

// AND of `pred` over the converter warps (named barrier 1).
__device__ __forceinline__ int conv_all(int pred) {
  int r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.s32 p, %1, 0;\n"
      " barrier.cta.red.and.pred q, 1, %2, p;\n selp.s32 %0, 1, 0, q;\n}"
      : "=r"(r)
      : "r"(pred), "n"(kConvThreads)
      : "memory");
  return r;
}

__device__ __forceinline__ void conv_sync() {
  asm volatile("barrier.cta.sync 1, %0;" ::"n"(kConvThreads) : "memory");
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ uint64_t desc_plain(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return desc_plain(addr, lbo, sbo) | (2ull << 61);  // layout type SWIZZLE_128B
}

// kind::tf32 instruction descriptor: D f32, A and B tf32, both K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes (one per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset inside a 1024-byte-aligned tile written with the 128-byte swizzle
__device__ __forceinline__ uint32_t swz128(uint32_t off) {
  return off ^ (((off >> 7) & 7u) << 4);
}

// ------------------------------------------------------------- the kernel

struct Run {
  long long o, n0, b0, nb;  // outer index, first line, first block, blocks
};

__device__ __forceinline__ Run make_run(const TcsArgs& a, bool contig, long long t, long long t_end) {
  Run r;
  const long long strip = t / a.nblk;
  r.b0 = t - strip * a.nblk;
  r.nb = min(a.nblk - r.b0, t_end - t);
  if (contig) {
    r.o = 0;
    r.n0 = strip * a.NL;
  } else {
    r.o = strip / a.strips_per_o;
    r.n0 = (strip - r.o * a.strips_per_o) * a.NL;
  }
  return r;
}

template <bool CONTIG>
__global__ void __launch_bounds__(kThreads, 1)
    k_tcs_pass(const __grid_constant__ CUtensorMap map, const __grid_constant__ TcsArgs a) {
  extern __shared__ unsigned char sm_raw[];
  // 1024-byte alignment for the swizzled tiles
  unsigned char* sm = sm_raw + ((1024u - (smem_addr(sm_raw) & 1023u)) & 1023u);
  uint64_t* full_tma = reinterpret_cast<uint64_t*>(sm);
  uint64_t* full_cv = full_tma + kMaxStages;
  uint64_t* empty = full_cv + kMaxStages;
  uint64_t* accf = empty + kMaxStages;
  uint64_t* acce = accf + kMaxSlots;
  uint64_t* done = acce + kMaxSlots;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  unsigned char* band_hi = sm + 1024;
  unsigned char* band_lo = sm + a.off_band_lo;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int R0 = 8 * (a.SB - 1);       // band row of slice 0
  const int RT = R0 + a.BO;            // band rows
  int tmem_cols = 32;
  while (tmem_cols < a.NACC * a.NB) tmem_cols <<= 1;

  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tslot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < kMaxStages; ++i) {
      mbar_init(&full_tma[i], 1);
      mbar_init(&full_cv[i], kConvThreads);
      mbar_init(&empty[i], kIssuers);
    }
    for (int i = 0; i < kMaxSlots; ++i) {
      mbar_init(&accf[i], 1);
      mbar_init(&acce[i], 128);
    }
    mbar_init(done, kIssuers);
    *abort_flag = 0;
    mbar_fence_init();
  }
  // the band, split into tf32 hi and lo: Bd[r][c] = w[c + R0 - r]
  for (int idx = tid; idx < RT * 2; idx += kThreads) {
    const int r = idx >> 1, cc = idx & 1;
    uint32_t h[4];
    float l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = cc * 4 + e + R0 - r;
      const float v = (k >= 0 && k < a.K) ? a.w[k] : 0.f;
      h[e] = to_tf32(v);
      l[e] = __uint_as_float(to_tf32(v - __uint_as_float(h[e])));
    }
    const uint32_t off = (r >> 3) * 256 + cc * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(band_hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(band_lo + off) = make_float4(l[0], l[1], l[2], l[3]);
  }
  fence_proxy_async_smem();
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tmem = *tslot;

  const long long t_begin = (long long)blockIdx.x * a.total / gridDim.x;
  const long long t_end = (long long)(blockIdx.x + 1) * a.total / gridDim.x;
  const int SB = a.SB;

  if (warp == kTmaWarp) {
    // ------------------------------------------------------------ TMA
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;           // parity of the stage ring's current round
      long long issued = 0;      // chunks issued
      bool ok = true;
      for (long long t = t_begin; t < t_end && ok;) {
        const Run r = make_run(a, CONTIG, t, t_end);
        t += r.nb;
        const long long x0 = r.b0 * 128 - a.anchor;
        const int nch = ((int)(r.nb - 1) * kBPS + SB + kSlicesPerChunk - 1) / kSlicesPerChunk;
        for (int c = 0; c < nch; ++c) {
          // the previous round's chunk in this stage has been multiplied
          if (issued >= a.NST && !wait_bar(&empty[st], ph ^ 1u, abort_flag, a.status)) {
            ok = false;
            break;
          }
          unsigned char* raw = sm + a.off_stage0 + st * a.stage_bytes;
          if (a.use_tma) {
            mbar_expect_tx(&full_tma[st], a.raw_bytes);
            const int xc = (int)(x0 + kChunk * c);
            if (CONTIG) {
              tma_load_3d(raw, &map, &full_tma[st], xc, (int)r.n0, 0);
            } else {
              for (int q = 0; q < a.NL / 32; ++q)
                tma_load_3d(raw + q * 4096, &map, &full_tma[st], (int)r.n0 + 32 * q, xc, (int)r.o);
            }
          } else {
            mbar_arrive(&full_tma[st]);
          }
          ++issued;
          if (++st == a.NST) {
            st = 0;
            ph ^= 1u;
          }
        }
      }
      // TMA loads still in flight land before the CTA exits
      for (long long g = issued - a.NST < 0 ? 0 : issued - a.NST; g < issued; ++g)
        wait_bar(&full_tma[g % a.NST], (uint32_t)((g / a.NST) & 1), nullptr, nullptr);
    }
  } else if (warp >= kMmaWarp && warp < kMmaWarp + kIssuers) {
    // ------------------------------------------------------------ MMA
    // Three threads issue the MMAs, block gbi by thread gbi % 3, so that one
    // block's MMAs, and its commit, come from one thread in order; every
    // issuer commits every stage (the stage-free barrier counts three).
    // Everything the issue loop needs is held in registers and advanced by
    // additions.
    if (lane == 0) {
      const uint32_t me = (uint32_t)(warp - kMmaWarp);
      const int nl = a.NL, nhh = a.NHH, nst = a.NST;
      const uint32_t nacc = (uint32_t)a.NACC, acc_mask = nacc - 1u;
      const int acc_shift = __ffs(a.NACC) - 1;
      const uint32_t slot_cols = (uint32_t)a.NB;
      const uint32_t idesc = idesc_tf32(128, nl);
      // band operand of slice tt: (SB - 1 - tt) * 256 bytes past the band start
      const uint64_t wh0 = desc_plain(smem_addr(band_hi), 128, 256) + (uint64_t)(16 * (SB - 1));
      const uint64_t wl0 = desc_plain(smem_addr(band_lo), 128, 256) + (uint64_t)(16 * (SB - 1));
      const uint32_t stage0 = smem_addr(sm + a.off_stage0);
      const uint32_t stage_bytes = a.stage_bytes, off_hi = a.off_hi, raw_bytes = a.raw_bytes;
      int st = 0;
      uint32_t ph = 0;
      uint32_t gb = 0;  // blocks started before this run
      bool ok = true;
      for (long long t = t_begin; t < t_end && ok;) {
        const Run r = make_run(a, CONTIG, t, t_end);
        t += r.nb;
        const int nb = (int)r.nb;
        const int nsl = (nb - 1) * kBPS + SB;
        const int nch = (nsl + kSlicesPerChunk - 1) / kSlicesPerChunk;
        for (int c = 0; c < nch && ok; ++c) {
          if (!wait_bar(&full_cv[st], ph, abort_flag, a.status)) {
            ok = false;
            break;
          }
          tmem_fence_after();
          const uint32_t raw = stage0 + (uint32_t)st * stage_bytes;
          // data operand of slice u of this stage: 32 bytes further along each row
          const uint64_t xh = desc_sw128(raw + off_hi, 16, 1024);
          const uint64_t xl = desc_sw128(raw + raw_bytes, 16, 1024);
          const int s0 = c * kSlicesPerChunk;
          const int u_lim = min(kSlicesPerChunk, nsl - s0);
          // blocks whose window meets slices s0 .. s0 + 3 (a block never starts
          // inside a stage: block starts are multiples of 16 slices)
          const int i_first = s0 < SB ? 0 : ((s0 - SB) >> 4) + 1;
          const int i_last = min(nb - 1, (s0 + kSlicesPerChunk - 1) >> 4);
          for (int i = i_first; i <= i_last; ++i) {
            const uint32_t gbi = gb + (uint32_t)i;
            if (gbi % kIssuers != me) continue;
            const int tt0 = s0 - kBPS * i;  // band slice of u = 0
            const int u_end = min(u_lim, SB - tt0);
            const uint32_t slot = gbi & acc_mask;
            if (tt0 == 0 && gbi >= nacc) {
              if (!wait_bar(&acce[slot], ((gbi >> acc_shift) - 1u) & 1u, abort_flag, a.status)) {
                ok = false;
                break;
              }
              tmem_fence_after();
            }
            // slot: [hi*hi accumulators 0 .. NHH-1 (slice tt into tt mod NHH)][cross terms]
            const uint32_t d_slot = tmem + slot * slot_cols;
            const uint32_t d_x = d_slot + (uint32_t)(nhh * nl);
            const uint64_t wh = wh0 - (uint64_t)(16 * tt0), wl = wl0 - (uint64_t)(16 * tt0);
            int hsel = tt0 % nhh;
#pragma unroll
            for (int u = 0; u < kSlicesPerChunk; ++u, hsel = (hsel + 1 == nhh) ? 0 : hsel + 1) {
              if (u < u_end) {
                const int tt = tt0 + u;
                const uint32_t d_hh = d_slot + (uint32_t)(hsel * nl);
                mma_tf32(d_hh, wh - 16 * u, xh + 2 * u, idesc, tt >= nhh ? 1u : 0u);  // hi * hi
                mma_tf32(d_x, wh - 16 * u, xl + 2 * u, idesc, tt > 0 ? 1u : 0u);      // hi * lo
                mma_tf32(d_x, wl - 16 * u, xh + 2 * u, idesc, 1u);                    // lo * hi
              }
            }
            if (tt0 + u_end == SB) mma_commit(&accf[slot]);
          }
          mma_commit(&empty[st]);
          if (++st == nst) {
            st = 0;
            ph ^= 1u;
          }
        }
        gb += (uint32_t)nb;
      }
      // every MMA issued has completed before TMEM is released
      mma_commit(done);
      wait_bar(done, 0, nullptr, nullptr);
    }
  } else if (warp >= kConvWarp0) {
    // ------------------------------------------------------ converters
    const int ct = tid - 32 * kConvWarp0;
    int st = 0;
    uint32_t ph = 0;
    bool ok = true;
    for (long long t = t_begin; t < t_end && ok;) {
      const Run r = make_run(a, CONTIG, t, t_end);
      t += r.nb;
      const long long x0 = r.b0 * 128 - a.anchor;
      const int nch = ((int)(r.nb - 1) * kBPS + SB + kSlicesPerChunk - 1) / kSlicesPerChunk;
      for (int c = 0; c < nch; ++c) {
        const int got = wait_bar(&full_tma[st], ph, abort_flag, a.status) ? 1 : 0;
        if (!conv_all(got)) {
          ok = false;
          break;
        }
        unsigned char* raw = sm + a.off_stage0 + st * a.stage_bytes;
        unsigned char* rlo = raw + a.raw_bytes;
        const long long xc = x0 + kChunk * c;
        if (!a.use_tma || xc < 0 || xc + kChunk > a.L) {
          // coordinates outside the axis (or everything without TMA)
          if (CONTIG) {
            for (int idx = ct; idx < kChunk * a.NL; idx += kConvThreads) {
              const int j = idx & 31, n = idx >> 5;
              const long long cc = xc + j;
              const bool inr = cc >= 0 && cc < a.L;
              if (inr && a.use_tma) continue;
              const long long row = r.n0 + n;
              float v = 0.f;
              if (row < a.rows) {
                const long long m = inr ? cc : map_coord(cc, a.L, a.mode);
                v = m < 0 ? a.cval : a.in[row * a.L + m];
              }
              *reinterpret_cast<float*>(raw + swz128((uint32_t)(n * 128 + j * 4))) = v;
            }
          } else {
            const int nl_shift = a.NL == 128 ? 7 : a.NL == 64 ? 6 : 5;
            for (int idx = ct; idx < kChunk * a.NL; idx += kConvThreads) {
              const int n = idx & (a.NL - 1), j = idx >> nl_shift;
              const long long cc = xc + j;
              const bool inr = cc >= 0 && cc < a.L;
              if (inr && a.use_tma) continue;
              const long long line = r.n0 + n;
              float v = 0.f;
              if (line < a.inner) {
                const long long m = inr ? cc : map_coord(cc, a.L, a.mode);
                v = m < 0 ? a.cval : a.in[(r.o * a.L + m) * a.inner + line];
              }
              *reinterpret_cast<float*>(
                  raw + swz128((uint32_t)((n >> 5) * 4096 + j * 128 + (n & 31) * 4))) = v;
            }
          }
          conv_sync();
        }
        if (CONTIG) {
          // split in place: raw <- tf32(x), lo <- x - tf32(x); the swizzle
          // is the same for both tiles, so physical offsets are used directly
          const uint32_t nvec = a.raw_bytes >> 4;
#pragma unroll 4
          for (uint32_t p = ct; p < nvec; p += kConvThreads) {
            const float4 v = *reinterpret_cast<const float4*>(raw + 16 * p);
            const uint32_t h0 = to_tf32(v.x), h1 = to_tf32(v.y), h2 = to_tf32(v.z),
                           h3 = to_tf32(v.w);
            *reinterpret_cast<uint4*>(raw + 16 * p) = make_uint4(h0, h1, h2, h3);
            *reinterpret_cast<float4*>(rlo + 16 * p) =
                make_float4(v.x - __uint_as_float(h0), v.y - __uint_as_float(h1),
                            v.z - __uint_as_float(h2), v.w - __uint_as_float(h3));
          }
        } else if (ct < 2 * a.NL) {
          // transpose 4 coordinates x 4 lines per thread into the K-major hi
          // and lo tiles. Phase (8 threads) p = 0..7 takes coordinate quad p
          // and line quad 8g + (p + s) % 8: conflict-free reads and writes.
          unsigned char* rhi = raw + a.off_hi;
          const int phs = ct >> 3, p = ct & 7;
          const int jq = p, nq = 8 * (phs >> 3) + ((p + (phs & 7)) & 7);
          float4 v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
            v[i] = *reinterpret_cast<const float4*>(
                raw + swz128((uint32_t)((nq >> 3) * 4096 + (4 * jq + i) * 128 + (nq & 7) * 16)));
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            float cv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
              cv[i] = e == 0 ? v[i].x : e == 1 ? v[i].y : e == 2 ? v[i].z : v[i].w;
            const uint32_t h0 = to_tf32(cv[0]), h1 = to_tf32(cv[1]), h2 = to_tf32(cv[2]),
                           h3 = to_tf32(cv[3]);
            const uint32_t off = swz128((uint32_t)((4 * nq + e) * 128 + jq * 16));
            *reinterpret_cast<uint4*>(rhi + off) = make_uint4(h0, h1, h2, h3);
            *reinterpret_cast<float4*>(rlo + off) =
                make_float4(cv[0] - __uint_as_float(h0), cv[1] - __uint_as_float(h1),
                            cv[2] - __uint_as_float(h2), cv[3] - __uint_as_float(h3));
          }
        }
        fence_proxy_async_smem();
        mbar_arrive(&full_cv[st]);
        if (++st == a.NST) {
          st = 0;
          ph ^= 1u;
        }
      }
    }
  } else {
    // -------------------------------------------------------- epilogue
    const uint32_t acc_mask = (uint32_t)a.NACC - 1u;
    const int acc_shift = __ffs(a.NACC) - 1;
    uint32_t gb = 0;
    bool ok = true;
    for (long long t = t_begin; t < t_end && ok;) {
      const Run r = make_run(a, CONTIG, t, t_end);
      t += r.nb;
      for (int i = 0; i < (int)r.nb; ++i) {
        const uint32_t gbi = gb + (uint32_t)i;
        const uint32_t slot = gbi & acc_mask;
        // warp-uniform outcome: the TMEM loads below are warp-collective
        if (!__all_sync(0xffffffffu, wait_bar(&accf[slot], (gbi >> acc_shift) & 1u, abort_flag,
                                              a.status))) {
          ok = false;
          break;
        }
        tmem_fence_after();
        const long long lb = (r.b0 + i) * 128;
        const uint32_t tbase = tmem + ((uint32_t)(32 * warp) << 16) + slot * (uint32_t)a.NB;
        const long long l = lb + 32 * warp + lane;  // this thread's output
        const int nq = a.NL / 32;
        auto store_group = [&](int q, const float (&v)[32]) {
          if (l >= a.L) return;
          const long long n = r.n0 + 32 * q;  // first line of this column group
          if (CONTIG) {
            // lines are rows: a warp stores 32 consecutive outputs of a row
            float* dst = a.out + n * a.L + l;
#pragma unroll
            for (int e = 0; e < 32; ++e)
              if (n + e < a.rows) dst[e * a.L] = v[e];
          } else {
            float* dst = a.out + (r.o * a.L + l) * a.inner + n;
            if (a.vec_out && n + 32 <= a.inner) {
#pragma unroll
              for (int e = 0; e < 32; e += 4)
                *reinterpret_cast<float4*>(dst + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
            } else {
#pragma unroll
              for (int e = 0; e < 32; ++e)
                if (n + e < a.inner) dst[e] = v[e];
            }
          }
        };
        auto sum_group = [&](int q, float (&v)[32]) {
          const uint32_t col = tbase + 32 * q;
          float x[32];
          tmem_ld32(col, v);
          for (int h = 1; h <= a.NHH; ++h) {
            tmem_ld32(col + h * a.NL, x);
#pragma unroll
            for (int e = 0; e < 32; ++e) v[e] = __fadd_rn(v[e], x[e]);
          }
        };
        if (nq <= 2) {
          // read every column group, release the slot, then store: the MMA
          // threads wait for this slot when the ring has no spare one
          float v0[32], v1[32];
          sum_group(0, v0);
          if (nq == 2) sum_group(1, v1);
          tmem_fence_before();
          mbar_arrive(&acce[slot]);
          store_group(0, v0);
          if (nq == 2) store_group(1, v1);
        } else {
          // per column group; the slot is released after the last group's reads
          for (int q = 0; q < nq; ++q) {
            float v[32];
            sum_group(q, v);
            if (q == nq - 1) {
              tmem_fence_before();
              mbar_arrive(&acce[slot]);
            }
            store_group(q, v);
          }
        }
      }
      gb += (uint32_t)r.nb;
    }
  }

  tmem_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tmem_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

// ----------------------------------------------------------------- host

struct TcsPlan {
  bool contig;
  int delta, K, anchor, BO, NL, NB, SB, NACC, NST, NHH;
  uint32_t raw_bytes, stage_bytes, off_band_lo, off_stage0, smem;
};

constexpr uint32_t kSmemLimit = 227u * 1024u;

bool plan_tcs(const PassDesc& d, TcsPlan& p) {
  if (d.w64 || d.tin != DT_F32 || d.tout != DT_F32 || d.K < 1) return false;
  p.contig = d.inner == 1;
  p.delta = p.contig ? (((-d.anchor) % 4) + 4) % 4 : 0;
  p.K = d.K + p.delta;
  p.anchor = d.anchor + p.delta;
  if (p.K > kTcsMaxTaps) return false;
  // hi*hi accumulators per block: splitting the sum over NHH accumulators
  // divides the round-toward-zero bias of the float32 accumulation by NHH
  p.NHH = p.K <= 64 ? 1 : p.K <= 160 ? 2 : 3;
  p.BO = 128;
  p.SB = (p.BO + p.K - 1 + 7) / 8;
  const int need = (p.SB + 15) / 16;  // blocks a slice feeds at most
  // lines per strip: the widest whose ring of slots (a power of two, NB =
  // (NHH + 1) NL TMEM columns each) holds every block a slice feeds; wider
  // strips make larger MMAs, which outweighs waiting for the epilogue when
  // the ring has no spare slot (the epilogue frees a slot before its stores)
  for (int pass = 1; pass < 2; ++pass) {
    for (int nl : {128, 64, 32}) {
      p.NL = nl;
      p.NB = (p.NHH + 1) * nl;
      int nacc = 1;
      while (nacc * 2 * p.NB <= 512 && nacc * 2 <= kMaxSlots) nacc *= 2;
      p.NACC = nacc;
      if (p.NACC < (pass == 0 ? need + 1 : need)) continue;
      const int RT = 8 * (p.SB - 1) + p.BO;
      p.raw_bytes = (uint32_t)p.NL * 128u;
      p.stage_bytes = (p.contig ? 2u : 3u) * p.raw_bytes;  // raw(=hi), lo [, hi]
      p.off_band_lo = 1024u + (uint32_t)RT * 32u;
      p.off_stage0 = (p.off_band_lo + (uint32_t)RT * 32u + 1023u) / 1024u * 1024u;
      if (p.off_stage0 + 2 * p.stage_bytes + 1024u > kSmemLimit) continue;
      p.NST = (int)std::min<uint32_t>(kMaxStages,
                                      (kSmemLimit - 1024u - p.off_stage0) / p.stage_bytes);
      p.smem = p.off_stage0 + p.NST * p.stage_bytes + 1024u;
      return true;
    }
  }
  return false;
}

int sm_count() {
  static int n[64] = {0};
  static std::mutex mu;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64) return 148;
  if (!n[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    n[dev] = v > 0 ? v : 148;
  }
  return n[dev];
}

}  // namespace

bool tcs_supports(const PassDesc& d) {
  TcsPlan p;
  return plan_tcs(d, p);
}

int launch_tcs_pass(const PassDesc& d, cudaStream_t st) {
  TcsPlan p;
  if (!plan_tcs(d, p)) return fail(CIMX_E_INVALID, "tensor-core pass: unsupported pass");
  TcsArgs a{};
  a.in = static_cast<const float*>(d.in);
  a.out = static_cast<float*>(d.out);
  a.L = d.L;
  a.K = p.K;
  a.anchor = p.anchor;
  a.mode = d.mode;
  a.cval = static_cast<float>(d.cval);
  a.status = device_status_word();
  for (int k = 0; k < p.delta; ++k) a.w[k] = 0.f;
  for (int k = 0; k < d.K; ++k) a.w[p.delta + k] = static_cast<float>(d.taps[k]);
  a.SB = p.SB;
  a.BO = p.BO;
  a.NL = p.NL;
  a.NB = p.NB;
  a.NACC = p.NACC;
  a.NHH = p.NHH;
  a.NST = p.NST;
  a.raw_bytes = p.raw_bytes;
  a.stage_bytes = p.stage_bytes;
  a.off_band_lo = p.off_band_lo;
  a.off_stage0 = p.off_stage0;
  a.off_hi = p.contig ? 0u : 2u * p.raw_bytes;
  a.nblk = (d.L + a.BO - 1) / a.BO;
  if (d.L >= (1ll << 31)) return fail(CIMX_E_INVALID, "tensor-core pass: axis too long");
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  const bool aligned_out = (reinterpret_cast<uintptr_t>(d.out) & 15) == 0;
  if (p.contig) {
    a.rows = d.outer;
    a.inner = 1;
    a.strips_per_o = 1;
    const long long strips = (d.outer + a.NL - 1) / a.NL;
    a.total = strips * a.nblk;
    if (d.outer >= (1ll << 31)) return fail(CIMX_E_INVALID, "tensor-core pass: too many lines");
    a.use_tma =
        make_tensor_map_3d(&map, d.in, DT_F32, d.L, d.outer, 1, kChunk, a.NL, true) ? 1 : 0;
    a.vec_out = (aligned_out && d.L % 4 == 0) ? 1 : 0;
  } else {
    a.rows = d.outer;
    a.inner = d.inner;
    a.strips_per_o = (d.inner + a.NL - 1) / a.NL;
    a.total = d.outer * a.strips_per_o * a.nblk;
    if (d.inner >= (1ll << 31) || d.outer >= (1ll << 31))
      return fail(CIMX_E_INVALID, "tensor-core pass: extent too large");
    a.use_tma =
        make_tensor_map_3d(&map, d.in, DT_F32, d.inner, d.L, d.outer, 32, kChunk, true) ? 1 : 0;
    a.vec_out = (aligned_out && d.inner % 4 == 0) ? 1 : 0;
  }
  if (a.total == 0) return CIMX_OK;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(k_tcs_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kSmemLimit);
    cudaFuncSetAttribute(k_tcs_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kSmemLimit);
  });
  const long long grid = std::min<long long>(a.total, sm_count());
  if (p.contig)
    k_tcs_pass<true><<<(unsigned)grid, kThreads, p.smem, st>>>(map, a);
  else
    k_tcs_pass<false><<<(unsigned)grid, kThreads, p.smem, st>>>(map, a);
  return cuda_fail(cudaGetLastError(), "tensor-core pass launch");
}

}  // namespace cimx

// ------------------------------------------------ bounded-wait self-test
//
// One CTA, one thread: an mbarrier expecting one arrival that nothing ever
// makes, waited on with the same helpers the TMA-fed kernels use (poll-count
// bound, `which` 0) or the tensor-core pass uses (%globaltimer bound, `which`
// 1). The wait runs out after `limit` polls / nanoseconds, records
// CIMX_E_TIMEOUT in the device status word and the kernel returns; no copy or
// MMA is in flight, so the context stays usable.
namespace cimx {
namespace {

__global__ void k_wait_selftest(int which, long long limit, int* status) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  abort_flag = 0;
  mbar_fence_init();
  bool ok;
  if (which == 0)
    ok = mbar_wait(&bar, 0, status, limit);
  else
    ok = wait_bar(&bar, 0, &abort_flag, status, (uint64_t)limit);
  // the barrier cannot have completed: nothing arrived on it
  if (ok && status) atomicExch(status, -1 /* CIMX_E_INVALID: the wait did not run out */);
}

}  // namespace
}  // namespace cimx

extern "C" CIMX_API int cimx_wait_selftest(int which, long long limit, void* stream) {
  using namespace cimx;
  if (which != 0 && which != 1) return fail(CIMX_E_INVALID, "which must be 0 or 1");
  // at most 2^24 polls or 0.1 s: the self-test must end quickly
  const long long cap = which == 0 ? (1ll << 24) : 100000000ll;
  if (limit < 1 || limit > cap)
    return fail(CIMX_E_INVALID, "limit out of range (1.." + std::to_string(cap) + ")");
  int* status = device_status_word();
  if (!status) return fail(CIMX_E_CUDA, "no device status word");
  k_wait_selftest<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(which, limit, status);
  return cuda_fail(cudaGetLastError(), "wait self-test launch");
}
