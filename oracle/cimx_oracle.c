/*
 * cimx_oracle.c — TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C CPU restatement of the per-output arithmetic of cuCIM's
 * separable correlation kernels. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU baseline use it; the product never calls it.
 *
 * What it restates (paths relative to python/cucim/src/cucim/skimage):
 *   - boundary index maps: _vendored/_ndimage_util.py:186-308
 *     (reflect/grid-mirror :196-217, mirror :218-247, nearest :248-255,
 *      grid-wrap :256-274, constant :290-307 with the fill value applied as in
 *      _vendored/_ndimage_filters_core.py:334-348 and
 *      filters/_separable_filtering.py:219-223);
 *   - the tap loop: k ascending, sum = sum + (W)x * w[k] contracted to a fused
 *     multiply-add (filters/_separable_filtering.py:728-747 and
 *     _vendored/_ndimage_filters.py:347-360 via
 *     _vendored/_ndimage_filters_core.py:307-309, which also skips zero taps);
 *   - the output cast cast<D>(sum): _vendored/_ndimage_filters_core.py:227-244,
 *     with the saturating float->integer conversion of the GPU
 *     (cvt.rzi; 8-bit results go through a saturating 16-bit conversion and
 *     are then truncated, which is how the CUDA compiler lowers an 8-bit cast).
 *
 * fmaf()/fma() from libm are correctly rounded, so the chain is the exact
 * IEEE fused chain the GPU runs. Build with -ffp-contract=off so that no
 * other expression gets contracted.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { M_REFLECT = 0, M_MIRROR = 1, M_NEAREST = 2, M_GRID_WRAP = 3, M_CONSTANT = 4 };

static inline int64_t map_index(int64_t ix, int64_t n, int mode) {
  switch (mode) {
    case M_REFLECT:
      if (ix < 0) ix = -1 - ix;
      ix %= 2 * n;
      if (2 * n - 1 - ix < ix) ix = 2 * n - 1 - ix;
      return ix;
    case M_MIRROR:
      if (n == 1) return 0;
      if (ix < 0) ix = -ix;
      ix = 1 + (ix - 1) % ((n - 1) * 2);
      if (2 * n - 2 - ix < ix) ix = 2 * n - 2 - ix;
      return ix;
    case M_NEAREST:
      if (ix < 0) return 0;
      if (ix > n - 1) return n - 1;
      return ix;
    case M_GRID_WRAP:
      ix %= n;
      if (ix < 0) ix += n;
      return ix;
    default: /* constant */
      return (ix < 0 || ix >= n) ? -1 : ix;
  }
}

/* ---- element access ------------------------------------------------------ */

static float half_to_float(uint16_t h) {
  uint32_t s = (uint32_t)(h >> 15) << 31;
  uint32_t e = (h >> 10) & 0x1f, m = h & 0x3ff, bits;
  if (e == 0) {
    if (m == 0) {
      bits = s;
    } else { /* subnormal */
      int sh = 0;
      while (!(m & 0x400)) { m <<= 1; ++sh; }
      m &= 0x3ff;
      bits = s | ((uint32_t)(127 - 15 - sh + 1) << 23) | (m << 13);
    }
  } else if (e == 31) {
    bits = s | 0x7f800000u | (m << 13);
  } else {
    bits = s | ((e - 15 + 127) << 23) | (m << 13);
  }
  float f;
  memcpy(&f, &bits, 4);
  return f;
}

/* round-to-nearest-even float -> half */
static uint16_t float_to_half(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  uint32_t s = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(s | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0));
  if (ax >= 0x477ff000u) return (uint16_t)(s | 0x7c00u); /* overflow to inf */
  if (ax < 0x38800000u) { /* subnormal or zero in half */
    float a;
    memcpy(&a, &ax, 4);
    /* half subnormal unit is 2^-24: scale and round to nearest even */
    float q = a * 16777216.0f; /* exact */
    float r = nearbyintf(q);
    return (uint16_t)(s | (uint32_t)r);
  }
  uint32_t mant = ax & 0x7fffffu;
  int32_t e = (int32_t)(ax >> 23) - 127 + 15;
  uint32_t hm = mant >> 13, rem = mant & 0x1fffu;
  uint32_t h = ((uint32_t)e << 10) | hm;
  if (rem > 0x1000u || (rem == 0x1000u && (hm & 1))) h += 1;
  return (uint16_t)(s | h);
}

static inline double load_d(const void* p, int dt, int64_t i) {
  switch (dt) {
    case 'B': return (double)((const uint8_t*)p)[i];
    case 'b': return (double)((const int8_t*)p)[i];
    case '?': return (double)((const uint8_t*)p)[i];
    case 'H': return (double)((const uint16_t*)p)[i];
    case 'h': return (double)((const int16_t*)p)[i];
    case 'I': return (double)((const uint32_t*)p)[i];
    case 'i': return (double)((const int32_t*)p)[i];
    case 'L': case 'Q': return (double)((const uint64_t*)p)[i];
    case 'l': case 'q': return (double)((const int64_t*)p)[i];
    case 'e': return (double)half_to_float(((const uint16_t*)p)[i]);
    case 'f': return (double)((const float*)p)[i];
    default: return ((const double*)p)[i];
  }
}

/* (float)x for every T, converting directly from T (no double rounding). */
static inline float load_f(const void* p, int dt, int64_t i) {
  switch (dt) {
    case 'L': case 'Q': return (float)((const uint64_t*)p)[i];
    case 'l': case 'q': return (float)((const int64_t*)p)[i];
    case 'd': return (float)((const double*)p)[i];
    default: return (float)load_d(p, dt, i);
  }
}

/* static_cast<T>(cval) followed by (W): the shared-memory kernel's fill value. */
double oracle_cval_as_input(double cval, int dt, int w64);

/* GPU float->integer conversion: truncate toward zero, saturate to
 * [lo, hi], NaN -> 0. */
static inline double sat_trunc(double a, double lo, double hi) {
  if (a != a) return 0.0;
  a = trunc(a);
  if (a < lo) return lo;
  if (a > hi) return hi;
  return a;
}

/* Conversion of a float/double value `a` to integer type dt as the CUDA
 * compiler lowers a C cast (8-bit targets: saturating 16-bit conversion, then
 * truncation to 8 bits). Returns the integer as a 64-bit pattern. */
static inline uint64_t c_cast_int(double a, int dt) {
  switch (dt) {
    case 'B': case 'b': case '?': {
      int64_t v = (int64_t)sat_trunc(a, -32768.0, 32767.0);
      return (uint64_t)(uint8_t)v;
    }
    case 'H': return (uint64_t)(uint16_t)(int64_t)sat_trunc(a, 0.0, 65535.0);
    case 'h': return (uint64_t)(uint16_t)(int16_t)(int64_t)sat_trunc(a, -32768.0, 32767.0);
    case 'I': return (uint64_t)(uint32_t)(int64_t)sat_trunc(a, 0.0, 4294967295.0);
    case 'i': return (uint64_t)(uint32_t)(int32_t)(int64_t)sat_trunc(a, -2147483648.0, 2147483647.0);
    case 'L': case 'Q': {
      if (a != a || a <= 0) return 0;
      if (a >= 18446744073709551616.0) return UINT64_MAX;
      return (uint64_t)trunc(a);
    }
    default: { /* int64 */
      if (a != a) return 0;
      if (a >= 9223372036854775808.0) return (uint64_t)INT64_MAX;
      if (a < -9223372036854775808.0) return (uint64_t)INT64_MIN;
      return (uint64_t)(int64_t)trunc(a);
    }
  }
}

static inline int is_unsigned(int dt) {
  return dt == 'B' || dt == 'H' || dt == 'I' || dt == 'L' || dt == 'Q' || dt == '?';
}

static inline void store_bits(void* p, int dt, int64_t i, uint64_t v) {
  switch (dt) {
    case 'B': case 'b': case '?': ((uint8_t*)p)[i] = (uint8_t)v; break;
    case 'H': case 'h': ((uint16_t*)p)[i] = (uint16_t)v; break;
    case 'I': case 'i': ((uint32_t*)p)[i] = (uint32_t)v; break;
    default: ((uint64_t*)p)[i] = v; break;
  }
}

/* cast<D>(a) of _vendored/_ndimage_filters_core.py:227-244 with a in W. */
static inline void store_cast(void* p, int dt, int64_t i, double a, int w64) {
  switch (dt) {
    case 'f': ((float*)p)[i] = (float)a; return;
    case 'd': ((double*)p)[i] = a; return;
    case 'e': ((uint16_t*)p)[i] = float_to_half((float)a); return;
    default: break;
  }
  (void)w64;
  if (is_unsigned(dt)) {
    /* (a >= 0) ? (B)a : -(B)(-a) */
    if (a >= 0) {
      store_bits(p, dt, i, c_cast_int(a, dt));
    } else {
      uint64_t v = c_cast_int(-a, dt);
      store_bits(p, dt, i, (uint64_t)(0 - v));
    }
  } else {
    store_bits(p, dt, i, c_cast_int(a, dt));
  }
}

double oracle_cval_as_input(double cval, int dt, int w64) {
  double t;
  switch (dt) {
    case 'f': t = (double)(float)cval; break;
    case 'd': t = cval; break;
    case 'e': t = (double)half_to_float(float_to_half((float)cval)); break;
    default: {
      /* static_cast<T>(double) for an integer T (saturating, NaN -> 0). */
      uint64_t bits = c_cast_int(cval, dt);
      switch (dt) {
        case 'B': case '?': t = (double)(uint8_t)bits; break;
        case 'b': t = (double)(int8_t)bits; break;
        case 'H': t = (double)(uint16_t)bits; break;
        case 'h': t = (double)(int16_t)bits; break;
        case 'I': t = (double)(uint32_t)bits; break;
        case 'i': t = (double)(int32_t)bits; break;
        case 'L': case 'Q': t = w64 ? (double)bits : (double)(float)bits; break;
        default: t = w64 ? (double)(int64_t)bits : (double)(float)(int64_t)bits; break;
      }
    }
  }
  return w64 ? t : (double)(float)t;
}

/*
 * One 1-D pass over the C-contiguous view (outer, L, inner) of `in`, along
 * the middle axis. taps[] hold the K weights already rounded to W (and
 * already reversed for a convolution); anchor = K/2 + origin; cval_w is the
 * fill value as a W value. threads > 1 splits the lines with OpenMP.
 */
/* n elements of `in` starting at index e, converted as load_f() converts
 * them, into dst (the common input types get a plain loop). */
static inline void load_row_f(const void* in, int tin, int64_t e, int64_t n, float* dst) {
  if (tin == 'f') {
    const float* s = (const float*)in + e;
    for (int64_t i = 0; i < n; ++i) dst[i] = s[i];
  } else if (tin == 'H') {
    const uint16_t* s = (const uint16_t*)in + e;
    for (int64_t i = 0; i < n; ++i) dst[i] = (float)s[i];
  } else if (tin == 'B') {
    const uint8_t* s = (const uint8_t*)in + e;
    for (int64_t i = 0; i < n; ++i) dst[i] = (float)s[i];
  } else {
    for (int64_t i = 0; i < n; ++i) dst[i] = load_f(in, tin, e + i);
  }
}

/* store_cast() of n float32 sums to consecutive elements from index e. */
static inline void store_row_f(void* out, int tout, int64_t e, int64_t n, const float* acc) {
  if (tout == 'f') {
    float* d = (float*)out + e;
    for (int64_t i = 0; i < n; ++i) d[i] = acc[i];
  } else {
    for (int64_t i = 0; i < n; ++i) store_cast(out, tout, e + i, (double)acc[i], 0);
  }
}

/* The float32 chain of oracle_correlate1d, organised for speed: the same
 * k-ascending fmaf() chain per output, with the boundary map evaluated once
 * per (border output, tap) instead of per element. A pass along the last
 * axis converts each line to float32 once and advances the chains of up to
 * ORACLE_LINE_BLOCK consecutive outputs together; a pass along another axis
 * runs over blocks of adjacent lines so that each tap reads a contiguous
 * row. The chains of different outputs are independent, so interleaving
 * them changes no result. Built twice (x86-64-v3 and baseline) and chosen
 * at load time: the hardware FMA of the first clone rounds exactly like
 * fmaf(). */
#define ORACLE_LINE_BLOCK 64
__attribute__((target_clones("arch=x86-64-v3", "default")))
static void corr_f32(const void* in, int tin, void* out, int tout, int64_t outer, int64_t L,
                     int64_t inner, const float* wf, int K, int anchor, float cval_f,
                     int skip_zero, int threads, const int64_t* bmap, int64_t lo_int,
                     int64_t hi_int) {
  /* bmap[(l < lo_int ? l : lo_int + l - hi_int) * K + k]: the mapped index
   * of tap k for the border outputs l < lo_int and l >= hi_int */
  const int64_t nblk = inner == 1 ? 1 : (inner + ORACLE_LINE_BLOCK - 1) / ORACLE_LINE_BLOCK;
  const int64_t nwork = outer * nblk;
#if defined(_OPENMP)
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
#else
  (void)threads;
#endif
  {
    float* line = inner == 1 ? (float*)malloc(sizeof(float) * (size_t)(L > 0 ? L : 1)) : 0;
#if defined(_OPENMP)
#pragma omp for schedule(dynamic, 1)
#endif
    for (int64_t wkey = 0; wkey < nwork; ++wkey) {
      float acc[ORACLE_LINE_BLOCK];
      float row[ORACLE_LINE_BLOCK];
      if (inner == 1) {
        if (!line) continue;
        const int64_t base = wkey * L;
        load_row_f(in, tin, base, L, line);
        for (int64_t l0 = lo_int; l0 < hi_int; l0 += ORACLE_LINE_BLOCK) {
          const int64_t n = hi_int - l0 < ORACLE_LINE_BLOCK ? hi_int - l0 : ORACLE_LINE_BLOCK;
          for (int64_t j = 0; j < n; ++j) acc[j] = 0.0f;
          for (int k = 0; k < K; ++k) {
            const float w = wf[k];
            if (skip_zero && w == 0.0f) continue;
            const float* src = line + l0 - anchor + k;
            for (int64_t j = 0; j < n; ++j) acc[j] = fmaf(src[j], w, acc[j]);
          }
          store_row_f(out, tout, base + l0, n, acc);
        }
        for (int64_t l = 0; l < L; ++l) {
          if (l >= lo_int && l < hi_int) continue;
          const int64_t* bm = bmap + (l < lo_int ? l : lo_int + l - hi_int) * K;
          float s = 0.0f;
          for (int k = 0; k < K; ++k) {
            const float w = wf[k];
            if (skip_zero && w == 0.0f) continue;
            s = fmaf(bm[k] < 0 ? cval_f : line[bm[k]], w, s);
          }
          store_row_f(out, tout, base + l, 1, &s);
        }
        continue;
      }
      const int64_t o = wkey / nblk, i0 = (wkey % nblk) * ORACLE_LINE_BLOCK;
      const int64_t nb = inner - i0 < ORACLE_LINE_BLOCK ? inner - i0 : ORACLE_LINE_BLOCK;
      const int64_t base = o * L * inner + i0;
      for (int64_t l = 0; l < L; ++l) {
        for (int64_t i = 0; i < nb; ++i) acc[i] = 0.0f;
        const int border = l < lo_int || l >= hi_int;
        const int64_t* bm = border ? bmap + (l < lo_int ? l : lo_int + l - hi_int) * K : 0;
        for (int k = 0; k < K; ++k) {
          const float w = wf[k];
          if (skip_zero && w == 0.0f) continue;
          const int64_t ix = border ? bm[k] : l - anchor + k;
          const float* src;
          if (ix < 0) {
            for (int64_t i = 0; i < nb; ++i) row[i] = cval_f;
            src = row;
          } else if (tin == 'f') {
            src = (const float*)in + base + ix * inner;
          } else {
            load_row_f(in, tin, base + ix * inner, nb, row);
            src = row;
          }
          for (int64_t i = 0; i < nb; ++i) acc[i] = fmaf(src[i], w, acc[i]);
        }
        store_row_f(out, tout, base + l * inner, nb, acc);
      }
    }
    free(line);
  }
}

void oracle_correlate1d(const void* in, int tin, void* out, int tout, int64_t outer,
                        int64_t L, int64_t inner, const double* taps, int K, int anchor,
                        int mode, double cval_w, int w64, int skip_zero, int threads) {
  const int64_t nlines = outer * inner;
  if (!w64) {
    /* float32 copies of the taps, any K (heap: tap counts reach the thousands) */
    float* wf = (float*)malloc(sizeof(float) * (size_t)(K > 0 ? K : 1));
    if (!wf) return;
    for (int k = 0; k < K; ++k) wf[k] = (float)taps[k];
    /* outputs l in [lo_int, hi_int) read only in-range inputs */
    int64_t lo_int = anchor < L ? anchor : L;
    int64_t hi_int = L - (K - 1 - anchor);
    if (hi_int < lo_int) hi_int = lo_int;
    const int64_t nborder = lo_int + (L - hi_int);
    int64_t* bmap = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nborder * K > 0 ? nborder * K : 1));
    if (!bmap) {
      free(wf);
      return;
    }
    for (int64_t l = 0; l < L; ++l) {
      if (l >= lo_int && l < hi_int) continue;
      int64_t* bm = bmap + (l < lo_int ? l : lo_int + l - hi_int) * K;
      for (int k = 0; k < K; ++k) bm[k] = map_index(l - anchor + k, L, mode);
    }
    corr_f32(in, tin, out, tout, outer, L, inner, wf, K, anchor, (float)cval_w, skip_zero,
             threads, bmap, lo_int, hi_int);
    free(bmap);
    free(wf);
    return;
  }
#if defined(_OPENMP)
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : 1)
#else
  (void)threads;
#endif
  for (int64_t line = 0; line < nlines; ++line) {
    const int64_t o = line / inner, i = line % inner;
    const int64_t base = o * L * inner + i;
    for (int64_t l = 0; l < L; ++l) {
      double s = 0.0;
      for (int k = 0; k < K; ++k) {
        const double w = taps[k];
        if (skip_zero && w == 0.0) continue;
        const int64_t ix = map_index(l - anchor + k, L, mode);
        double x;
        if (ix < 0) {
          x = cval_w;
        } else {
          const int64_t e = base + ix * inner;
          if (tin == 'L' || tin == 'Q') x = (double)((const uint64_t*)in)[e];
          else if (tin == 'l' || tin == 'q') x = (double)((const int64_t*)in)[e];
          else x = load_d(in, tin, e);
        }
        s = fma(x, w, s);
      }
      store_cast(out, tout, base + l * inner, s, 1);
    }
  }
}

/* Elementwise cast of a W-typed array (float32 when w64 == 0) into dtype dt
 * with cast<D>() semantics; used for checking the cast table alone. */
void oracle_cast(const void* in, int w64, void* out, int tout, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    const double a = w64 ? ((const double*)in)[i] : (double)((const float*)in)[i];
    store_cast(out, tout, i, a, w64);
  }
}

/* The fold of cuCIM's min / max kernels: CUDA's fmin / fmax on the GPU,
 * which behave as IEEE 754-2019 minimumNumber / maximumNumber: a nan
 * operand is ignored (nan only if both are), and -0 orders below +0 whatever
 * the operand order. (The C library's fmin / fmax may return either zero
 * for a pair of opposite-signed zeros; glibc returns the second operand.)
 * Checked against the GPU output on windows that mix -0 and +0. */
static double min_number(double a, double b) {
  if (isnan(a)) return b;
  if (isnan(b)) return a;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}

static double max_number(double a, double b) {
  if (isnan(a)) return b;
  if (isnan(b)) return a;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

/* minimum_filter1d / maximum_filter1d (_vendored/_ndimage_filters.py:1362-1497,
 * _get_min_or_max_kernel without weights): value = x[l] as a double, then
 * every window element in order folded with fmin / fmax (cval outside the
 * array in constant mode), stored with cast<D>(). */
void oracle_min_max1d(const void* in, int tin, void* out, int tout, int64_t outer, int64_t L,
                      int64_t inner, int size, int anchor, int mode, double cval, int is_max) {
  for (int64_t o = 0; o < outer; ++o)
    for (int64_t l = 0; l < L; ++l)
      for (int64_t i = 0; i < inner; ++i) {
        const int64_t base = o * L * inner + i;
        double value = load_d(in, tin, base + l * inner);
        for (int k = 0; k < size; ++k) {
          const int64_t m = map_index(l - anchor + k, L, mode);
          const double v = m < 0 ? cval : load_d(in, tin, base + m * inner);
          value = is_max ? max_number(v, value) : min_number(v, value);
        }
        store_cast(out, tout, base + l * inner, value, 1);
      }
}

/* rgb2gray's kernel body (color/colorconv.py:1038-1046),
 *   gray = 0.2125 * r + 0.7154 * g + 0.0721 * b   (double),
 * as the CUDA compiler evaluates it: cuCIM compiles it with NVRTC's default
 * --fmad=true (CuPy passes no options), which contracts the first product
 * into the first addition and the last product into the second:
 * fma(0.0721, b, fma(0.2125, r, 0.7154 * g)). Checked against the GPU
 * output of the same expression on 4.2 M float32 and uint8 pixels (no
 * other association matched all of them). rgb holds n (r, g, b) triples
 * already converted to double. */
void oracle_rgb2gray(const double* rgb, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    const double r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
    out[i] = fma(0.0721, b, fma(0.2125, r, 0.7154 * g));
  }
}

/* out[i] = fma(a[i], b[i], c[i]) in float32 (w64 == 0) or float64, correctly
 * rounded (libm): the multiply-add chains of cupy.tensordot's GEMM in
 * meijering. */
void oracle_fma(const void* a, const void* b, const void* c, int64_t n, int w64, void* out) {
  for (int64_t i = 0; i < n; ++i) {
    if (w64)
      ((double*)out)[i] = fma(((const double*)a)[i], ((const double*)b)[i], ((const double*)c)[i]);
    else
      ((float*)out)[i] = fmaf(((const float*)a)[i], ((const float*)b)[i], ((const float*)c)[i]);
  }
}

/* One scale of frangi's epilogue (filters/ridges.py:228-319): the sum of
 * squared eigenvalues r_g and the vesselness, for n voxels of nd = 2 or 3
 * eigenvalue images sorted ascending by magnitude, float32 (w64 == 0) or
 * float64. cuCIM's kernels compute r_g = l1*l1; r_g += l2*l2; (r_g += l3*l3;)
 * with the CUDA compiler's contraction, fma(l1, l1, l2*l2) then
 * fma(l3, l3, .), and the exponentials in double with the C math library's
 * exp, which agreed with the GPU's on every one of 2 M voxels. rg (if not
 * NULL) receives r_g; v the vesselness of this scale. */
#define ORACLE_FRANGI_BODY(F, FMA, FMAX, FABS)                                      \
  for (int64_t i = 0; i < n; ++i) {                                                 \
    const F e1 = ((const F*)l1)[i], e2 = ((const F*)l2)[i];                         \
    const F e3 = nd == 3 ? ((const F*)l3)[i] : (F)0;                                \
    F r_g = FMA(e1, e1, e2 * e2);                                                   \
    if (nd == 3) r_g = FMA(e3, e3, r_g);                                            \
    if (rg) ((F*)rg)[i] = r_g;                                                      \
    if (!v) continue;                                                               \
    F result;                                                                       \
    if (nd == 2) {                                                                  \
      F r_b = FABS(e1) / FMAX(e2, (F)1.0e-10);                                      \
      r_b = r_b * r_b;                                                              \
      result = (F)exp(-(double)r_b / beta_sq);                                      \
      result = (F)((double)result * (1.0 - exp(-(double)r_g / gamma_sq)));         \
    } else {                                                                        \
      const F lam2 = FMAX(e2, (F)1.0e-10), lam3 = FMAX(e3, (F)1.0e-10);             \
      F r_a = lam2 / lam3;                                                          \
      r_a = r_a * r_a;                                                              \
      const F r_b = (e1 * e1) / (lam2 * lam3);                                      \
      result = (F)(1.0 - exp(-(double)r_a / alpha_sq));                             \
      result = (F)((double)result * exp(-(double)r_b / beta_sq));                   \
      result = (F)((double)result * (1.0 - exp(-(double)r_g / gamma_sq)));         \
    }                                                                               \
    ((F*)v)[i] = result;                                                            \
  }

void oracle_frangi_scale(const void* l1, const void* l2, const void* l3, int nd, int64_t n,
                         int w64, double alpha_sq, double beta_sq, double gamma_sq, void* rg,
                         void* v) {
  if (w64) {
    ORACLE_FRANGI_BODY(double, fma, fmax, fabs)
  } else {
    ORACLE_FRANGI_BODY(float, fmaf, fmaxf, fabsf)
  }
}
#undef ORACLE_FRANGI_BODY
