/*
 * cimx.h — C ABI of libcimx.so, the B200 (sm_100a) separable n-D filtering
 * library behind the cucim_b200 Python package.
 *
 * Every entry point takes plain pointers and sizes, enqueues its work on the
 * CUDA stream it is given (a cudaStream_t passed as void*, NULL = legacy
 * default stream) and returns 0 on success or a negative CIMX_E* code.
 * cimx_last_error_string() describes the last failure on the calling thread.
 * Nothing here synchronises the stream unless the comment says so.
 *
 * The arithmetic each entry performs is the arithmetic of the cuCIM code it
 * replaces (paths are relative to python/cucim/src/cucim/skimage in
 * rapidsai/cucim):
 *   - taps are applied in ascending order as one fused multiply-add chain
 *     per output, sum = fma(x[k], w[k], sum), starting from +0, in the
 *     weights type W (float32 or float64);
 *   - the result is stored with cuCIM's cast<D>() rule
 *     (_vendored/_ndimage_filters_core.py:227-244);
 *   - boundary modes follow _vendored/_ndimage_util.py:186-308.
 */
#ifndef CIMX_H_
#define CIMX_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CIMX_API __attribute__((visibility("default")))
#else
#define CIMX_API
#endif

#define CIMX_MAX_NDIM 8

/* Element types: the numpy dtype.char of the array ('B','b','H','h','I','i',
 * 'L'/'Q','l'/'q','e','f','d'). cimx_correlate1d and cimx_separable also take
 * complex64 'F' and complex128 'D' (cuCIM's complex<float> / complex<double>
 * kernels, _vendored/_ndimage_util.py:35-37: W is complex whenever the input or
 * the weights are; the output must then be complex). */
typedef struct CimxArray {
  void* data;                       /* device pointer */
  int32_t dtype;                    /* numpy dtype.char, e.g. 'f' */
  int32_t ndim;                     /* 0..CIMX_MAX_NDIM */
  int64_t shape[CIMX_MAX_NDIM];
  int64_t strides[CIMX_MAX_NDIM];   /* bytes */
} CimxArray;

/* Boundary modes (filters map 'wrap' to 'grid-wrap' before calling). */
enum {
  CIMX_MODE_REFLECT = 0,   /* 'reflect' == 'grid-mirror'  (d c b a | a b c d | d c b a) */
  CIMX_MODE_MIRROR = 1,    /* 'mirror'                    (d c b | a b c d | c b a)   */
  CIMX_MODE_NEAREST = 2,   /* 'nearest'                   (a a a | a b c d | d d d)   */
  CIMX_MODE_GRID_WRAP = 3, /* 'grid-wrap' (and 'wrap' for filters) (a b c d | a b c d) */
  CIMX_MODE_CONSTANT = 4,  /* 'constant'                  (k k k | a b c d | k k k)   */
};

/* Per-pass flags. */
enum {
  CIMX_F_W64 = 1 << 0,          /* weights type W is float64 (else float32) */
  CIMX_F_CONVOLVE = 1 << 1,     /* taps are applied reversed (convolve1d) */
  CIMX_F_CVAL_AS_INPUT = 1 << 2,/* constant mode: halo value is (W)(T)cval as in the
                                   shared-memory kernel (filters/_separable_filtering.py:219-223);
                                   otherwise (W)cval as in the elementwise kernel
                                   (_vendored/_ndimage_filters_core.py:334-348) */
  CIMX_F_SKIP_ZERO_TAPS = 1 << 3,/* zero taps are skipped, as the elementwise kernel does
                                   (_vendored/_ndimage_filters_core.py:307-309) */
  CIMX_F_COMPLEX_TAPS = 1 << 4, /* `taps` holds K (re, im) pairs: complex weights. W is then
                                   complex<float> (complex<double> with CIMX_F_W64); the
                                   output must be complex64 or complex128. The taps are used
                                   as given: correlate1d's conjugation of complex weights
                                   (_vendored/_ndimage_filters.py:242-244) is the caller's */
};

/* Library-level flags for multi-pass calls. */
enum {
  CIMX_L_NO_FUSION = 1 << 0,    /* force one launch per pass (ping-pong through scratch) */
  CIMX_L_TENSOR_BF16X3 = 1 << 1,/* run float32 -> float32 passes with at least 16 taps along
                                   lines of at least 2048 samples (where they measured faster
                                   than the plain kernels) on the
                                   tensor cores: banded-Toeplitz products of bfloat16 hi/lo
                                   splits, float32 accumulation (not bit-identical to the
                                   float32 chain; an addition of this library) */
  CIMX_L_TENSOR_TF32X3 = 1 << 2,/* the same on tf32 hi/lo splits (hi*hi + hi*lo + lo*hi), in a
                                   streaming TMA-fed kernel: about ten times more accurate
                                   than BF16X3 (a relative error per product near 2^-21) and
                                   faster; takes precedence when both bits are set */
  CIMX_L_TENSOR_ALL_LINES = 1 << 3,/* with a tensor bit: every eligible pass on the tensor
                                   cores whatever its line length (testing, measurement) */
  /* Schedule choices. Each selects between kernels that give bit-identical
   * results; the autotuner (cimx_tune_*) picks among them per call signature. */
  CIMX_L_NO_VOLUME = 1 << 4,    /* 3-D short filters: stream + slab launches instead of the
                                   single-launch volume kernel */
  CIMX_L_NO_STREAM = 1 << 5,    /* leading-axis passes on the generic kernel, not k_stream */
  CIMX_L_NO_ROWSTREAM = 1 << 6, /* (y, x) passes on the slab kernel, not the row stream */
  CIMX_L_NO_TUNE = 1 << 7,      /* this call neither consults nor fills the tuning table */
  CIMX_L_ZCHUNK_SHIFT = 8,      /* bits 8-9: volume-kernel z chunk, 0 = automatic,
                                   1/2/3 = 32/64/128 slices */
  CIMX_L_SLAB_SPAN_SHIFT = 10,  /* bits 10-11: slabs each slab-kernel CTA walks (float
                                   input), 0 = automatic (about 4), 1/2/3 = 1/2/8 */
};

/* One 1-D correlation pass of a separable filter. */
typedef struct CimxPass {
  int32_t axis;        /* axis of the input it runs along */
  int32_t ntaps;       /* K >= 1 */
  int32_t origin;      /* cuCIM origin; anchor = K/2 + origin (after the convolve flip) */
  int32_t mode;        /* CIMX_MODE_* */
  double cval;         /* constant-mode fill value as given by the caller */
  int32_t flags;       /* CIMX_F_* */
  int32_t reserved;
  const double* taps;  /* host pointer to K taps (rounded to W inside) */
} CimxPass;

/* Error codes. */
enum {
  CIMX_OK = 0,
  CIMX_E_INVALID = -1,     /* bad argument (shape, axis, mode, ntaps, origin) */
  CIMX_E_DTYPE = -2,       /* unsupported element type */
  CIMX_E_CUDA = -3,        /* a CUDA call failed */
  CIMX_E_NOMEM = -4,       /* scratch allocation failed */
  CIMX_E_LAYOUT = -5,      /* array is not C-contiguous where required */
  CIMX_E_TIMEOUT = -6,     /* a bounded device-side wait gave up */
};

/* Version of this ABI (major*100 + minor). */
CIMX_API int cimx_abi_version(void);  /* 101: CimxBatchTile row pitches */

/* Description of the last error raised on the calling thread. */
CIMX_API const char* cimx_last_error_string(void);

/* Status word of the current device: 0, or CIMX_E_TIMEOUT if a bounded
 * device-side wait (TMA tile loads) gave up since the last clear. Reads the
 * word synchronously; clear != 0 resets it. No counterpart in cuCIM, whose
 * kernels have no device-side waits. */
CIMX_API int cimx_device_status(int clear);

/* Self-test of the device-side timeout path. Launches one thread that waits
 * on an mbarrier nothing arrives on, with the bounded wait of the TMA-fed
 * kernels (which 0: `limit` polls, 1..2^24) or of the tensor-core pass
 * (which 1: `limit` nanoseconds of %globaltimer, 1..1e8). The wait runs
 * out, records CIMX_E_TIMEOUT in the status word read by
 * cimx_device_status() and the kernel returns, leaving the context usable.
 * No counterpart in cuCIM, whose kernels have no device-side waits. */
CIMX_API int cimx_wait_selftest(int which, long long limit, void* stream);

/* Scratch allocator hook (default: cudaMallocAsync / cudaFreeAsync on the
 * call's stream). Both functions receive the stream the call runs on. */
typedef void* (*cimx_alloc_fn)(size_t nbytes, void* stream, void* user);
typedef void (*cimx_free_fn)(void* ptr, size_t nbytes, void* stream, void* user);
CIMX_API int cimx_set_allocator(cimx_alloc_fn alloc, cimx_free_fn release, void* user);

/* The schedule autotuner of cimx_separable (and of every entry built on
 * it). A pass list can run on several kernel schedules with bit-identical
 * results (CIMX_L_NO_VOLUME, CIMX_L_NO_STREAM, CIMX_L_NO_ROWSTREAM,
 * CIMX_L_NO_FUSION, the z chunk bits); with a tensor flag the tensor-core
 * and plain passes are candidates too. The tuner keys a table on the call
 * signature (dtypes, shape, each pass's axis, taps, anchor, mode and flags,
 * the tensor flags), one table per device model:
 *   CIMX_TUNE_OFF  the built-in rules only;
 *   CIMX_TUNE_USE  recorded schedules where present (the default);
 *   CIMX_TUNE_ON   an unseen signature is timed on the call's own arrays (each
 *                  candidate once to warm up and three times between CUDA
 *                  events; this synchronises the stream, and is skipped while
 *                  the stream is being captured) and the fastest recorded.
 * A call that sets a schedule flag itself, or CIMX_L_NO_TUNE, is not tuned.
 * Environment: CIMX_TUNE = 0/1/2 sets the initial mode; CIMX_TUNE_CACHE
 * names a JSON file read at first use and rewritten after each newly tuned
 * signature. cuCIM chooses its kernel by a fixed rule instead
 * (_vendored/_ndimage_filters.py:284-297); no counterpart there. */
enum { CIMX_TUNE_OFF = 0, CIMX_TUNE_USE = 1, CIMX_TUNE_ON = 2 };
/* Sets the mode (mode < 0: leaves it) and returns the previous one. */
CIMX_API int cimx_tune_mode(int mode);
/* Merges the entries of a JSON table file; writes the whole table. */
CIMX_API int cimx_tune_load(const char* path);
CIMX_API int cimx_tune_save(const char* path);
CIMX_API int cimx_tune_clear(void);
/* The table as JSON text into buf (truncated to size - 1 characters, NUL
 * terminated); returns the size the whole text needs, NUL included. */
CIMX_API long long cimx_tune_dump(char* buf, long long size);

/* One 1-D correlation (or convolution) along `axis`.
 * Replaces the shared-memory kernel driver _shmem_convolve1d
 * (filters/_separable_filtering.py:977-1070) and the elementwise correlate
 * kernel call (_vendored/_ndimage_filters.py:224-257 -> _vendored/_ndimage_filters_core.py:166-214).
 * `in` and `out` must be C-contiguous with equal shapes and must not overlap. */
CIMX_API int cimx_correlate1d(const CimxArray* in, const CimxArray* out, const double* taps,
                     int ntaps, int axis, int origin, int mode, double cval,
                     int flags, void* stream);

/* A sequence of 1-D passes applied in order, intermediates stored in the
 * output's dtype exactly like _run_1d_filters
 * (_vendored/_ndimage_filters_core.py:124-163). Consecutive passes are fused
 * into one launch when the shapes allow it; the result is bit-identical to
 * running them one by one. Scratch (one temporary of the output's shape and
 * dtype) is taken from the allocator only when passes are not fused.
 * Used by gaussian_filter, uniform_filter, sobel, prewitt
 * (_vendored/_ndimage_filters.py:363-396, 447-521, 580-686, 720-803). */
CIMX_API int cimx_separable(const CimxArray* in, const CimxArray* out, const CimxPass* passes,
                   int npasses, int lib_flags, void* stream);

/* cimx_separable for callers that cannot allocate device memory (code
 * running inside someone else's stream capture, plug-ins whose host
 * application owns every allocation, pipelines that forbid allocation after
 * start-up). No counterpart in cuCIM: it is an addition of this library.
 * The same arguments as cimx_separable except lib_flags; the results equal
 * cimx_separable's with CIMX_L_NO_FUSION and no tensor flags, because the
 * passes always run on the generic kernels, one launch each. The ping-pong
 * intermediate lives in a 64 MiB static device array that every GPU loading
 * the library holds until exit; the call makes no cudaMalloc/cudaFree or
 * other allocating call. Limits: the intermediate (element count x output
 * itemsize, needed when npasses >= 2) must fit in 64 MiB and each pass may
 * have at most 1024 float32 / 512 float64 taps; larger requests, and a pass
 * whose taps would need device memory, return CIMX_E_INVALID with a
 * message. The first call on a device (and the first after cudaDeviceReset)
 * resolves the array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture. All calls share the one array, which keeps the
 * last call's contents: calls that overlap on the GPU (concurrent streams)
 * race on it. */
CIMX_API int cimx_separable_noalloc(const CimxArray* in, const CimxArray* out,
                                    const CimxPass* passes, int npasses, void* stream);

/* out = sqrt(sum_i d_i^2) with d_i = separable(in, passes[i*passes_per_axis ...]),
 * i = 0..naxes-1, with cuCIM's rounding order: out = d_0*d_0 (rounded),
 * then out += (d_i*d_i rounded) for i >= 1, then sqrt. Replaces
 * generic_gradient_magnitude as driven by gaussian_gradient_magnitude
 * (_vendored/_ndimage_filters.py:1012-1097, :1100-1157) and the magnitude
 * branch of the skimage edge filters (filters/edges.py:148-241, where each
 * chain is the edge pass followed by the smoothing passes).
 * `out` must be float32 or float64. */
CIMX_API int cimx_gradient_magnitude(const CimxArray* in, const CimxArray* out,
                            const CimxPass* passes, int naxes, int passes_per_axis,
                            void* stream);

/* Laplacian as a sum of per-axis chains: out = chain_0(in), then
 * tmp = chain_a(in); out += tmp (in out's dtype) for a >= 1. `passes` holds
 * naxes chains of passes_per_axis passes each (axis a's chain at
 * passes + a * passes_per_axis). Replaces generic_laplace as driven by
 * laplace and gaussian_laplace (_vendored/_ndimage_filters.py:806-1009: one
 * correlate1d with [1, -2, 1], or one gaussian_filter with order 2 on the
 * axis, per axis). */
CIMX_API int cimx_laplace(const CimxArray* in, const CimxArray* out, const CimxPass* passes,
                          int naxes, int passes_per_axis, void* stream);

/* acc = term * term (first != 0) or acc + term * term, each operation rounded
 * on its own; and acc = sqrt(acc) in place. float32 or float64, equal
 * dtypes and shapes, C-contiguous: the `output *= output; tmp *= tmp;
 * output += tmp; cupy.sqrt(output, output)` of generic_gradient_magnitude
 * with a user derivative (_vendored/_ndimage_filters.py:1012-1097). */
CIMX_API int cimx_square_accumulate(const CimxArray* acc, const CimxArray* term, int first,
                                    void* stream);
CIMX_API int cimx_sqrt(const CimxArray* a, void* stream);

/* acc = acc + term (op CIMX_COMBINE_ADD) or acc - term (CIMX_COMBINE_SUBTRACT)
 * in acc's dtype: integers wrap, floats round to nearest. Both arrays have
 * the same dtype and shape and are C-contiguous. The in-place `output += tmp`
 * of generic_laplace (_vendored/_ndimage_filters.py:888) and `out -= ...` of
 * difference_of_gaussians (filters/_gaussian.py:164). */
enum { CIMX_COMBINE_ADD = 0, CIMX_COMBINE_SUBTRACT = 1 };
CIMX_API int cimx_combine(const CimxArray* acc, const CimxArray* term, int op, void* stream);

/* out = image + (image - blurred) * amount, each operation rounded on its
 * own, then clipped to [lo, hi] when `clip` (nan passes through): the
 * elementwise part of skimage's unsharp mask (filters/_unsharp_mask.py:12-20).
 * float32 or float64, equal dtypes and shapes, C-contiguous. */
CIMX_API int cimx_unsharp(const CimxArray* image, const CimxArray* blurred, const CimxArray* out,
                          double amount, int clip, double lo, double hi, void* stream);

/* *result = 1 when some element of `a` (float32/float64) is below zero, else 0;
 * waits for the stream (filters/_unsharp_mask.py:145, cp.any(fimg < 0)). */
CIMX_API int cimx_any_negative(const CimxArray* a, int* result, void* stream);

/* minimum_filter1d (is_max 0) / maximum_filter1d (is_max 1) of `size`
 * elements along `axis` (_vendored/_ndimage_filters.py:1362-1497): the
 * element itself, then the window in order, folded with fmin / fmax in
 * double (nan-ignoring); cval (as a double) outside the array in constant
 * mode; cast<D>() on store. C-contiguous arrays of any real dtype. The fold
 * runs in float32 where every value it sees is exact there (inputs of at
 * most float32 precision, a cval float32 holds): the same results. */
CIMX_API int cimx_min_max_1d(const CimxArray* in, const CimxArray* out, int size, int axis,
                             int origin, int mode, double cval, int is_max, void* stream);

/* Closed-form eigenvalues of symmetric 2x2 / 3x3 matrices given as the
 * upper-triangular element images in row-major order ((00,01,11) or
 * (00,01,02,11,12,22)). `out` holds nelems==3 ? 2 : 3 images of the same
 * shape. sort: 0 = ascending, 1 = descending; abs_sort sorts by magnitude.
 * Follows feature/corner.py:473-527 (2x2) and :566-647 (3x3, float64 inside). */
CIMX_API int cimx_eigvals_sym(const CimxArray* elems, int nelems, const CimxArray* out,
                     int sort, int abs_sort, void* stream);

/* rgb2gray: gray = 0.2125 R + 0.7154 G + 0.0721 B computed in float64,
 * stored in gray's dtype; rgb is (..., 3) C-contiguous float32/float64
 * (color/colorconv.py:1038-1095). When rgb is uint8 it is first scaled by
 * float32(1/255) as img_as_float32 does (util/dtype.py:360-361). */
CIMX_API int cimx_rgb2gray(const CimxArray* rgb, const CimxArray* gray, void* stream);

/* Elementwise conversion into a float32/float64 array (util/dtype.py:219-372):
 * op 0 = astype; op 1 = img_as_float (integers scaled by 1/max of their type
 * in float32 for <= 16-bit inputs, float64 otherwise; signed results clipped
 * at -1); op 2 = astype then negation (frangi with black_ridges=False,
 * filters/ridges.py:411-413). */
CIMX_API int cimx_convert(const CimxArray* in, const CimxArray* out, int op, void* stream);

/* numpy.gradient along `axis` with unit spacing and edge_order=1, used by
 * hessian_matrix(use_gaussian_derivatives=False) (feature/corner.py:370-382). */
CIMX_API int cimx_gradient_fd(const CimxArray* in, const CimxArray* out, int axis, void* stream);

/* One scale of frangi's epilogue (filters/ridges.py:228-319 and :436-475):
 * from the eigenvalues (sorted ascending by magnitude) compute the vesselness
 * and store it (first != 0) or fold it into `out` with a NaN-propagating
 * maximum. gamma = NaN selects cuCIM's automatic gamma: half the square root
 * of the largest sum of squared eigenvalues of the first scale, kept on the
 * device in *gamma_state (8 bytes of device memory owned by the caller); no
 * host synchronisation is needed. */
CIMX_API int cimx_frangi_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out,
                                    double alpha, double beta, double gamma, int first,
                                    void* gamma_state, void* stream);

/* ---------------------------------------------------------------------
 * Whole filters in one call, for hosts without the Python layer. Each entry
 * restates cuCIM's host-side rules in C++ (per-axis arguments, sigma and
 * radius cut-offs, tap generation, the weights type, the choice between
 * cuCIM's shared-memory and elementwise kernels) and runs the same kernels
 * as the Python package. Modes are CIMX_MODE_* codes ('wrap' passed as
 * CIMX_MODE_GRID_WRAP); `algorithm` is cuCIM's algorithm= keyword.
 * --------------------------------------------------------------------- */
enum {
  CIMX_ALGO_AUTO = 0,           /* algorithm=None */
  CIMX_ALGO_SHARED_MEMORY = 1,  /* algorithm='shared_memory' */
  CIMX_ALGO_ELEMENTWISE = 2,    /* algorithm='elementwise' */
};

/* The float64 correlation taps of a Gaussian (derivative) of `order` with
 * 2 * radius + 1 taps, written to taps[0 .. 2 * radius]: cuCIM's
 * _gaussian_kernel1d (_vendored/_ndimage_filters.py:689-717), with numpy's
 * pairwise summation order for the normalisation and the C library's exp().
 * numpy's own exp() differs from the C library's in the last bit for a few
 * percent of arguments on hosts where numpy uses its AVX-512 code, so cuCIM's
 * float64 taps themselves depend on the host. Over a sweep of sigmas
 * (0.3-40, truncate 4, 8 and 100) the taps here are within 5 ulp of numpy's
 * (orders 0 and 1; orders 2 and 3: 11 ulp of the largest tap, their
 * polynomial cancelling near its roots), and bit for bit equal
 * once rounded to float32, the weights type of float32 inputs and of every
 * input of 16 bits or fewer; the test suite checks both. */
CIMX_API int cimx_gaussian_taps(double sigma, int order, int radius, double* taps);

/* gaussian_filter (_vendored/_ndimage_filters.py:580-686) over `naxes` axes
 * (`axes` NULL: all axes, naxes == ndim), with per-axis sigma, order
 * (NULL: 0), radius (NULL or a negative entry: int(truncate * sigma + 0.5))
 * and mode. Axes with sigma <= 1e-15 or radius 0 are skipped; with none left
 * the input is copied (cast) into the output. */
CIMX_API int cimx_gaussian_nd(const CimxArray* in, const CimxArray* out, const double* sigma,
                              const int* order, const int* radius, const int* modes,
                              const int* axes, int naxes, double truncate, double cval,
                              int algorithm, int lib_flags, void* stream);

/* uniform_filter (_vendored/_ndimage_filters.py:447-521): per-axis size,
 * mode and origin (NULL: 0) over `axes` (NULL: all); sizes of 1 skipped. */
CIMX_API int cimx_uniform_nd(const CimxArray* in, const CimxArray* out, const int* sizes,
                             const int* modes, const int* origins, const int* axes, int naxes,
                             double cval, int algorithm, int lib_flags, void* stream);

/* sobel (prewitt = 0) or prewitt (prewitt = 1) along `axis`
 * (_vendored/_ndimage_filters.py:720-803): [-1, 0, 1] along `axis`, [1, 2, 1]
 * or [1, 1, 1] along the other axes; `modes` holds one mode per axis. */
CIMX_API int cimx_sobel_nd(const CimxArray* in, const CimxArray* out, int axis,
                           const int* modes, double cval, int prewitt, int algorithm,
                           int lib_flags, void* stream);

/* gaussian_gradient_magnitude (_vendored/_ndimage_filters.py:1100-1157)
 * with per-axis sigma; modes[a] is the mode of every pass of the derivative
 * along axis a (generic_gradient_magnitude passes one mode per derivative);
 * `out` float32 or float64. */
CIMX_API int cimx_gaussian_gradient_magnitude_nd(const CimxArray* in, const CimxArray* out,
                                                 const double* sigma, const int* modes,
                                                 double truncate, double cval, int algorithm,
                                                 void* stream);

/* hessian_matrix (feature/corner.py:257-384): the ndim * (ndim + 1) / 2
 * upper-triangular element images, in the order of
 * combinations_with_replacement(axes, 2) (axes reversed when order_xy, 2-D
 * only), written to elems[], each of the image's float type (float32 for
 * inputs of 16 bits or fewer and float32, else float64). `sigma` holds one
 * value per axis. use_gaussian_derivatives != 0: Gaussian-derivative
 * filters at sigma / sqrt(2), truncate 8 (or 100 when some sigma <= 1)
 * (corner.py:161-254); 0: skimage gaussian then numpy.gradient twice.
 * Integer images are first converted as img_as_float does. Scratch: the
 * converted image and ndim gradient images from the allocator. */
CIMX_API int cimx_hessian(const CimxArray* in, const CimxArray* elems, int nelems,
                          const double* sigma, int mode, double cval,
                          int use_gaussian_derivatives, int order_xy, int lib_flags,
                          void* stream);

/* cimx_ridge_filter with CIMX_RIDGE_FRANGI: frangi vesselness
 * (filters/ridges.py:322-476) of a 2-D or 3-D image over
 * `nsigmas` scales: per scale the Gaussian-derivative Hessian, its
 * eigenvalues sorted ascending by magnitude, and the vesselness folded into
 * `out` (the image's float type) with a maximum. gamma = NaN selects the
 * automatic gamma of the first scale, kept on the device (no host
 * synchronisation). black_ridges = 0 negates the image first. Scratch: the
 * image, the Hessian elements, their eigenvalues and the gradients. */
CIMX_API int cimx_frangi(const CimxArray* in, const CimxArray* out, const double* sigmas,
                         int nsigmas, double alpha, double beta, double gamma, int black_ridges,
                         int mode, double cval, int lib_flags, void* stream);

/* The ridge filters of filters/ridges.py over `nsigmas` scales, each built
 * on the Gaussian-derivative Hessian and its closed-form eigenvalues, 2-D or
 * 3-D images, `out` of the image's float type:
 *   CIMX_RIDGE_FRANGI    frangi (:322-476), gamma NaN = automatic;
 *   CIMX_RIDGE_MEIJERING meijering (:50-146), alpha NaN = 1 / (ndim + 1);
 *   CIMX_RIDGE_SATO      sato (:148-225);
 *   CIMX_RIDGE_HESSIAN   the hybrid hessian filter (:479-595): frangi with
 *                        gamma NaN = 15, then outputs <= 0 set to 1.
 * Arguments a filter does not use are ignored. Nothing synchronises the
 * host: the automatic gamma and meijering's normalising maximum stay on the
 * device. Scratch: the image, the Hessian elements, their eigenvalues and
 * the gradients. */
enum {
  CIMX_RIDGE_FRANGI = 0,
  CIMX_RIDGE_MEIJERING = 1,
  CIMX_RIDGE_SATO = 2,
  CIMX_RIDGE_HESSIAN = 3,
};
CIMX_API int cimx_ridge_filter(const CimxArray* in, const CimxArray* out, int kind,
                               const double* sigmas, int nsigmas, double alpha, double beta,
                               double gamma, int black_ridges, int mode, double cval,
                               int lib_flags, void* stream);

/* Per-scale epilogues of meijering and sato on the eigenvalue images of one
 * scale (descending, as hessian_matrix_eigvals returns them), folded into
 * `out` with a NaN-propagating maximum that starts from 0 (first != 0).
 * meijering (filters/ridges.py:102-146): eigenvalues below 1e-12 in
 * magnitude zeroed, mixed by the circulant matrix (1 on the diagonal, alpha
 * elsewhere) as ascending multiply-add chains, the mixed value of largest
 * magnitude clipped at 0 and divided by its maximum over the image, reduced
 * into `state` (16 bytes of device memory owned by the caller) on the device.
 * sato (:203-225): the geometric mean (powf) of the clipped eigenvalues but
 * the lowest, times sigma^2. */
CIMX_API int cimx_meijering_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out,
                                       double alpha, int first, void* state, void* stream);
CIMX_API int cimx_sato_accumulate(const CimxArray* eigs, int ndim, const CimxArray* out,
                                  double sigma, int first, void* stream);

/* a[a <= 0] = 1 in place (the last step of filters/ridges.py:479-595). */
CIMX_API int cimx_nonpositive_to_one(const CimxArray* a, void* stream);

/* The mask= argument of the skimage edge filters (filters/edges.py:75-85):
 * `mask` (any real or bool dtype, nonzero = inside) is eroded with the
 * full-connectivity footprint (the whole 3 x ... x 3 neighbourhood) with
 * border value 0, and `result` (float32/float64, same shape, both
 * C-contiguous) is multiplied by it in place. */
CIMX_API int cimx_mask_erode_multiply(const CimxArray* result, const CimxArray* mask,
                                      void* stream);

/* out = a * b elementwise (float32/float64, equal shapes, C-contiguous): the
 * derivative products of structure_tensor (feature/corner.py:146-156). */
CIMX_API int cimx_multiply(const CimxArray* a, const CimxArray* b, const CimxArray* out,
                           void* stream);

/* Corner measures of feature/corner.py from their input images (all of one
 * float dtype and shape, C-contiguous):
 *   CIMX_CORNER_KITCHEN_ROSENFELD  inputs imx, imy, imxx, imxy, imyy (:940-1004);
 *   CIMX_CORNER_HARRIS_K           inputs Arr, Acc, Arc; param = k   (:1007-1021);
 *   CIMX_CORNER_HARRIS_EPS         inputs Arr, Acc, Arc; param = eps (:1024-1038);
 *   CIMX_CORNER_SHI_TOMASI         inputs Arr, Acc, Arc              (:1116-1128);
 *   CIMX_CORNER_FOERSTNER          inputs Arr, Acc, Arc; out = w, out2 = q (:1192-1213).
 * Each evaluates cuCIM's kernel expression in the same types. */
enum {
  CIMX_CORNER_KITCHEN_ROSENFELD = 0,
  CIMX_CORNER_HARRIS_K = 1,
  CIMX_CORNER_HARRIS_EPS = 2,
  CIMX_CORNER_SHI_TOMASI = 3,
  CIMX_CORNER_FOERSTNER = 4,
};
CIMX_API int cimx_corner_response(int kind, const CimxArray* inputs, int ninputs,
                                  const CimxArray* out, const CimxArray* out2, double param,
                                  void* stream);

/* One scale of frangi from the Hessian elements themselves, (00, 01, 11) or
 * (00, 01, 02, 11, 12, 22): the eigenvalues (ascending by magnitude) and the
 * vesselness in one kernel, folded into `out` like cimx_frangi_accumulate,
 * without storing the eigenvalue images. For the first scale with the
 * automatic gamma (gamma NaN, first != 0), whose gamma needs the image-wide
 * maximum first, and for float64 images on every scale, the eigenvalues go
 * through scratch memory as in cimx_eigvals_sym + cimx_frangi_accumulate.
 * Results are bit-identical to that pair. filters/ridges.py:425-475. */
CIMX_API int cimx_frangi_hessian_accumulate(const CimxArray* H, int nelems,
                                            const CimxArray* out, double alpha, double beta,
                                            double gamma, int first, void* gamma_state,
                                            void* stream);

/* One tile of a batch for cimx_batch_gray_gauss_sobel. */
typedef struct CimxBatchTile {
  const uint8_t* rgb;   /* device: height rows of width x 3 uint8 (pixels interleaved) */
  float* out;           /* device: height rows of width float32 */
  int32_t height, width;
  int32_t ntaps;        /* gaussian taps of this tile (odd, <= max_taps) */
  int32_t taps_offset;  /* index of the tile's first tap in `taps` */
  int64_t first_block;  /* index of the tile's first 64 x 64 output block; tiles in
                           ascending order, the first at 0 */
  int64_t rgb_pitch;    /* bytes from one rgb row to the next (0: 3 * width); a region
                           of a larger slide image passes the slide's row pitch */
  int64_t out_pitch;    /* float32 elements from one output row to the next (0: width) */
} CimxBatchTile;

/* For every tile of a batch: rgb2gray (color/colorconv.py:1038-1095 with the
 * uint8 -> float32 scaling of util/dtype.py:360-361), a gaussian with the
 * tile's own float32 taps and mode 'nearest' (skimage.filters.gaussian,
 * _shared/filters.py:21-166), then the sobel gradient magnitude with mode
 * 'reflect' (filters/edges.py:148-306: edge taps `edge_taps` along one axis,
 * `smooth_taps` along the other, both as correlation taps after the
 * convolution flip), float32 out — one persistent launch over the tiles'
 * 64 x 64 output blocks (`nblocks` in all). Results are bit-identical to the
 * three per-tile calls. `tiles` and `taps` are device memory prepared by the
 * caller, so the launch can be captured in a CUDA graph and replayed;
 * `edge_taps` and `smooth_taps` are 3 host floats read at the call.
 * No counterpart in cuCIM, which runs the three functions per tile. */
CIMX_API int cimx_batch_gray_gauss_sobel(const CimxBatchTile* tiles, int ntiles,
                                         long long nblocks, const float* taps, int max_taps,
                                         const float* edge_taps, const float* smooth_taps,
                                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CIMX_H_ */
