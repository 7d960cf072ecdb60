// cimx_ops.cu — whole-filter entry points for hosts without the Python layer:
// gaussian_filter, uniform_filter, sobel / prewitt,
// gaussian_gradient_magnitude, hessian_matrix and frangi, each one C call.
//
// The Python package builds pass lists with cuCIM's host rules and calls
// cimx_separable; these entries restate the same host rules in C++ (per-axis
// arguments, the sigma and radius cut-offs, Gaussian tap generation in
// float64, the weights type, the choice between cuCIM's two kernels, which
// fixes how constant-mode fill values are rounded and whether zero taps are
// skipped) and run the same kernels. Paths are relative to
// python/cucim/src/cucim/skimage in rapidsai/cucim: FLT =
// _vendored/_ndimage_filters.py, UTIL = _vendored/_ndimage_util.py,
// SEP = filters/_separable_filtering.py.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

// ------------------------------------------------------------------ taps

// numpy's pairwise summation of a contiguous float64 vector (the order in
// which numpy's add.reduce adds; restated so that the sum of the Gaussian
// taps is the same double): blocks of up to 128 summed with 8 partial sums,
// larger vectors split in two at a multiple of 8.
double pairwise_sum(const double* a, int64_t n) {
  if (n < 8) {
    double r = 0.0;
    for (int64_t i = 0; i < n; ++i) r += a[i];
    return r;
  }
  if (n <= 128) {
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int64_t i = 8;
    for (; i < n - (n % 8); i += 8)
      for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += a[i];
    return res;
  }
  int64_t n2 = n / 2;
  n2 -= n2 % 8;
  return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
}

// FLT:689-717 in float64, correlation order. Order 0: exp(-0.5 / sigma^2 *
// x^2) normalised by its sum. Order n: the polynomial q_n (q -> q' + q * p'
// applied n times to q_0 = 1, p' = -x / sigma^2) evaluated at x and
// multiplied by the Gaussian, reversed. exp() is the C library's; see
// cimx_gaussian_taps in include/cimx.h for how that relates to numpy's.
int gaussian_taps(double sigma, int order, int radius, std::vector<double>& out) {
  if (order < 0) return fail(CIMX_E_INVALID, "order must be non-negative");
  if (radius < 0) return fail(CIMX_E_INVALID, "radius must be non-negative");
  const int K = 2 * radius + 1;
  const double sigma2 = sigma * sigma;
  const double c = -0.5 / sigma2;
  std::vector<double> phi(K);
  for (int k = 0; k < K; ++k) {
    const long long x = k - radius;
    phi[k] = std::exp(c * static_cast<double>(x * x));
  }
  const double s = pairwise_sum(phi.data(), K);
  for (int k = 0; k < K; ++k) phi[k] /= s;
  if (order == 0) {
    out = phi;
    return CIMX_OK;
  }
  // q <- (D + P) q, D[i][i+1] = i + 1 (derivative), P[i+1][i] = 1 / -sigma^2
  std::vector<double> q(order + 1, 0.0), nq(order + 1);
  q[0] = 1.0;
  const double pd = 1.0 / -sigma2;
  for (int it = 0; it < order; ++it) {
    for (int i = 0; i <= order; ++i) {
      double acc = 0.0;
      if (i + 1 <= order) acc = std::fma(static_cast<double>(i + 1), q[i + 1], acc);
      if (i >= 1) acc = std::fma(pd, q[i - 1], acc);
      nq[i] = acc;
    }
    q = nq;
  }
  out.assign(K, 0.0);
  for (int k = 0; k < K; ++k) {
    const double x = static_cast<double>(k - radius);
    double xp = 1.0, acc = 0.0;
    for (int p = 0; p <= order; ++p) {
      acc = std::fma(xp, q[p], acc);
      xp *= x;
    }
    out[K - 1 - k] = acc * phi[k];
  }
  return CIMX_OK;
}

// ------------------------------------------------------ host-side rules

bool is_float(int dt) { return dt == DT_F16 || dt == DT_F32 || dt == DT_F64; }
bool is_unsigned(int dt) {
  return dt == DT_U8 || dt == DT_U16 || dt == DT_U32 || dt == DT_U64 || dt == DT_U64Q ||
         dt == '?';
}

// numpy.promote_types(dtype, float32) == float64 (UTIL:35-46 for float
// weights; FLT:658 for the Gaussian taps)
bool weights_f64(int dt) {
  return !(dt == DT_F16 || dt == DT_F32 || dt == DT_I8 || dt == DT_U8 || dt == DT_I16 ||
           dt == DT_U16 || dt == '?');
}

// skimage's _supported_float_type (_shared/utils.py:1131-1179)
int supported_float(int dt) { return weights_f64(dt) ? DT_F64 : DT_F32; }

// The shared-memory kernel's tile in bytes (SEP:17-88).
int64_t smem_bytes(int ndim, int axis, int K, int anchor, int itemsize) {
  const int hpn = std::max(K - anchor, anchor);
  int bx, by, bz, halo;
  if (ndim == 2) {
    bx = axis == 1 ? 16 : 32;
    by = axis == 1 ? 16 : 8;
    bz = 1;
    halo = (hpn + (axis == 1 ? bx : by) - 1) / (axis == 1 ? bx : by);
  } else if (axis == 2) {
    bx = 16, by = 4, bz = 4;
    halo = (hpn + bx - 1) / bx;
  } else {
    bx = 32, by = 4, bz = 4;
    const int d = axis == 1 ? by : bz;
    halo = (hpn + d - 1) / d;
  }
  const int ppb = std::max(4, halo);
  return (int64_t)(ppb + 2 * halo) * bx * by * bz * itemsize;
}

// Which of cuCIM's kernels a pass runs (FLT:271-344): true = shared memory.
int choose_shared(int ndim, int axis, int K, int anchor, int mode, double cval, int in_dt,
                  int algorithm, bool* shared) {
  const bool constant = mode == CIMX_MODE_CONSTANT;
  int alg = algorithm;
  if (alg == CIMX_ALGO_AUTO) {
    alg = (ndim == 2 && K <= 256 && !(cval < 0 && constant && is_unsigned(in_dt)))
              ? CIMX_ALGO_SHARED_MEMORY
              : CIMX_ALGO_ELEMENTWISE;
  } else if (alg == CIMX_ALGO_SHARED_MEMORY) {
    if (constant && (!std::isfinite(cval) || (cval < 0 && is_unsigned(in_dt))))
      alg = CIMX_ALGO_ELEMENTWISE;
  } else if (alg != CIMX_ALGO_ELEMENTWISE) {
    return fail(CIMX_E_INVALID, "algorithm must be 'shared_memory', 'elementwise' or None");
  }
  if (alg == CIMX_ALGO_SHARED_MEMORY) {
    if (ndim != 2 && ndim != 3)
      return fail(CIMX_E_INVALID,
                  "shared_memory not implemented for ndim=" + std::to_string(ndim));
    if ((constant && !std::isfinite(cval)) ||
        (K > 32 && smem_bytes(ndim, axis, K, anchor, dtype_size(in_dt)) > 49152))
      alg = CIMX_ALGO_ELEMENTWISE;
  }
  *shared = alg == CIMX_ALGO_SHARED_MEMORY;
  return CIMX_OK;
}

// A pass list under construction: CimxPass structs and the taps they point at.
struct Passes {
  std::vector<std::vector<double>> taps;
  std::vector<CimxPass> items;

  // One correlation pass (origin 0) with float64 taps `w`; `in_dt` is the
  // dtype the pass reads, `w_f64` the weights type.
  int add(int ndim, int axis, std::vector<double> w, int mode, double cval, int in_dt,
          bool w_f64, int algorithm, bool convolve = false, int origin = 0) {
    const int K = (int)w.size();
    int o = origin;
    if (convolve) {
      o = -o;
      if (K % 2 == 0) o -= 1;
    }
    bool shared = false;
    int rc = choose_shared(ndim, axis, K, K / 2 + o, mode, cval, in_dt, algorithm, &shared);
    if (rc) return rc;
    taps.push_back(std::move(w));
    CimxPass p{};
    p.axis = axis;
    p.ntaps = K;
    p.origin = origin;
    p.mode = mode;
    p.cval = cval;
    p.flags = (w_f64 ? CIMX_F_W64 : 0) | (convolve ? CIMX_F_CONVOLVE : 0) |
              (shared ? CIMX_F_CVAL_AS_INPUT : CIMX_F_SKIP_ZERO_TAPS);
    items.push_back(p);
    return CIMX_OK;
  }
  const CimxPass* data() {
    for (size_t i = 0; i < items.size(); ++i) items[i].taps = taps[i].data();
    return items.data();
  }
  int size() const { return (int)items.size(); }
};

int check_cval(int mode, double cval, int out_dt) {
  if (mode == CIMX_MODE_CONSTANT && !is_float(out_dt) && !std::isfinite(cval))
    return fail(CIMX_E_INVALID, "Non-finite cval is not supported for outputs with integer dtype.");
  return CIMX_OK;
}

// UTIL:110-127: axes (NULL = all), normalised and unique.
int resolve_axes(const int* axes, int naxes, int ndim, std::vector<int>& out) {
  out.clear();
  if (!axes) {
    if (naxes != ndim)
      return fail(CIMX_E_INVALID, "naxes must equal ndim when axes is NULL");
    for (int a = 0; a < ndim; ++a) out.push_back(a);
    return CIMX_OK;
  }
  if (naxes < 0 || naxes > ndim) return fail(CIMX_E_INVALID, "too many axes");
  for (int i = 0; i < naxes; ++i) {
    int a = axes[i];
    if (a < -ndim || a >= ndim)
      return fail(CIMX_E_INVALID, "axis " + std::to_string(a) + " is out of bounds for array "
                                  "of dimension " + std::to_string(ndim));
    a = (a + ndim) % ndim;
    if (std::find(out.begin(), out.end(), a) != out.end())
      return fail(CIMX_E_INVALID, "axes must be unique");
    out.push_back(a);
  }
  return CIMX_OK;
}

int64_t numel(const CimxArray* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

// A C-contiguous CimxArray over `data` with a's shape and dtype `dt`.
CimxArray dense_like(const CimxArray* a, void* data, int dt) {
  CimxArray r{};
  r.data = data;
  r.dtype = dt;
  r.ndim = a->ndim;
  int64_t stride = dtype_size(dt);
  for (int d = a->ndim - 1; d >= 0; --d) {
    r.shape[d] = a->shape[d];
    r.strides[d] = stride;
    stride *= a->shape[d];
  }
  return r;
}

// Scratch buffers of one call, released on the call's stream at scope exit.
struct Scratch {
  cudaStream_t st;
  std::vector<std::pair<void*, size_t>> bufs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (auto& b : bufs) scratch_free(b.first, b.second, st);
  }
  void* get(size_t n) {
    void* p = scratch_alloc(std::max<size_t>(n, 16), st);
    if (p) bufs.emplace_back(p, std::max<size_t>(n, 16));
    return p;
  }
};

// gaussian_filter's pass list (FLT:580-686) for the axes `ax` with per-axis
// sigma, order, radius (negative: from truncate) and mode.
int gaussian_passes(const CimxArray* in, int out_dt, const std::vector<int>& ax,
                    const double* sigma, const int* order, const int* radius, const int* modes,
                    double truncate, double cval, int algorithm, Passes& pl) {
  const int ndim = in->ndim;
  const bool w64 = weights_f64(in->dtype);
  for (size_t i = 0; i < ax.size(); ++i) {
    if (!(sigma[i] > 1e-15)) continue;  // omit axes with sigma ~= 0
    int rc = check_mode(modes[i]);
    if (rc) return rc;
    if ((rc = check_cval(modes[i], cval, out_dt))) return rc;
    const int r = radius && radius[i] >= 0 ? radius[i]
                                           : (int)(truncate * sigma[i] + 0.5);
    if (r <= 0) continue;
    std::vector<double> w;
    if ((rc = gaussian_taps(sigma[i], order ? order[i] : 0, r, w))) return rc;
    const int pass_in = pl.size() == 0 ? in->dtype : out_dt;
    if ((rc = pl.add(ndim, ax[i], std::move(w), modes[i], cval, pass_in, w64, algorithm)))
      return rc;
  }
  return CIMX_OK;
}

}  // namespace
}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_gaussian_taps(double sigma, int order, int radius, double* taps) {
  if (!taps) return fail(CIMX_E_INVALID, "taps is NULL");
  std::vector<double> w;
  int rc = gaussian_taps(sigma, order, radius, w);
  if (rc) return rc;
  std::copy(w.begin(), w.end(), taps);
  return CIMX_OK;
}

int cimx_gaussian_nd(const CimxArray* in, const CimxArray* out, const double* sigma,
                     const int* order, const int* radius, const int* modes, const int* axes,
                     int naxes, double truncate, double cval, int algorithm, int lib_flags,
                     void* stream) {
  if (!in || !out) return fail(CIMX_E_INVALID, "input or output is NULL");
  if (naxes > 0 && (!sigma || !modes)) return fail(CIMX_E_INVALID, "sigma or modes is NULL");
  std::vector<int> ax;
  int rc = resolve_axes(axes, naxes, in->ndim, ax);
  if (rc) return rc;
  Passes pl;
  if ((rc = gaussian_passes(in, out->dtype, ax, sigma, order, radius, modes, truncate, cval,
                            algorithm, pl)))
    return rc;
  return cimx_separable(in, out, pl.data(), pl.size(), lib_flags, stream);
}

int cimx_uniform_nd(const CimxArray* in, const CimxArray* out, const int* sizes,
                    const int* modes, const int* origins, const int* axes, int naxes,
                    double cval, int algorithm, int lib_flags, void* stream) {
  if (!in || !out) return fail(CIMX_E_INVALID, "input or output is NULL");
  if (naxes > 0 && (!sizes || !modes)) return fail(CIMX_E_INVALID, "sizes or modes is NULL");
  std::vector<int> ax;
  int rc = resolve_axes(axes, naxes, in->ndim, ax);
  if (rc) return rc;
  // FLT:447-521: taps full(size, 1 / size) in promote(dtype, float32); sizes
  // of 1 (or less) are skipped
  const bool w64 = weights_f64(in->dtype);
  Passes pl;
  for (size_t i = 0; i < ax.size(); ++i) {
    if ((rc = check_mode(modes[i]))) return rc;
    if ((rc = check_cval(modes[i], cval, out->dtype))) return rc;
    const int s = sizes[i];
    const int o = origins ? origins[i] : 0;
    if (s < 1) return fail(CIMX_E_INVALID, "incorrect filter size");
    if (s / 2 + o < 0 || s / 2 + o >= s) return fail(CIMX_E_INVALID, "invalid origin");
    if (s <= 1) continue;
    std::vector<double> w(s, 1.0 / s);
    const int pass_in = pl.size() == 0 ? in->dtype : out->dtype;
    if ((rc = pl.add(in->ndim, ax[i], std::move(w), modes[i], cval, pass_in, w64, algorithm,
                     false, o)))
      return rc;
  }
  return cimx_separable(in, out, pl.data(), pl.size(), lib_flags, stream);
}

int cimx_sobel_nd(const CimxArray* in, const CimxArray* out, int axis, const int* modes,
                  double cval, int prewitt, int algorithm, int lib_flags, void* stream) {
  if (!in || !out || !modes) return fail(CIMX_E_INVALID, "NULL argument");
  const int ndim = in->ndim;
  if (ndim < 1) return fail(CIMX_E_INVALID, "sobel needs ndim >= 1");
  if (axis < -ndim || axis >= ndim) return fail(CIMX_E_INVALID, "axis out of range");
  axis = (axis + ndim) % ndim;
  // FLT:782-803: [-1, 0, 1] along `axis`, [1, 2, 1] (sobel) or [1, 1, 1]
  // (prewitt) along every other axis, correlation, in axis order; integer
  // taps, so the weights type is promote(dtype, float32)
  const bool w64 = weights_f64(in->dtype);
  Passes pl;
  int rc;
  for (int a = 0; a < ndim; ++a) {
    if ((rc = check_mode(modes[a]))) return rc;
    if ((rc = check_cval(modes[a], cval, out->dtype))) return rc;
    std::vector<double> w = a == axis ? std::vector<double>{-1.0, 0.0, 1.0}
                            : prewitt ? std::vector<double>{1.0, 1.0, 1.0}
                                      : std::vector<double>{1.0, 2.0, 1.0};
    const int pass_in = pl.size() == 0 ? in->dtype : out->dtype;
    if ((rc = pl.add(ndim, a, std::move(w), modes[a], cval, pass_in, w64, algorithm))) return rc;
  }
  return cimx_separable(in, out, pl.data(), pl.size(), lib_flags, stream);
}

int cimx_gaussian_gradient_magnitude_nd(const CimxArray* in, const CimxArray* out,
                                        const double* sigma, const int* modes, double truncate,
                                        double cval, int algorithm, void* stream) {
  if (!in || !out || !sigma || !modes) return fail(CIMX_E_INVALID, "NULL argument");
  const int ndim = in->ndim;
  if (ndim < 1) return fail(CIMX_E_INVALID, "ndim must be >= 1");
  // FLT:1100-1157 -> FLT:1012-1097: per axis a, gaussian_filter with order
  // e_a over all axes, every pass of that chain in axis a's mode; the chains
  // all have the same passes count (the radius depends only on sigma)
  std::vector<int> ax(ndim);
  for (int a = 0; a < ndim; ++a) ax[a] = a;
  Passes all;
  int per_axis = -1;
  for (int a = 0; a < ndim; ++a) {
    std::vector<int> ord(ndim, 0);
    ord[a] = 1;
    std::vector<int> chain_modes(ndim, modes[a]);
    Passes pl;
    int rc = gaussian_passes(in, out->dtype, ax, sigma, ord.data(), nullptr, chain_modes.data(),
                             truncate, cval, algorithm, pl);
    if (rc) return rc;
    if (per_axis < 0) per_axis = pl.size();
    for (int i = 0; i < pl.size(); ++i) {
      all.taps.push_back(pl.taps[i]);
      all.items.push_back(pl.items[i]);
    }
  }
  return cimx_gradient_magnitude(in, out, all.data(), ndim, per_axis, stream);
}

int cimx_hessian(const CimxArray* in, const CimxArray* elems, int nelems, const double* sigma,
                 int mode, double cval, int use_gaussian_derivatives, int order_xy,
                 int lib_flags, void* stream) {
  if (!in || !elems || !sigma) return fail(CIMX_E_INVALID, "NULL argument");
  const int ndim = in->ndim;
  if (ndim < 1) return fail(CIMX_E_INVALID, "ndim must be >= 1");
  if (nelems != ndim * (ndim + 1) / 2)
    return fail(CIMX_E_INVALID, "nelems must be ndim * (ndim + 1) / 2");
  if (order_xy && ndim > 2) return fail(CIMX_E_INVALID, "Order 'xy' is only supported for 2D images.");
  int rc = check_mode(mode);
  if (rc) return rc;
  const int F = supported_float(in->dtype);
  for (int i = 0; i < nelems; ++i) {
    if (elems[i].dtype != F)
      return fail(CIMX_E_DTYPE, "Hessian elements must have the image's float type");
    if (elems[i].ndim != ndim) return fail(CIMX_E_INVALID, "output shape not correct");
    for (int d = 0; d < ndim; ++d)
      if (elems[i].shape[d] != in->shape[d])
        return fail(CIMX_E_INVALID, "output shape not correct");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = numel(in);
  if (n == 0) return CIMX_OK;
  const size_t fb = (size_t)n * dtype_size(F);
  Scratch scratch(st);

  // img_as_float, then astype(_supported_float_type) (corner.py:300-301)
  CimxArray img = *in;
  if (in->dtype != F) {
    void* p = scratch.get(fb);
    if (!p) return fail(CIMX_E_NOMEM, "scratch allocation for the float image failed");
    img = dense_like(in, p, F);
    if ((rc = cimx_convert(in, &img, 1, stream))) return rc;
  }
  std::vector<int> ax(ndim);
  for (int a = 0; a < ndim; ++a) ax[a] = a;
  std::vector<int> modes(ndim, mode);
  std::vector<int> pair_axes;  // combinations_with_replacement(axes, 2)
  std::vector<int> order(ndim);
  for (int a = 0; a < ndim; ++a) order[a] = order_xy ? ndim - 1 - a : a;
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ndim; ++i)
    for (int j = i; j < ndim; ++j) pairs.emplace_back(order[i], order[j]);

  std::vector<CimxArray> grads(ndim);
  for (int a = 0; a < ndim; ++a) {
    void* p = scratch.get(fb);
    if (!p) return fail(CIMX_E_NOMEM, "scratch allocation for the gradients failed");
    grads[a] = dense_like(in, p, F);
  }
  if (use_gaussian_derivatives) {
    // corner.py:161-254: sigma / sqrt(2) for each of the two derivative
    // chains; truncate 8 when every sigma exceeds 1, else 100
    bool all_gt1 = true;
    for (int a = 0; a < ndim; ++a) all_gt1 = all_gt1 && sigma[a] > 1;
    const double truncate = all_gt1 ? 8.0 : 100.0;
    const double sq1_2 = 1.0 / std::sqrt(2.0);
    std::vector<double> ss(ndim);
    for (int a = 0; a < ndim; ++a) ss[a] = sq1_2 * sigma[a];
    if (ndim == 1) {
      std::vector<int> o(1, 1);
      if ((rc = cimx_gaussian_nd(&img, &grads[0], ss.data(), o.data(), nullptr, modes.data(),
                                 nullptr, 1, truncate, cval, CIMX_ALGO_AUTO, lib_flags, stream)))
        return rc;
      return cimx_gaussian_nd(&grads[0], &elems[0], ss.data(), o.data(), nullptr, modes.data(),
                              nullptr, 1, truncate, cval, CIMX_ALGO_AUTO, lib_flags, stream);
    }
    // Every chain runs its axis-0 pass first, and chains share it: the
    // gradients along axes >= 1 all start with the order-0 pass on the image,
    // H[a0][a1] for a1 >= 1 all start with the order-0 pass on gradient a0.
    // Each shared pass runs once into scratch and the rest of each chain is a
    // call over the remaining axes: the same passes in the same order, so the
    // results are bit-identical.
    std::vector<int> rest_axes, rest_modes(ndim - 1, mode);
    std::vector<double> rest_sigma;
    for (int a = 1; a < ndim; ++a) {
      rest_axes.push_back(a);
      rest_sigma.push_back(ss[a]);
    }
    void* lp = scratch.get(2 * fb);
    if (!lp) return fail(CIMX_E_NOMEM, "scratch allocation for the shared passes failed");
    CimxArray lead[2] = {dense_like(in, lp, F), dense_like(in, static_cast<char*>(lp) + fb, F)};
    const int axis0[1] = {0};
    // lead[o] = the axis-0 pass of order o on `src`
    auto lead_pass = [&](const CimxArray* src, int o, const CimxArray* dst) {
      const int ord[1] = {o};
      return cimx_gaussian_nd(src, dst, ss.data(), ord, nullptr, modes.data(), axis0, 1,
                              truncate, cval, CIMX_ALGO_AUTO, lib_flags, stream);
    };
    // the rest of a chain of orders e_b over axes 1..ndim-1
    auto rest = [&](const CimxArray* src, int b, const CimxArray* dst) {
      std::vector<int> ord(ndim - 1, 0);
      if (b >= 1) ord[b - 1] = 1;
      return cimx_gaussian_nd(src, dst, rest_sigma.data(), ord.data(), nullptr,
                              rest_modes.data(), rest_axes.data(), ndim - 1, truncate, cval,
                              CIMX_ALGO_AUTO, lib_flags, stream);
    };
    if ((rc = lead_pass(&img, 1, &lead[1])) || (rc = rest(&lead[1], 0, &grads[0]))) return rc;
    if ((rc = lead_pass(&img, 0, &lead[0]))) return rc;
    for (int a = 1; a < ndim; ++a)
      if ((rc = rest(&lead[0], a, &grads[a]))) return rc;
    // H elements grouped by their gradient; each group's two axis-0 passes once
    for (int a0 = 0; a0 < ndim; ++a0) {
      bool done[2] = {false, false};
      for (int i = 0; i < nelems; ++i) {
        if (pairs[i].first != a0) continue;
        const int b = pairs[i].second, o0 = b == 0 ? 1 : 0;
        if (!done[o0]) {
          if ((rc = lead_pass(&grads[a0], o0, &lead[o0]))) return rc;
          done[o0] = true;
        }
        if ((rc = rest(&lead[o0], b, &elems[i]))) return rc;
      }
    }
    return CIMX_OK;
  }
  // corner.py:364-384: skimage gaussian (truncate 4; the channel axis of a
  // (..., 3) 3-D image excluded), then numpy.gradient twice
  void* p = scratch.get(fb);
  if (!p) return fail(CIMX_E_NOMEM, "scratch allocation for the smoothed image failed");
  CimxArray sm = dense_like(in, p, F);
  std::vector<int> sax;
  std::vector<double> ssig;
  std::vector<int> smodes;
  const bool channel = ndim == 3 && in->shape[2] == 3;
  for (int a = 0; a < ndim; ++a)
    if (!(channel && a == 2)) {
      sax.push_back(a);
      ssig.push_back(sigma[a]);
      smodes.push_back(mode);
    }
  if ((rc = cimx_gaussian_nd(&img, &sm, ssig.data(), nullptr, nullptr, smodes.data(), sax.data(),
                             (int)sax.size(), 4.0, cval, CIMX_ALGO_AUTO, lib_flags, stream)))
    return rc;
  for (int a = 0; a < ndim; ++a)
    if ((rc = cimx_gradient_fd(&sm, &grads[a], a, stream))) return rc;
  for (int i = 0; i < nelems; ++i)
    if ((rc = cimx_gradient_fd(&grads[pairs[i].first], &elems[i], pairs[i].second, stream)))
      return rc;
  return CIMX_OK;
}

int cimx_ridge_filter(const CimxArray* in, const CimxArray* out, int kind, const double* sigmas,
                      int nsigmas, double alpha, double beta, double gamma, int black_ridges,
                      int mode, double cval, int lib_flags, void* stream) {
  if (!in || !out || (nsigmas > 0 && !sigmas)) return fail(CIMX_E_INVALID, "NULL argument");
  if (kind < CIMX_RIDGE_FRANGI || kind > CIMX_RIDGE_HESSIAN)
    return fail(CIMX_E_INVALID, "unknown ridge filter");
  const int ndim = in->ndim;
  if (ndim != 2 && ndim != 3)
    return fail(CIMX_E_INVALID,
                "The parameter `image` must be a 2-dimensional or 3-dimensional array");
  const int F = supported_float(in->dtype);
  if (out->dtype != F) return fail(CIMX_E_DTYPE, "the output must have the image's float type");
  if (out->ndim != ndim) return fail(CIMX_E_INVALID, "output shape not correct");
  for (int d = 0; d < ndim; ++d)
    if (out->shape[d] != in->shape[d]) return fail(CIMX_E_INVALID, "output shape not correct");
  int rc = check_mode(mode);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = numel(in);
  if (n == 0) return CIMX_OK;
  const size_t fb = (size_t)n * dtype_size(F);
  const bool zero_init = kind == CIMX_RIDGE_MEIJERING || kind == CIMX_RIDGE_SATO;
  cudaError_t e;
  if (zero_init && (e = cudaMemsetAsync(out->data, 0, fb, st)) != cudaSuccess)
    return cuda_fail(e, "ridge output");
  if (nsigmas == 0) return CIMX_OK;
  const int nelems = ndim * (ndim + 1) / 2;
  Scratch scratch(st);

  // ridges.py:107-109, :200-202, :410-413: astype(float type), negated
  // when black_ridges is False
  void* p = scratch.get(fb);
  if (!p) return fail(CIMX_E_NOMEM, "scratch allocation for the image failed");
  CimxArray img = dense_like(in, p, F);
  if ((rc = cimx_convert(in, &img, black_ridges ? 0 : 2, stream))) return rc;
  std::vector<CimxArray> H(nelems), ev(ndim);
  for (int i = 0; i < nelems; ++i) {
    if (!(p = scratch.get(fb))) return fail(CIMX_E_NOMEM, "scratch allocation failed");
    H[i] = dense_like(in, p, F);
  }
  // eigenvalue images for meijering and sato (frangi's stay in registers)
  for (int i = 0; i < ndim && kind != CIMX_RIDGE_FRANGI && kind != CIMX_RIDGE_HESSIAN; ++i) {
    if (!(p = scratch.get(fb))) return fail(CIMX_E_NOMEM, "scratch allocation failed");
    ev[i] = dense_like(in, p, F);
  }
  void* state = scratch.get(16);
  if (!state) return fail(CIMX_E_NOMEM, "scratch allocation failed");
  if ((e = cudaMemsetAsync(state, 0, 16, st)) != cudaSuccess) return cuda_fail(e, "ridge state");
  if (kind == CIMX_RIDGE_MEIJERING && std::isnan(alpha)) alpha = 1.0 / (ndim + 1);
  if (kind == CIMX_RIDGE_HESSIAN && std::isnan(gamma)) gamma = 15.0;
  const bool frangi_like = kind == CIMX_RIDGE_FRANGI || kind == CIMX_RIDGE_HESSIAN;
  std::vector<double> sig(ndim);
  for (int s = 0; s < nsigmas; ++s) {
    std::fill(sig.begin(), sig.end(), sigmas[s]);
    if ((rc = cimx_hessian(&img, H.data(), nelems, sig.data(), mode, cval, 1, 0, lib_flags,
                           stream)))
      return rc;
    // meijering and sato take hessian_matrix_eigvals, descending
    // (corner.py:824-858); frangi's eigenvalues are computed inside its
    // epilogue kernel
    if (!frangi_like && (rc = cimx_eigvals_sym(H.data(), nelems, ev.data(), 1, 0, stream)))
      return rc;
    const int first = s == 0 ? 1 : 0;
    if (frangi_like)
      rc = cimx_frangi_hessian_accumulate(H.data(), nelems, out, alpha, beta, gamma, first, state,
                                          stream);
    else if (kind == CIMX_RIDGE_MEIJERING)
      rc = cimx_meijering_accumulate(ev.data(), ndim, out, alpha, first, state, stream);
    else
      rc = cimx_sato_accumulate(ev.data(), ndim, out, sigmas[s], first, stream);
    if (rc) return rc;
  }
  if (kind == CIMX_RIDGE_HESSIAN) return cimx_nonpositive_to_one(out, stream);
  return CIMX_OK;
}

int cimx_frangi(const CimxArray* in, const CimxArray* out, const double* sigmas, int nsigmas,
                double alpha, double beta, double gamma, int black_ridges, int mode,
                double cval, int lib_flags, void* stream) {
  return cimx_ridge_filter(in, out, CIMX_RIDGE_FRANGI, sigmas, nsigmas, alpha, beta, gamma,
                           black_ridges, mode, cval, lib_flags, stream);
}

}  // extern "C"
