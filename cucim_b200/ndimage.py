"""Drop-in for cuCIM's vendored ndimage separable filters.

Same names, signatures, defaults, dtype rules and errors as
cucim.skimage._vendored.ndimage (python/cucim/src/cucim/skimage/_vendored/
_ndimage_filters.py, cited as FLT below); every filter runs in libcimx's
sm_100a kernels through the C ABI of include/cimx.h. Arrays may be torch
CUDA tensors, CuPy arrays or any __cuda_array_interface__ / DLPack object;
results come back as the input's array type.
"""

import contextlib
import ctypes
import math
import warnings

import numpy as np
import torch

from . import _arrays, _lib, _util

__all__ = [
    "correlate1d", "convolve1d", "uniform_filter1d", "uniform_filter",
    "gaussian_filter1d", "gaussian_filter", "prewitt", "sobel",
    "generic_gradient_magnitude", "gaussian_gradient_magnitude",
    "generic_laplace", "laplace", "gaussian_laplace",
    "minimum_filter1d", "maximum_filter1d",
]


class _PassList:
    """A list of CimxPass structs plus the tap arrays they point into."""

    def __init__(self):
        self.keep = []
        self.items = []

    def add(self, axis, taps, origin, mode, cval, flags):
        t, ptr = _lib.taps_pointer(taps)
        self.keep.append(t)
        p = _lib.CimxPass()
        # complex taps are (re, im) pairs in t
        ntaps = t.size // 2 if flags & _lib.F_COMPLEX_TAPS else t.size
        p.axis, p.ntaps, p.origin = axis, ntaps, origin
        p.mode, p.cval, p.flags, p.reserved = _lib.MODE_CODES[mode], float(cval), flags, 0
        p.taps = ptr
        self.items.append(p)

    def array(self):
        arr = (_lib.CimxPass * max(1, len(self.items)))(*self.items)
        return arr

    def __len__(self):
        return len(self.items)


def _check_cval(mode, cval, out_dtype):
    """UTIL:27-32."""
    if mode == "constant" and np.dtype(out_dtype).kind in "iu" and not np.isfinite(cval):
        raise NotImplementedError(
            "Non-finite cval is not supported for outputs with integer dtype."
        )


def _build_passes(in_dtype, out_dtype, ndim, specs, cval, algorithm):
    """Resolve (axis, weights, mode, origin, convolve) specs into CimxPasses.

    The first pass reads the input's dtype, later ones the output's (the
    intermediates of _run_1d_filters, _vendored/_ndimage_filters_core.py:145).
    """
    pl = _PassList()
    for i, (axis, w, mode, origin, convolve) in enumerate(specs):
        w = np.asarray(w)
        if w.ndim != 1 or w.size < 1:
            raise RuntimeError("incorrect filter size")
        K = w.size
        axis = _util.normalize_axis(axis, ndim)
        origin = _util.check_origin(origin, K)
        mode = "grid-wrap" if mode == "wrap" else mode
        _util.check_mode(mode)
        pass_in = in_dtype if i == 0 else out_dtype
        if mode == "constant":
            _check_cval(mode, cval, out_dtype)
        flags = _util.pass_flags(pass_in, ndim, axis, K, origin, mode, cval, w.dtype,
                                 convolve, algorithm)
        pl.add(axis, w, origin, mode, cval, flags)
    return pl


# algorithm="tensor" and "tensor_bf16x3": additions of this library (cuCIM
# accepts only "shared_memory", "elementwise" and None). float32 -> float32
# passes with at least 16 taps along lines of at least 2048 samples (where
# they measured faster; see tensor_cores_everywhere) run on the tensor cores
# as banded-Toeplitz products with float32 accumulation: "tensor" splits operands into tf32
# hi + lo (TF32x3, max relative error near 1e-6), "tensor_bf16x3" into
# bfloat16 hi + lo (BF16x3, near 1e-5). Results are close to, not
# bit-identical with, the float32 chain. Other passes run as usual.
TENSOR = "tensor"
TENSOR_BF16X3 = "tensor_bf16x3"
_TENSOR_FLAGS = {TENSOR: _lib.L_TENSOR_TF32X3, TENSOR_BF16X3: _lib.L_TENSOR_BF16X3}


_EXTRA_LIB_FLAGS = 0


@contextlib.contextmanager
def pass_by_pass():
    """Within this block every filter runs one launch per 1-D pass, through
    one scratch volume of the output dtype (the schedule of _run_1d_filters,
    _vendored/_ndimage_filters_core.py:124-163), instead of the fused
    kernels. The results are bit-identical; it only runs slower. A testing
    and debugging aid, not thread-safe."""
    global _EXTRA_LIB_FLAGS
    old = _EXTRA_LIB_FLAGS
    _EXTRA_LIB_FLAGS = old | _lib.L_NO_FUSION
    try:
        yield
    finally:
        _EXTRA_LIB_FLAGS = old


@contextlib.contextmanager
def schedule(lib_flags):
    """Within this block every filter runs with the given CIMX_L_* schedule
    flags (for example _lib.L_NO_VOLUME | _lib.L_NO_ROWSTREAM), which the
    autotuner then leaves alone. All schedules give bit-identical results;
    a testing and measurement aid, not thread-safe."""
    global _EXTRA_LIB_FLAGS
    old = _EXTRA_LIB_FLAGS
    _EXTRA_LIB_FLAGS = old | int(lib_flags)
    try:
        yield
    finally:
        _EXTRA_LIB_FLAGS = old


def _hashable(obj):
    """`obj` with lists turned into tuples, or None when it cannot be a key."""
    if not isinstance(obj, list):
        try:  # scalars and tuples of scalars: already a key
            hash(obj)
            return obj
        except TypeError:
            pass
    if isinstance(obj, (list, tuple)):
        items = tuple(_hashable(o) for o in obj)
        return None if any(i is None and o is not None for i, o in zip(items, obj)) else items
    try:
        hash(obj)
    except TypeError:
        return None
    return obj


# Resolved pass lists (CimxPass arrays and the tap arrays they point into),
# keyed by everything they depend on: repeated calls with the same filter
# skip the tap arithmetic and the struct building.
_PASS_CACHE = {}


@contextlib.contextmanager
def tensor_cores_everywhere():
    """Within this block algorithm="tensor" / "tensor_bf16x3" runs every
    eligible pass on the tensor cores, whatever its line length. By default
    only passes along lines of at least 2048 samples do (on shorter lines the
    plain kernels measured faster). A testing and measurement aid, not
    thread-safe."""
    global _EXTRA_LIB_FLAGS
    old = _EXTRA_LIB_FLAGS
    _EXTRA_LIB_FLAGS = old | _lib.L_TENSOR_ALL_LINES
    try:
        yield
    finally:
        _EXTRA_LIB_FLAGS = old


def _complex_output(output, in_dt):
    """_get_output (UTIL:49-71) when the output is complex: the default is
    the input's dtype promoted to complex64; a dtype-like real output is
    promoted with a warning, a dtype name or an array must be complex."""
    if output is None:
        return None, np.promote_types(in_dt, np.complex64)
    if isinstance(output, str):
        if np.dtype(output).kind != "c":
            raise RuntimeError("output must have complex dtype")
        return output, None
    if _arrays.is_dtype_like(output):
        dt = _arrays.np_dtype(output) if isinstance(output, torch.dtype) else np.dtype(output)
        if dt.kind != "c":
            warnings.warn("promoting specified output dtype to complex")
            return np.promote_types(dt, np.complex64), None
        return output, None
    if _arrays.np_dtype(_arrays.as_tensor(output)).kind != "c":
        raise RuntimeError("output must have complex dtype")
    return output, None


def _run(input, specs, output, cval, algorithm=None, cache_key=None, complex_weights=False):
    """Apply the pass list to `input` into `output` (FLT:363-396 semantics).
    `cache_key`: a hashable description of `specs` (None: not cached).
    Complex input or weights give a complex output (CORE:195-203)."""
    x = _arrays.as_tensor(input)
    xc = x.contiguous()
    if x.dtype.is_complex or complex_weights:
        output, default_dt = _complex_output(output, _arrays.np_dtype(xc))
        slot = _arrays.output_slot(output, input, xc, dtype=default_dt)
    else:
        slot = _arrays.output_slot(output, input, xc)
    out_dt = slot.dtype
    lib_flags = _EXTRA_LIB_FLAGS
    if algorithm in _TENSOR_FLAGS:
        lib_flags, algorithm = lib_flags | _TENSOR_FLAGS[algorithm], None
    key = None
    if cache_key is not None:
        # torch dtypes stand for the numpy ones here (one-to-one, and cheaper)
        key = (cache_key, xc.dtype, slot.work.dtype, xc.dim(), _hashable(cval), algorithm)
    hit = _PASS_CACHE.get(key) if key is not None else None
    if hit is None:
        in_dt = _arrays.np_dtype(xc)
        pl = _build_passes(in_dt, out_dt, xc.dim(), specs() if callable(specs) else specs, cval,
                           algorithm)
        hit = (pl, pl.array(), len(pl))
        if key is not None and len(_PASS_CACHE) < 1024:
            _PASS_CACHE[key] = hit
    _, arr, npasses = hit
    a_in = _arrays.to_cimx(xc)
    a_out = _arrays.to_cimx(slot.work)
    rc = _lib.lib.cimx_separable(ctypes.byref(a_in), ctypes.byref(a_out), arr, npasses,
                                 lib_flags, _arrays.stream_of(xc))
    _lib.check(rc, "separable filter")
    return slot.result()


# --------------------------------------------------------------- correlate1d

def _correlate_or_convolve1d(input, weights, axis, output, mode, cval, origin,
                             convolution, algorithm):
    x = _arrays.as_tensor(input)
    axis = _util.normalize_axis(axis, x.dim())
    w = _weights_to_host(weights)
    if not convolution and w.dtype.kind == "c":
        # numpy.correlate conjugates the weights rather than the input
        w = w.conj()
    if algorithm not in (None, "shared_memory", "elementwise", TENSOR, TENSOR_BF16X3):
        raise ValueError("algorithm must be 'shared_memory', 'elementwise' or None")
    if algorithm == "shared_memory" and mode == "constant" and (
        not np.isfinite(cval) or (cval < 0 and _arrays.np_dtype(x).kind == "u")
    ):
        warnings.warn(
            f"{cval=} and input.dtype={_arrays.np_dtype(x)} is unsupported for algorithm "
            "'shared_memory', falling back to elementwise"
        )
    return _run(input, [(axis, w, mode, origin, convolution)], output, cval, algorithm,
                complex_weights=w.dtype.kind == "c")


def _weights_to_host(weights):
    if isinstance(weights, np.ndarray):
        return weights
    if isinstance(weights, torch.Tensor):
        return weights.detach().cpu().numpy()
    if hasattr(weights, "__cuda_array_interface__") or hasattr(weights, "__dlpack__"):
        return _arrays.as_tensor(weights).cpu().numpy()
    return np.asarray(weights)


def correlate1d(input, weights, axis=-1, output=None, mode="reflect", cval=0.0, origin=0,
                *, algorithm=None):
    """One-dimensional correlation along `axis` (FLT:135-178)."""
    return _correlate_or_convolve1d(input, weights, axis, output, mode, cval, origin, False,
                                    algorithm)


def convolve1d(input, weights, axis=-1, output=None, mode="reflect", cval=0.0, origin=0,
               *, algorithm=None):
    """One-dimensional convolution along `axis` (FLT:180-221)."""
    return _correlate_or_convolve1d(input, weights, axis, output, mode, cval, origin, True,
                                    algorithm)


# -------------------------------------------------------------- uniform

def uniform_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0, origin=0,
                     *, algorithm=None):
    """FLT:399-444."""
    x = _arrays.as_tensor(input)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    w = np.full(size, 1 / size, dtype=wdt)
    return correlate1d(input, w, axis, output, mode, cval, origin, algorithm=algorithm)


def uniform_filter(input, size=3, output=None, mode="reflect", cval=0.0, origin=0, axes=None,
                   *, algorithm=None):
    """FLT:447-521."""
    x = _arrays.as_tensor(input)
    axes = _util.check_axes(axes, x.dim())
    n = len(axes)
    sizes = _util.fix_sequence_arg(size, n, "size", int)
    origins = _util.fix_sequence_arg(origin, n, "origin", int)
    modes = _util.fix_sequence_arg(mode, n, "mode", _util.check_mode)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)

    def specs():
        return [(ax, np.full(s, 1 / s, dtype=wdt), m, o, False)
                for ax, s, m, o in zip(axes, sizes, modes, origins) if s > 1]

    key = _hashable(("uniform", tuple(axes), tuple(sizes), tuple(modes), tuple(origins)))
    return _run(input, specs, output, cval, algorithm, cache_key=key)


# ------------------------------------------------------------- gaussian

_TAPS = {}


def _gaussian_kernel1d(sigma, order, radius, dtype=np.float64):
    """Memoised _gaussian_taps (read-only arrays: the taps of a sigma, order,
    radius and dtype never change)."""
    key = (float(sigma), int(order), int(radius), np.dtype(dtype).str)
    w = _TAPS.get(key)
    if w is None:
        w = _gaussian_taps(sigma, order, radius, dtype)
        w.setflags(write=False)
        if len(_TAPS) < 4096:
            _TAPS[key] = w
    return w


def _gaussian_taps(sigma, order, radius, dtype=np.float64):
    """Gaussian (derivative) correlation taps, FLT:689-717.

    Order 0: the normalised exp(-x^2 / (2 sigma^2)) in float64 (returned as
    float64 whatever `dtype` says, as cuCIM does). Order n: the Gaussian times
    the polynomial q_n obtained by applying q -> q' + q * p' (p' = -x/sigma^2)
    n times to q_0 = 1, reversed into correlation order and cast to `dtype`.
    The numpy expressions are evaluated in the same order as cuCIM's so the
    float64 taps are identical.
    """
    if order < 0:
        raise ValueError("order must be non-negative")
    sigma2 = sigma * sigma
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / sigma2 * x**2)
    phi /= phi.sum()
    if order == 0:
        return phi
    powers = np.arange(order + 1)
    coeffs = np.zeros(order + 1)
    coeffs[0] = 1
    # derivative operator on polynomial coefficients plus multiplication by p'
    op = np.diag(powers[1:], 1) + np.diag(np.ones(order) / -sigma2, -1)
    for _ in range(order):
        coeffs = op.dot(coeffs)
    qx = (x[:, None] ** powers).dot(coeffs)
    return np.ascontiguousarray((qx * phi)[::-1], dtype=dtype)


def _gaussian_specs(ndim, in_dtype, sigma, order, mode, truncate, radius, axes):
    """Per-axis gaussian passes of gaussian_filter (FLT:580-686); None when
    every sigma is below 1e-15 (the filter is then a copy)."""
    axes = _util.check_axes(axes, ndim)
    n = len(axes)
    sigmas = _util.fix_sequence_arg(sigma, n, "sigma", float)
    if n == 0 or all(s < 1e-15 for s in sigmas):
        return None
    orders = _util.fix_sequence_arg(order, n, "order", int)
    modes = _util.fix_sequence_arg(mode, n, "mode", str)
    radiuses = _util.fix_sequence_arg(radius, n, "radius")
    truncate = float(truncate)
    wdt = np.promote_types(np.dtype(in_dtype), np.float32)
    cache = {}
    specs = []
    for i in range(n):
        if not sigmas[i] > 1e-15:
            continue
        key = (sigmas[i], orders[i], radiuses[i])
        if key not in cache:
            r = radiuses[i]
            if r is None:
                r = int(truncate * float(sigmas[i]) + 0.5)
            cache[key] = None if r <= 0 else _gaussian_kernel1d(sigmas[i], orders[i], r, wdt)
        w = cache[key]
        _util.check_mode(modes[i] if modes[i] != "wrap" else "grid-wrap")
        if w is not None:
            specs.append((axes[i], w, modes[i], 0, False))
    return specs


def gaussian_filter(input, sigma, order=0, output=None, mode="reflect", cval=0.0,
                    truncate=4.0, radius=None, axes=None, *, algorithm=None):
    """Multi-dimensional Gaussian filter (FLT:580-686)."""
    x = _arrays.as_tensor(input)

    def specs():
        return _gaussian_specs(x.dim(), _arrays.np_dtype(x), sigma, order, mode, truncate,
                               radius, axes) or []

    key = _hashable(("gaussian", sigma, order, mode, truncate, radius, axes))
    return _run(input, specs, output, cval, algorithm, cache_key=key)


def gaussian_filter1d(input, sigma, axis=-1, order=0, output=None, mode="reflect", cval=0.0,
                      truncate=4.0, *, algorithm=None):
    """One-dimensional Gaussian filter (FLT:524-577)."""
    x = _arrays.as_tensor(input)
    radius = int(float(truncate) * float(sigma) + 0.5)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    w = _gaussian_kernel1d(sigma, int(order), radius, wdt)
    return correlate1d(input, w, axis, output, mode, cval, algorithm=algorithm)


# ------------------------------------------------------------ sobel/prewitt

def _prewitt_or_sobel(input, axis, output, mode, cval, smooth, algorithm):
    """FLT:782-803: [-1, 0, 1] along `axis`, `smooth` along the others."""
    x = _arrays.as_tensor(input)
    axis = _util.normalize_axis(axis, x.dim())
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    _util.check_mode(mode)

    def specs():
        diff = np.array([-1, 0, 1], dtype=wdt)
        return [(a, diff if a == axis else smooth, mode, 0, False) for a in range(x.dim())]

    key = _hashable(("prewitt_or_sobel", axis, mode, tuple(np.asarray(smooth).tolist()),
                     np.asarray(smooth).dtype.str))
    return _run(input, specs, output, cval, algorithm, cache_key=key)


def sobel(input, axis=-1, output=None, mode="reflect", cval=0.0, *, algorithm=None):
    """Sobel filter along `axis` (FLT:751-779)."""
    x = _arrays.as_tensor(input)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    return _prewitt_or_sobel(input, axis, output, mode, cval, np.array([1, 2, 1], dtype=wdt),
                             algorithm)


def prewitt(input, axis=-1, output=None, mode="reflect", cval=0.0, *, algorithm=None):
    """Prewitt filter along `axis` (FLT:720-748)."""
    x = _arrays.as_tensor(input)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    return _prewitt_or_sobel(input, axis, output, mode, cval, np.ones(3, dtype=wdt), algorithm)


# ------------------------------------------------------ gradient magnitude

def _gradient_magnitude(input, chains, output, cval, algorithm=None):
    """sqrt(sum over chains of chain(input)^2), FLT:1012-1097 rounding."""
    x = _arrays.as_tensor(input)
    xc = x.contiguous()
    slot = _arrays.output_slot(output, input, xc)
    out_dt = slot.dtype
    if out_dt.kind != "f" or out_dt.itemsize < 4:
        raise NotImplementedError("gradient magnitude supports float32/float64 outputs only")
    lens = {len(c) for c in chains}
    if len(lens) != 1:
        raise RuntimeError("gradient chains must have equal length")
    pl = _PassList()
    for chain in chains:
        sub = _build_passes(_arrays.np_dtype(xc), out_dt, xc.dim(), chain, cval, algorithm)
        pl.keep += sub.keep
        pl.items += sub.items
    arr = pl.array()
    a_in = _arrays.to_cimx(xc)
    a_out = _arrays.to_cimx(slot.work)
    rc = _lib.lib.cimx_gradient_magnitude(ctypes.byref(a_in), ctypes.byref(a_out), arr,
                                          len(chains), lens.pop(), _arrays.stream_of(xc))
    _lib.check(rc, "gradient magnitude")
    return slot.result()


def _combine(acc, term, op):
    """acc (+|-)= term in acc's dtype (libcimx; integers wrap)."""
    a_acc, a_t = _arrays.to_cimx(acc), _arrays.to_cimx(term)
    rc = _lib.lib.cimx_combine(ctypes.byref(a_acc), ctypes.byref(a_t), op,
                               _arrays.stream_of(acc))
    _lib.check(rc, "combine")


def _laplace_sum(input, chains, output, cval, algorithm=None):
    """sum over chains of chain(input), accumulated in the output dtype
    (FLT:806-890 with the derivative of each axis a pass chain)."""
    x = _arrays.as_tensor(input)
    xc = x.contiguous()
    slot = _arrays.output_slot(output, input, xc)
    out_dt = slot.dtype
    lens = {len(c) for c in chains}
    if len(lens) != 1:
        raise RuntimeError("laplace chains must have equal length")
    if algorithm in _TENSOR_FLAGS:
        algorithm = None  # the composite runs the plain passes
    pl = _PassList()
    for chain in chains:
        sub = _build_passes(_arrays.np_dtype(xc), out_dt, xc.dim(), chain, cval, algorithm)
        pl.keep += sub.keep
        pl.items += sub.items
    arr = pl.array()
    a_in = _arrays.to_cimx(xc)
    a_out = _arrays.to_cimx(slot.work)
    rc = _lib.lib.cimx_laplace(ctypes.byref(a_in), ctypes.byref(a_out), arr, len(chains),
                               lens.pop(), _arrays.stream_of(xc))
    _lib.check(rc, "laplace")
    return slot.result()


def generic_laplace(input, derivative2, output=None, mode="reflect", cval=0.0,
                    extra_arguments=(), extra_keywords=None, *, axes=None):
    """FLT:806-890 with a user-supplied second-derivative callable: the
    first axis into `output`, every further axis into one temporary of the
    output dtype that is added in place (in libcimx, integers wrap)."""
    if extra_keywords is None:
        extra_keywords = {}
    x = _arrays.as_tensor(input)
    axes = _util.check_axes(axes, x.dim())
    n = len(axes)
    slot = _arrays.output_slot(output, input, x.contiguous())
    if n == 0:
        # elementwise copy with conversion: an empty pass list
        _run(input, [], slot.work, cval)
        return slot.result()
    modes = _util.fix_sequence_arg(mode, n, "mode", _util.check_mode)

    def into(res, dst):
        r = _arrays.as_tensor(res)
        if r.data_ptr() != dst.data_ptr():
            dst.copy_(r)

    into(derivative2(input, axes[0], slot.work, modes[0], cval, *extra_arguments,
                     **extra_keywords), slot.work)
    if n > 1:
        tmp = torch.empty_like(slot.work)
        for i in range(1, n):
            into(derivative2(input, axes[i], tmp, modes[i], cval, *extra_arguments,
                             **extra_keywords), tmp)
            _combine(slot.work, tmp, _lib.COMBINE_ADD)
    return slot.result()


def laplace(input, output=None, mode="reflect", cval=0.0, *, axes=None, algorithm=None):
    """Laplace filter from [1, -2, 1] second differences (FLT:893-930): one
    correlate1d per axis, summed in the output dtype."""
    x = _arrays.as_tensor(input)
    axes = _util.check_axes(axes, x.dim())
    if not axes:
        return generic_laplace(input, None, output, mode, cval, axes=axes)
    modes = _util.fix_sequence_arg(mode, len(axes), "mode", _util.check_mode)
    wdt = np.promote_types(_arrays.np_dtype(x), np.float32)
    w = np.array([1, -2, 1], dtype=wdt)
    chains = [[(ax, w, m, 0, False)] for ax, m in zip(axes, modes)]
    return _laplace_sum(input, chains, output, cval, algorithm)


def gaussian_laplace(input, sigma, output=None, mode="reflect", cval=0.0, *, axes=None,
                     algorithm=None, **kwargs):
    """Laplace filter from Gaussian second derivatives (FLT:933-1009): per
    filtered axis a gaussian_filter with order 2 on that axis (sigma 0 on the
    axes not filtered) in that axis' mode, summed in the output dtype."""
    x = _arrays.as_tensor(input)
    ndim = x.dim()
    axes = _util.check_axes(axes, ndim)
    if not axes:
        return generic_laplace(input, None, output, mode, cval, axes=axes)
    n = len(axes)
    sigmas = _util.fix_sequence_arg(sigma, n, "sigma", float)
    if n < ndim:
        full = [0.0] * ndim
        for s_, ax in zip(sigmas, axes):
            full[ax] = s_
        sigmas = full
    modes = _util.fix_sequence_arg(mode, n, "mode", _util.check_mode)
    truncate = kwargs.pop("truncate", 4.0)
    radius = kwargs.pop("radius", None)
    if kwargs:
        raise TypeError(f"unexpected keyword arguments {sorted(kwargs)}")
    chains = []
    for ax, m in zip(axes, modes):
        order = [0] * ndim
        order[ax] = 2
        specs = _gaussian_specs(ndim, _arrays.np_dtype(x), sigmas, order, m, truncate, radius,
                                None)
        chains.append(specs if specs is not None else [])
    # every chain drops the same zero-sigma axes, so the chains have equal length
    return _laplace_sum(input, chains, output, cval, algorithm)


def _min_or_max_1d(input, size, axis, output, mode, cval, origin, is_max):
    """FLT:1412-1448: one launch of libcimx's min/max kernel."""
    x = _arrays.as_tensor(input)
    if x.dtype.is_complex:
        raise NotImplementedError("complex arrays are not supported")
    size = int(size)
    if size < 1:
        raise RuntimeError("incorrect filter size")
    axis = _util.normalize_axis(axis, x.dim())
    origin = _util.check_origin(origin, size)
    mode = "grid-wrap" if mode == "wrap" else mode
    _util.check_mode(mode)
    xc = x.contiguous()
    slot = _arrays.output_slot(output, input, xc)
    a_in, a_out = _arrays.to_cimx(xc), _arrays.to_cimx(slot.work)
    rc = _lib.lib.cimx_min_max_1d(ctypes.byref(a_in), ctypes.byref(a_out), size, axis, origin,
                                  _lib.MODE_CODES[mode], float(cval), 1 if is_max else 0,
                                  _arrays.stream_of(xc))
    _lib.check(rc, "min/max filter")
    return slot.result()


def minimum_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0, origin=0):
    """Minimum over `size` elements along `axis` (FLT:1362-1385)."""
    return _min_or_max_1d(input, size, axis, output, mode, cval, origin, False)


def maximum_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0, origin=0):
    """Maximum over `size` elements along `axis` (FLT:1388-1411)."""
    return _min_or_max_1d(input, size, axis, output, mode, cval, origin, True)


def generic_gradient_magnitude(input, derivative, output=None, mode="reflect", cval=0.0,
                               extra_arguments=(), extra_keywords=None, *, axes=None):
    """FLT:1012-1097 with a user-supplied derivative callable: the squares,
    sums and square root run in libcimx, each operation rounded on its own
    as CuPy's in-place operators round it."""
    if extra_keywords is None:
        extra_keywords = {}
    x = _arrays.as_tensor(input)
    ndim = x.dim()
    axes = _util.check_axes(axes, ndim)
    modes = _util.fix_sequence_arg(mode, len(axes), "mode", _util.check_mode)
    slot = _arrays.output_slot(output, input, x.contiguous())
    if ndim == 0:
        slot.work.copy_(x)
        return slot.result()
    if slot.dtype.kind != "f" or slot.dtype.itemsize < 4:
        raise NotImplementedError(
            "generic_gradient_magnitude supports float32 / float64 outputs only")

    def into(res, dst):
        r = _arrays.as_tensor(res)
        if r.data_ptr() != dst.data_ptr():
            dst.copy_(r)

    def square_acc(acc, term, first):
        a_acc, a_t = _arrays.to_cimx(acc), _arrays.to_cimx(term)
        rc = _lib.lib.cimx_square_accumulate(ctypes.byref(a_acc), ctypes.byref(a_t),
                                             1 if first else 0, _arrays.stream_of(acc))
        _lib.check(rc, "gradient magnitude")

    acc = slot.work
    into(derivative(input, axes[0], acc, modes[0], cval, *extra_arguments, **extra_keywords),
         acc)
    square_acc(acc, acc, True)
    if len(axes) > 1:
        tmp = torch.empty_like(acc)
        for i in range(1, len(axes)):
            into(derivative(input, axes[i], tmp, modes[i], cval, *extra_arguments,
                            **extra_keywords), tmp)
            square_acc(acc, tmp, False)
    a_acc = _arrays.to_cimx(acc)
    _lib.check(_lib.lib.cimx_sqrt(ctypes.byref(a_acc), _arrays.stream_of(acc)), "sqrt")
    return slot.result()


def gaussian_gradient_magnitude(input, sigma, output=None, mode="reflect", cval=0.0, *,
                                axes=None, algorithm=None, **kwargs):
    """Gradient magnitude with Gaussian derivatives (FLT:1100-1157)."""
    x = _arrays.as_tensor(input)
    ndim = x.dim()
    axes = _util.check_axes(axes, ndim)
    modes = _util.fix_sequence_arg(mode, len(axes), "mode", _util.check_mode)
    truncate = kwargs.pop("truncate", 4.0)
    radius = kwargs.pop("radius", None)
    if kwargs:
        raise TypeError(f"unexpected keyword arguments {sorted(kwargs)}")
    chains = []
    for ax, m in zip(axes, modes):
        order = [0] * ndim
        order[ax] = 1
        specs = _gaussian_specs(ndim, _arrays.np_dtype(x), sigma, order, m, truncate, radius,
                                None)
        chains.append(specs if specs is not None else [])
    return _gradient_magnitude(input, chains, output, cval, algorithm)
