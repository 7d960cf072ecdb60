"""Parity oracle — TEST INFRASTRUCTURE ONLY.

A CPU restatement (numpy + the C core in cimx_oracle.c) of cuCIM's separable
filtering path: the host-side dtype rules, the choice between the
shared-memory and elementwise kernels (which decides how a constant-mode fill
value is rounded and whether zero taps are skipped), the per-axis ping-pong,
and the composite operations built on it. Only tests/, the smoke check and
bench.py's CPU baseline may import this module; the library never does.

Citations are relative to python/cucim/src/cucim/skimage in rapidsai/cucim
(cuCIM 26.10.00). FLT = _vendored/_ndimage_filters.py,
CORE = _vendored/_ndimage_filters_core.py, UTIL = _vendored/_ndimage_util.py,
SEP = filters/_separable_filtering.py.
"""

import ctypes
import math
from itertools import combinations_with_replacement

import numpy as np

from . import build_oracle

_lib = ctypes.CDLL(build_oracle.build())
_lib.oracle_correlate1d.argtypes = [
    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
    ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
    ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
]
_lib.oracle_correlate1d.restype = None
_lib.oracle_cval_as_input.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int]
_lib.oracle_cval_as_input.restype = ctypes.c_double
_lib.oracle_cast.argtypes = [
    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
]
_lib.oracle_cast.restype = None
_lib.oracle_min_max1d.argtypes = [
    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
    ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_double, ctypes.c_int,
]
_lib.oracle_min_max1d.restype = None
_lib.oracle_rgb2gray.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
_lib.oracle_rgb2gray.restype = None
_lib.oracle_fma.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                            ctypes.c_int, ctypes.c_void_p]
_lib.oracle_fma.restype = None
_lib.oracle_frangi_scale.argtypes = [
    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
    ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
    ctypes.c_void_p,
]
_lib.oracle_frangi_scale.restype = None

MODES = {
    "reflect": 0, "grid-mirror": 0, "mirror": 1, "nearest": 2,
    "grid-wrap": 3, "wrap": 3, "constant": 4,
}
# The mode names UTIL:95-108 accepts ('grid-reflect' passes the check but has
# no boundary code in UTIL:186-308, so cuCIM fails on it later).
_VALID_MODES = (
    "reflect", "constant", "nearest", "mirror", "wrap", "grid-mirror",
    "grid-wrap", "grid-reflect",
)

# sharedMemPerBlock on every CUDA device cuCIM targets (48 KiB, SEP:130-152).
SHARED_BLOCK_BYTES = 49152

THREADS = 1  # OpenMP threads the C core may use


def _dchar(dt):
    return ord(np.dtype(dt).char)


# ---------------------------------------------------------------- dtype rules

_NEW_FLOAT = {
    "f": np.float32, "d": np.float64, "e": np.float32, "b": np.float32,
    "B": np.float32, "h": np.float32, "H": np.float32, "?": np.float32,
}


def supported_float_type(dt):
    """_shared/utils.py:1131-1179."""
    dt = np.dtype(dt)
    if dt.kind == "c":
        raise ValueError("complex valued input is not supported")
    return np.dtype(_NEW_FLOAT.get(dt.char, np.float64))


def weights_dtype(input_dtype, w_dtype):
    """UTIL:35-46 with use_cucim_casting=True."""
    w_dtype = np.dtype(w_dtype)
    in_dtype = np.dtype(input_dtype)
    if w_dtype.kind == "c" or in_dtype.kind == "c":
        real = np.empty(0, in_dtype).real.dtype
        return np.promote_types(real, np.complex64)
    if w_dtype.kind in "iub":
        return supported_float_type(w_dtype)
    return np.promote_types(np.dtype(input_dtype), np.float32)


def img_as_float(image):
    """util/dtype.py:489 -> _convert (:219), uint/int -> float branch (:355-372)."""
    image = np.asarray(image)
    dt = image.dtype
    out_t = supported_float_type(dt)
    if dt.kind == "f":
        return image.astype(out_t) if dt != out_t else image
    if dt.kind == "b":
        return image.astype(out_t)
    info = np.iinfo(dt)
    comp = np.float32 if dt.itemsize <= 4 and out_t == np.float32 else np.float64
    if out_t == np.float64:
        comp = np.float64
    scale = comp(1.0 / info.max)
    res = np.multiply(image.astype(comp), scale, dtype=comp)
    if dt.kind == "i":
        res = np.maximum(res, comp(-1.0))
    return res.astype(out_t)


def convert_to_float(image, preserve_range):
    """_shared/utils.py:1019-1052."""
    image = np.asarray(image)
    if image.dtype == np.float16:
        return image.astype(np.float32)
    if preserve_range:
        if image.dtype.char not in "df":
            image = image.astype(supported_float_type(image.dtype))
        return image
    return img_as_float(image)


# ------------------------------------------------------------ argument checks

def check_mode(mode):
    """UTIL:95-108."""
    if mode not in _VALID_MODES:
        raise RuntimeError(f"boundary mode not supported (actual: {mode})")
    if mode == "grid-reflect":
        raise RuntimeError(f"boundary mode not supported (actual: {mode})")
    return mode


def check_origin(origin, width):
    """UTIL:88-92."""
    origin = int(origin)
    if (width // 2 + origin < 0) or (width // 2 + origin >= width):
        raise ValueError("invalid origin")
    return origin


def fix_sequence_arg(arg, ndim, name, conv=lambda x: x):
    """UTIL:74-85."""
    if isinstance(arg, str):
        return [conv(arg)] * ndim
    try:
        arg = iter(arg)
    except TypeError:
        return [conv(arg)] * ndim
    lst = [conv(x) for x in arg]
    if len(lst) != ndim:
        raise RuntimeError(f"{name} must have length equal to input rank")
    return lst


def check_axes(axes, ndim):
    """UTIL:111-127."""
    if axes is None:
        return tuple(range(ndim))
    if np.isscalar(axes):
        axes = (int(axes),)
    else:
        axes = tuple(int(a) for a in axes)
        for ax in axes:
            if ax < -ndim or ax > ndim - 1:
                raise np.exceptions.AxisError(f"specified axis: {ax} is out of range")
        axes = tuple(a % ndim for a in axes)
    if len(set(axes)) != len(axes):
        raise ValueError("axes must be unique")
    return axes


# ------------------------------------------------------------- kernel choice

def _smem_bytes(ndim, axis, K, anchor, itemsize):
    """SEP:17-69 (_get_constants) and SEP:72-88 (_get_smem_shape)."""
    hpn = max(K - anchor, anchor)
    if ndim == 2:
        bx, by, bz = (16, 16, 1) if axis == 1 else (32, 8, 1)
        halo = math.ceil(hpn / (bx if axis == 1 else by))
    else:
        if axis == 2:
            bx, by, bz = 16, 4, 4
            halo = math.ceil(hpn / bx)
        elif axis == 1:
            bx, by, bz = 32, 4, 4
            halo = math.ceil(hpn / by)
        else:
            bx, by, bz = 32, 4, 4
            halo = math.ceil(hpn / bz)
    ppb = max(4, halo)
    return (ppb + 2 * halo) * bx * by * bz * itemsize


def choose_path(ndim, axis, K, anchor, mode, cval, in_dtype, algorithm=None):
    """FLT:271-344: 'shared_memory' or 'elementwise' for one correlate1d call."""
    in_dtype = np.dtype(in_dtype)
    default = algorithm is None
    if default:
        if ndim == 2 and K <= 256 and not (cval < 0 and mode == "constant" and in_dtype.kind == "u"):
            algorithm = "shared_memory"
        else:
            algorithm = "elementwise"
    elif algorithm == "shared_memory":
        if mode == "constant" and (not np.isfinite(cval) or (cval < 0 and in_dtype.kind == "u")):
            algorithm = "elementwise"
    elif algorithm != "elementwise":
        raise ValueError("algorithm must be 'shared_memory', 'elementwise' or None")
    if algorithm == "shared_memory":
        if ndim not in (2, 3):
            raise NotImplementedError(f"shared_memory not implemented for ndim={ndim}")
        # compile failure on a non-finite fill value (SEP:219-223) and the
        # shared-memory size check (SEP:1007-1017) fall back to elementwise
        if mode == "constant" and not np.isfinite(cval):
            return "elementwise"
        if K > 32 and _smem_bytes(ndim, axis, K, anchor, in_dtype.itemsize) > SHARED_BLOCK_BYTES:
            return "elementwise"
    return algorithm


def pass_params(in_dtype, ndim, axis, weights, mode, cval, origin, convolve, algorithm=None):
    """Everything the per-output arithmetic of one correlate1d call depends on.

    Returns (taps_in_W (float64 array), anchor, mode_code, cval_w, w64, skip_zero).
    """
    weights = np.asarray(weights)
    if weights.ndim != 1 or weights.size < 1:
        raise RuntimeError("incorrect filter size")
    K = weights.size
    origin = check_origin(origin, K)
    if mode == "wrap":
        mode = "grid-wrap"
    check_mode(mode)
    if convolve:
        weights = weights[::-1]
        origin = -origin
        if K % 2 == 0:
            origin -= 1
    anchor = K // 2 + origin
    wdt = weights_dtype(in_dtype, weights.dtype)
    w64 = wdt == np.float64
    taps = weights.astype(wdt).astype(np.float64)
    path = choose_path(ndim, axis, K, anchor, mode, cval, in_dtype, algorithm)
    if path == "shared_memory":
        cval_w = _lib.oracle_cval_as_input(float(cval), _dchar(in_dtype), int(w64))
        skip_zero = False
    else:
        cval_w = float(cval) if w64 else float(np.float32(cval))
        skip_zero = True
    return taps, anchor, MODES[mode], cval_w, int(w64), int(skip_zero), path


def get_output(output, input, shape=None, complex_output=False):
    """UTIL:49-71."""
    shape = input.shape if shape is None else shape
    if output is None:
        dt = np.promote_types(input.dtype, np.complex64) if complex_output else input.dtype
        return np.empty(shape, dtype=dt)
    if isinstance(output, str):
        if complex_output and np.dtype(output).kind != "c":
            raise RuntimeError("output must have complex dtype")
        return np.empty(shape, dtype=np.dtype(output))
    if isinstance(output, (type, np.dtype)):
        dt = np.dtype(output)
        if complex_output and dt.kind != "c":
            dt = np.promote_types(dt, np.complex64)
        return np.empty(shape, dtype=dt)
    if output.shape != shape:
        raise RuntimeError("output shape not correct")
    if complex_output and output.dtype.kind != "c":
        raise RuntimeError("output must have complex dtype")
    return output


# --------------------------------------------------------------- 1-D passes

def _run_pass(x, out, axis, taps, anchor, mode_code, cval_w, w64, skip_zero):
    x = np.ascontiguousarray(x)
    assert out.flags.c_contiguous and out.shape == x.shape
    shape = x.shape
    outer = int(np.prod(shape[:axis], dtype=np.int64))
    L = shape[axis]
    inner = int(np.prod(shape[axis + 1:], dtype=np.int64))
    t = np.ascontiguousarray(taps, dtype=np.float64)
    _lib.oracle_correlate1d(
        x.ctypes.data, ord(x.dtype.char), out.ctypes.data, ord(out.dtype.char),
        outer, L, inner, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t.size,
        anchor, mode_code, cval_w, w64, skip_zero, THREADS,
    )
    return out


def _map_coords(ix, n, mode):
    """UTIL:186-308 on an index array: the coordinate each index reads, -1
    outside the array in constant mode."""
    ix = np.asarray(ix, dtype=np.int64)
    inside = (ix >= 0) & (ix < n)
    if mode == "constant":
        return np.where(inside, ix, -1)
    if mode == "nearest":
        return np.clip(ix, 0, n - 1)
    if mode == "grid-wrap":
        return np.mod(ix, n)
    if mode in ("reflect", "grid-mirror"):
        m = np.where(ix < 0, -1 - ix, ix) % (2 * n)
        return np.where(inside, ix, np.minimum(m, 2 * n - 1 - m))
    if mode == "mirror":
        if n == 1:
            return np.zeros_like(ix)
        m = np.abs(ix)
        m = 1 + (m - 1) % (2 * n - 2)
        return np.where(inside, ix, np.minimum(m, 2 * n - 2 - m))
    raise RuntimeError(f"boundary mode not supported (actual: {mode})")


def _complex_correlate1d(input, weights, axis, out, mode, cval, origin, algorithm, convolve):
    """cuCIM's correlate kernels instantiated with W = complex<float> /
    complex<double> (FLT:224-244, CORE:195-203, SEP:720-760). Per output:
    sum = (W)0, then for each tap (skipped by the elementwise kernel when it
    is 0 + 0i) sum = sum + value * w with the complex product
    (x.r w.r - x.i w.i, x.i w.r + x.r w.i) contracted into
    p.r = fma(x.r, w.r, -(x.i w.i)), p.i = fma(x.i, w.r, x.r w.i) and each
    part added with one rounding; out = (D)sum part by part. value: the
    input's parts; a real input x is (x, +0), except in the elementwise
    kernel outside constant mode, whose cast<W>() rule gives a negative or
    NaN float x the imaginary part -0; the fill value is cast<W>(cval)
    (elementwise) or (W)(T)cval (shared memory)."""
    x = np.asarray(input)
    weights = np.asarray(weights)
    K = weights.size
    origin = check_origin(origin, K)
    if mode == "wrap":
        mode = "grid-wrap"
    check_mode(mode)
    if convolve:
        weights = weights[::-1]
        origin = -origin
        if K % 2 == 0:
            origin -= 1
    anchor = K // 2 + origin
    wdt = weights_dtype(x.dtype, weights.dtype)
    R = np.float64 if wdt == np.complex128 else np.float32
    taps = weights.astype(wdt)
    path = choose_path(x.ndim, axis, K, anchor, mode, cval, x.dtype, algorithm)
    elementwise = path != "shared_memory"
    # the fill value as W
    if elementwise:
        cre, cim = R(cval), R(0.0) if cval >= 0 else R(-0.0)
    else:
        t = x.dtype if x.dtype.kind != "c" else np.empty(0, x.dtype).real.dtype
        if t.kind in "iu":
            cre = R(_lib.oracle_cval_as_input(float(cval), _dchar(x.dtype), int(R == np.float64)))
        else:
            cre = R(np.asarray(cval).astype(t))
        cim = R(0.0)
    xs = np.moveaxis(x, axis, -1)
    if x.dtype.kind == "c":
        xr, xi = xs.real.astype(R), xs.imag.astype(R)
    else:
        xr = xs.astype(R)
        neg = elementwise and mode != "constant" and x.dtype.kind == "f"
        xi = np.where(~(xr >= 0), R(-0.0), R(0.0)).astype(R) if neg else np.zeros_like(xr)
    L = xs.shape[-1]
    pos = np.arange(L)
    sr = np.zeros(xs.shape, R)
    si = np.zeros(xs.shape, R)
    for k in range(K):
        wr, wi = R(taps[k].real), R(taps[k].imag)
        if elementwise and wr == 0 and wi == 0:
            continue
        m = _map_coords(pos - anchor + k, L, mode)
        inside = m >= 0
        vr = np.where(inside, xr[..., np.maximum(m, 0)], cre).astype(R)
        vi = np.where(inside, xi[..., np.maximum(m, 0)], cim).astype(R)
        pr = fma(vr, wr, -(vi * wi))
        pi = fma(vi, wr, vr * wi)
        sr = (sr + pr).astype(R)
        si = (si + pi).astype(R)
    cdt = np.empty(0, out.dtype).real.dtype
    res = np.empty(xs.shape, out.dtype)
    res.real = sr.astype(cdt)
    res.imag = si.astype(cdt)
    out[...] = np.moveaxis(res, -1, axis)
    return out


def correlate1d(input, weights, axis=-1, output=None, mode="reflect", cval=0.0,
                origin=0, *, algorithm=None, convolve=False):
    """FLT:135-178 / FLT:180-221 -> FLT:271-344."""
    input = np.asarray(input)
    weights = np.asarray(weights)
    if input.dtype.kind == "c" or weights.dtype.kind == "c":
        axis = axis % input.ndim if input.ndim else 0
        if weights.dtype.kind == "c" and not convolve:
            weights = weights.conj()  # numpy.correlate conjugates the weights
        out = get_output(output, input, complex_output=True)
        return _complex_correlate1d(input, weights, axis, out, mode, cval, origin, algorithm,
                                    convolve)
    axis = axis % input.ndim if input.ndim else 0
    params = pass_params(input.dtype, input.ndim, axis, weights, mode, cval, origin,
                         convolve, algorithm)
    out = get_output(output, input)
    if out.dtype.kind in "iu" and mode == "constant" and params[-1] == "elementwise" \
            and not np.isfinite(cval):
        raise NotImplementedError(
            "Non-finite cval is not supported for outputs with integer dtype.")
    if out.flags.c_contiguous and not np.shares_memory(out, input):
        _run_pass(input, out, axis, *params[:-1])  # straight into the output
        return out
    res = np.empty(input.shape, out.dtype)
    _run_pass(input, res, axis, *params[:-1])
    out[...] = res
    return out


def convolve1d(input, weights, axis=-1, output=None, mode="reflect", cval=0.0,
               origin=0, *, algorithm=None):
    return correlate1d(input, weights, axis, output, mode, cval, origin,
                       algorithm=algorithm, convolve=True)


def run_1d_correlates(input, axes, weight_list, output, modes, cval, origins=0,
                      algorithm=None, convolve=False):
    """CORE:124-163 with FLT:363-396: passes in axis order, intermediates in
    the output dtype, ping-pong between output and one temporary."""
    input = np.asarray(input)
    output = get_output(output, input)
    axes = check_axes(axes, input.ndim)
    n = len(axes)
    modes = fix_sequence_arg(modes, n, "mode", check_mode)
    modes = ["grid-wrap" if m == "wrap" else m for m in modes]
    origins = fix_sequence_arg(origins, n, "origin", int)
    work = [(ax, w, m, o) for ax, w, m, o in zip(axes, weight_list, modes, origins) if w is not None]
    if not work:
        output[...] = input
        return output
    cur = input
    direct = output.flags.c_contiguous and not np.shares_memory(output, input)
    for i, (ax, w, m, o) in enumerate(work):
        last = i == len(work) - 1
        res = output if (last and direct) else np.empty(input.shape, output.dtype)
        correlate1d(cur, w, ax, res, m, cval, o, algorithm=algorithm, convolve=convolve)
        cur = res
    if cur is not output:
        output[...] = cur
    return output


# ------------------------------------------------------------- filter family

def gaussian_kernel1d(sigma, order, radius, dtype=np.float64):
    """FLT:689-717 (order 0 returns float64 regardless of `dtype`)."""
    if order < 0:
        raise ValueError("order must be non-negative")
    sigma2 = sigma * sigma
    x = np.arange(-radius, radius + 1)
    phi_x = np.exp(-0.5 / sigma2 * x**2)
    phi_x /= phi_x.sum()
    if order == 0:
        return phi_x
    exponent_range = np.arange(order + 1)
    q = np.zeros(order + 1)
    q[0] = 1
    D = np.diag(exponent_range[1:], 1)
    P = np.diag(np.ones(order) / -sigma2, -1)
    Q_deriv = D + P
    for _ in range(order):
        q = Q_deriv.dot(q)
    q = (x[:, None] ** exponent_range).dot(q)
    return np.ascontiguousarray((q * phi_x)[::-1], dtype=dtype)


def gaussian_filter(input, sigma, order=0, output=None, mode="reflect", cval=0.0,
                    truncate=4.0, radius=None, axes=None, *, algorithm=None):
    """FLT:580-686."""
    input = np.asarray(input)
    axes = check_axes(axes, input.ndim)
    n = len(axes)
    sigmas = fix_sequence_arg(sigma, n, "sigma", float)
    if n == 0 or all(s < 1e-15 for s in sigmas):
        out = get_output(output, input)
        out[...] = input
        return out
    orders = fix_sequence_arg(order, n, "order", int)
    modes = fix_sequence_arg(mode, n, "mode", str)
    radiuses = fix_sequence_arg(radius, n, "radius")
    truncate = float(truncate)
    wdt = np.promote_types(input.dtype, np.float32)
    params = [(axes[i], sigmas[i], orders[i], modes[i], radiuses[i])
              for i in range(n) if sigmas[i] > 1e-15]
    ws = []
    for _, s, o, _, r in params:
        if r is None:
            r = int(truncate * float(s) + 0.5)
        ws.append(None if r <= 0 else gaussian_kernel1d(s, o, r, dtype=wdt))
    return run_1d_correlates(input, [p[0] for p in params], ws, output,
                             [p[3] for p in params], cval, 0, algorithm)


def gaussian_filter1d(input, sigma, axis=-1, order=0, output=None, mode="reflect",
                      cval=0.0, truncate=4.0, *, algorithm=None):
    """FLT:524-577."""
    input = np.asarray(input)
    radius = int(float(truncate) * float(sigma) + 0.5)
    wdt = np.promote_types(input.dtype, np.float32)
    w = gaussian_kernel1d(sigma, int(order), radius, wdt)
    return correlate1d(input, w, axis, output, mode, cval, algorithm=algorithm)


def uniform_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0,
                     origin=0, *, algorithm=None):
    """FLT:399-444."""
    input = np.asarray(input)
    wdt = np.promote_types(input.dtype, np.float32)
    w = np.full(size, 1 / size, dtype=wdt)
    return correlate1d(input, w, axis, output, mode, cval, origin, algorithm=algorithm)


def uniform_filter(input, size=3, output=None, mode="reflect", cval=0.0, origin=0,
                   axes=None, *, algorithm=None):
    """FLT:447-521."""
    input = np.asarray(input)
    axes = check_axes(axes, input.ndim)
    n = len(axes)
    sizes = fix_sequence_arg(size, n, "size", int)
    origins = fix_sequence_arg(origin, n, "origin", int)
    modes = fix_sequence_arg(mode, n, "mode", str)
    wdt = np.promote_types(input.dtype, np.float32)
    ws = [None if s <= 1 else np.full(s, 1 / s, dtype=wdt) for s in sizes]
    return run_1d_correlates(input, axes, ws, output, modes, cval, origins, algorithm)


def _prewitt_or_sobel(input, axis, output, mode, cval, smooth, algorithm):
    """FLT:782-803."""
    input = np.asarray(input)
    axis = axis % input.ndim
    wdt = np.promote_types(input.dtype, np.float32)
    diff = np.array([-1, 0, 1], dtype=wdt)
    ws = [diff if a == axis else smooth for a in range(input.ndim)]
    return run_1d_correlates(input, tuple(range(input.ndim)), ws, output,
                             (mode,) * input.ndim, cval, 0, algorithm)


def sobel(input, axis=-1, output=None, mode="reflect", cval=0.0, *, algorithm=None):
    """FLT:751-779."""
    input = np.asarray(input)
    wdt = np.promote_types(input.dtype, np.float32)
    return _prewitt_or_sobel(input, axis, output, mode, cval,
                             np.array([1, 2, 1], dtype=wdt), algorithm)


def prewitt(input, axis=-1, output=None, mode="reflect", cval=0.0, *, algorithm=None):
    """FLT:720-748."""
    input = np.asarray(input)
    wdt = np.promote_types(input.dtype, np.float32)
    return _prewitt_or_sobel(input, axis, output, mode, cval,
                             np.ones(3, dtype=wdt), algorithm)


def gaussian_gradient_magnitude(input, sigma, output=None, mode="reflect", cval=0.0,
                                *, axes=None, algorithm=None, **kwargs):
    """FLT:1100-1157 over generic_gradient_magnitude FLT:1012-1097 (float outputs)."""
    input = np.asarray(input)
    ndim = input.ndim
    axes = check_axes(axes, ndim)
    modes = fix_sequence_arg(mode, len(axes), "mode", check_mode)
    output = get_output(output, input)
    if output.dtype.kind != "f":
        raise NotImplementedError("integer output")

    def deriv(ax, m):
        order = [0] * ndim
        order[ax] = 1
        return gaussian_filter(input, sigma, order, output.dtype, m, cval,
                               algorithm=algorithm, **kwargs)

    acc = deriv(axes[0], modes[0])
    acc = acc * acc
    for i in range(1, len(axes)):
        t = deriv(axes[i], modes[i])
        acc = acc + t * t
    output[...] = np.sqrt(acc)
    return output


# ---------------------------------------------------------- skimage layer

def sk_gaussian(image, sigma=1, mode="nearest", cval=0, preserve_range=False,
                truncate=4.0, *, channel_axis=None, out=None):
    """_shared/filters.py:21-166."""
    image = np.asarray(image)
    if not np.iterable(sigma):
        if sigma < 0:
            raise ValueError("Sigma values less than zero are not valid")
    elif any(s < 0 for s in sigma):
        raise ValueError("Sigma values less than zero are not valid")
    if channel_axis is not None:
        axes = tuple(a for a in range(image.ndim) if a != channel_axis % image.ndim)
    else:
        axes = tuple(range(image.ndim))
    image = convert_to_float(image, preserve_range)
    image = image.astype(supported_float_type(image.dtype), copy=False)
    res = gaussian_filter(image, sigma, output=image.dtype, mode=mode, cval=cval,
                          truncate=truncate, axes=axes)
    if out is not None:
        out[...] = res
        return out
    return res


def _min_or_max_1d(input, size, axis, output, mode, cval, origin, is_max):
    """FLT:1412-1497 (min/max kernel without weights) in the C oracle."""
    input = np.ascontiguousarray(np.asarray(input))
    size = int(size)
    if size < 1:
        raise RuntimeError("incorrect filter size")
    axis = axis % input.ndim
    origin = check_origin(origin, size)
    mode = "grid-wrap" if mode == "wrap" else mode
    check_mode(mode)
    out = get_output(output, input)
    res = np.empty(input.shape, out.dtype)
    shape = input.shape
    outer = int(np.prod(shape[:axis], dtype=np.int64))
    inner = int(np.prod(shape[axis + 1:], dtype=np.int64))
    _lib.oracle_min_max1d(input.ctypes.data, ord(input.dtype.char), res.ctypes.data,
                          ord(res.dtype.char), outer, shape[axis], inner, size,
                          size // 2 + origin, MODES[mode], float(cval), int(is_max))
    out[...] = res
    return out


def minimum_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0, origin=0):
    """FLT:1362-1385."""
    return _min_or_max_1d(input, size, axis, output, mode, cval, origin, False)


def maximum_filter1d(input, size, axis=-1, output=None, mode="reflect", cval=0.0, origin=0):
    """FLT:1388-1411."""
    return _min_or_max_1d(input, size, axis, output, mode, cval, origin, True)


def generic_gradient_magnitude(input, derivative, output=None, mode="reflect", cval=0.0,
                               extra_arguments=(), extra_keywords=None, *, axes=None):
    """FLT:1012-1097: output = d0, output *= output, then tmp = d_i,
    tmp *= tmp, output += tmp for the other axes, sqrt in place (numpy
    operations in the output dtype)."""
    input = np.asarray(input)
    if extra_keywords is None:
        extra_keywords = {}
    axes = check_axes(axes, input.ndim)
    modes = fix_sequence_arg(mode, len(axes), "mode", check_mode)
    out = get_output(output, input)
    out[...] = derivative(input, axes[0], out, modes[0], cval, *extra_arguments,
                          **extra_keywords)
    np.multiply(out, out, out=out)
    if len(axes) > 1:
        tmp = np.empty_like(out)
        for i in range(1, len(axes)):
            tmp[...] = derivative(input, axes[i], tmp, modes[i], cval, *extra_arguments,
                                  **extra_keywords)
            np.multiply(tmp, tmp, out=tmp)
            np.add(out, tmp, out=out)
    np.sqrt(out, out=out)
    return out


def generic_laplace(input, derivative2, output=None, mode="reflect", cval=0.0,
                    extra_arguments=(), extra_keywords=None, *, axes=None):
    """FLT:806-890: derivative2 along the first axis into the output, every
    further axis into a temporary of the output dtype added in place (numpy
    add in that dtype: integers wrap, floats round to nearest)."""
    input = np.asarray(input)
    if extra_keywords is None:
        extra_keywords = {}
    axes = check_axes(axes, input.ndim)
    out = get_output(output, input)
    if len(axes) == 0:
        out[...] = input
        return out
    modes = fix_sequence_arg(mode, len(axes), "mode", check_mode)
    out[...] = derivative2(input, axes[0], out, modes[0], cval, *extra_arguments,
                           **extra_keywords)
    if len(axes) > 1:
        tmp = np.empty_like(out)
        for i in range(1, len(axes)):
            tmp[...] = derivative2(input, axes[i], tmp, modes[i], cval, *extra_arguments,
                                   **extra_keywords)
            np.add(out, tmp, out=out)
    return out


def laplace(input, output=None, mode="reflect", cval=0.0, *, axes=None, algorithm=None):
    """FLT:893-930: correlate1d with [1, -2, 1] per axis, summed."""
    input = np.asarray(input)
    w = np.array([1, -2, 1], dtype=np.promote_types(input.dtype, np.float32))

    def derivative2(inp, axis, out, m, c):
        return correlate1d(inp, w, axis, out, m, c, algorithm=algorithm)

    return generic_laplace(input, derivative2, output, mode, cval, axes=axes)


def gaussian_laplace(input, sigma, output=None, mode="reflect", cval=0.0, *, axes=None,
                     algorithm=None, **kwargs):
    """FLT:933-1009: per axis a gaussian_filter with order 2 on that axis
    (sigma 0 on the axes not filtered), summed."""
    input = np.asarray(input)
    axes = check_axes(axes, input.ndim)
    n = len(axes)
    sigma = fix_sequence_arg(sigma, n, "sigma", float)
    if n < input.ndim:
        full = [0] * input.ndim
        for s_, ax in zip(sigma, axes):
            full[ax] = s_
        sigma = full

    def derivative2(inp, axis, out, m, c, sig, **kw):
        order = [0] * inp.ndim
        order[axis] = 2
        return gaussian_filter(inp, sig, order, out, m, c, algorithm=algorithm, **kw)

    return generic_laplace(input, derivative2, output, mode, cval, extra_arguments=(sigma,),
                           extra_keywords=kwargs, axes=axes)


def difference_of_gaussians(image, low_sigma, high_sigma=None, *, mode="nearest", cval=0,
                            channel_axis=None, truncate=4.0):
    """filters/_gaussian.py:13-174."""
    image = img_as_float(image)
    spatial_dims = image.ndim - 1 if channel_axis is not None else image.ndim
    if np.isscalar(low_sigma):
        low_sigma = (low_sigma,) * spatial_dims
    low_sigma = tuple(map(float, low_sigma))
    if high_sigma is None:
        high_sigma = tuple(low * 1.6 for low in low_sigma)
    elif np.isscalar(high_sigma):
        high_sigma = (high_sigma,) * spatial_dims
    high_sigma = tuple(map(float, high_sigma))
    out = sk_gaussian(image, sigma=low_sigma, mode=mode, cval=cval, channel_axis=channel_axis,
                      truncate=truncate)
    out -= sk_gaussian(image, sigma=high_sigma, mode=mode, cval=cval,
                       channel_axis=channel_axis, truncate=truncate)
    return out


def unsharp_mask(image, radius=1.0, amount=1.0, preserve_range=False, *, channel_axis=None):
    """filters/_unsharp_mask.py:12-160."""
    image = np.asarray(image)
    float_dtype = supported_float_type(image.dtype)
    vrange = None
    if preserve_range:
        fimg = image.astype(float_dtype, copy=False)
    else:
        fimg = img_as_float(image).astype(float_dtype, copy=False)
        vrange = [-1.0, 1.0] if np.any(fimg < 0) else [0.0, 1.0]

    def single(img):
        img = np.ascontiguousarray(img)
        blurred = sk_gaussian(img, sigma=radius, mode="reflect")
        amt = img.dtype.type(amount)
        result = img + (img - blurred) * amt
        if vrange is not None:
            lo, hi = img.dtype.type(vrange[0]), img.dtype.type(vrange[1])
            result = np.where(result < lo, lo, np.where(result > hi, hi, result))
        return result.astype(img.dtype, copy=False)

    if channel_axis is not None:
        result = np.empty_like(fimg, dtype=float_dtype)
        ax = channel_axis % fimg.ndim
        for c in range(image.shape[ax]):
            sl = tuple(c if d == ax else slice(None) for d in range(fimg.ndim))
            result[sl] = single(fimg[sl])
        return result
    return single(fimg)


_SOBEL_SMOOTH = np.array([1, 2, 1]) / 4
_PREWITT_SMOOTH = np.full((3,), 1 / 3)
_SCHARR_SMOOTH = np.array([3, 10, 3]) / 16
_FARID_SMOOTH = np.array([0.0376593171958126, 0.249153396177344, 0.426374573253687,
                          0.249153396177344, 0.0376593171958126])
_FARID_EDGE = np.array([0.109603762960254, 0.276690988455557, 0, -0.276690988455557,
                        -0.109603762960254])


def generic_edge_filter(image, *, smooth_weights, edge_weights=(1, 0, -1), axis=None,
                        mode="reflect"):
    """filters/edges.py:148-241 (cval is accepted there but never forwarded)."""
    image = np.asarray(image)
    ndim = image.ndim
    if axis is None:
        axes = list(range(ndim))
    elif np.isscalar(axis):
        axes = [axis]
    else:
        axes = list(axis)
    mag = len(axes) > 1
    if image.dtype.kind == "f":
        fdt = supported_float_type(image.dtype)
        image = image.astype(fdt, copy=False)
    else:
        image = img_as_float(image)
        fdt = image.dtype
    ew = np.asarray(edge_weights, dtype=fdt)
    sw = np.asarray(smooth_weights, dtype=fdt)
    if mag:
        ew = (ew / fdt.type(math.sqrt(ndim))).astype(fdt)
    output = None
    for i, ed in enumerate(axes):
        ax_out = convolve1d(image, ew, axis=ed, mode=mode, output=fdt)
        for sd in sorted(set(range(ndim)) - {ed % ndim}):
            ax_out = convolve1d(ax_out, sw, axis=sd, mode=mode, output=fdt)
        if mag:
            ax_out = (ax_out * ax_out).astype(fdt)
        output = ax_out if i == 0 else (output + ax_out).astype(fdt)
    if mag:
        output = np.sqrt(output).astype(fdt)
    return output


def mask_filter_result(result, mask):
    """filters/edges.py:75-85: binary erosion of the mask with the
    full-connectivity footprint and border value 0 (scipy.ndimage's
    binary_erosion, the same definition), then result *= mask."""
    if mask is None:
        return result
    import scipy.ndimage as sndi

    mask = np.asarray(mask)
    eroded = sndi.binary_erosion(mask, np.ones((3,) * mask.ndim, bool), border_value=0)
    return (result * eroded).astype(result.dtype)


def sk_sobel(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    return mask_filter_result(
        generic_edge_filter(image, smooth_weights=_SOBEL_SMOOTH, axis=axis, mode=mode), mask)


def sk_prewitt(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    return mask_filter_result(
        generic_edge_filter(image, smooth_weights=_PREWITT_SMOOTH, axis=axis, mode=mode), mask)


def sk_scharr(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """filters/edges.py:362-422."""
    return mask_filter_result(
        generic_edge_filter(image, smooth_weights=_SCHARR_SMOOTH, axis=axis, mode=mode), mask)


def sk_farid(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """filters/edges.py:783-850."""
    return mask_filter_result(
        generic_edge_filter(image, smooth_weights=_FARID_SMOOTH, edge_weights=_FARID_EDGE,
                            axis=axis, mode=mode), mask)


def hessian_matrix_gaussian(image, sigma=1, mode="reflect", cval=0, order="rc"):
    """feature/corner.py:161-254 (use_gaussian_derivatives=True)."""
    image = img_as_float(np.asarray(image))
    image = image.astype(supported_float_type(image.dtype), copy=False)
    ndim = image.ndim
    if np.isscalar(sigma):
        sigma = (sigma,) * ndim
    truncate = 8 if all(s > 1 for s in sigma) else 100
    sq1_2 = 1 / math.sqrt(2)
    ss = tuple(sq1_2 * s for s in sigma)
    orders = [tuple([0] * d + [1] + [0] * (ndim - d - 1)) for d in range(ndim)]
    grads = [gaussian_filter(image, ss, order=orders[d], mode=mode, cval=cval,
                             truncate=truncate) for d in range(ndim)]
    axes = list(range(ndim))
    if order == "xy":
        axes = axes[::-1]
    return [gaussian_filter(grads[a0], ss, order=orders[a1], mode=mode, cval=cval,
                            truncate=truncate)
            for a0, a1 in combinations_with_replacement(axes, 2)]


def gradient(f, axis=None):
    """numpy/cupy gradient with unit spacing and edge_order=1."""
    f = np.asarray(f)
    axes = range(f.ndim) if axis is None else [axis]
    outs = []
    for ax in axes:
        out = np.empty_like(f)
        sl = [slice(None)] * f.ndim

        def S(s):
            sl2 = list(sl)
            sl2[ax] = s
            return tuple(sl2)

        out[S(slice(1, -1))] = (f[S(slice(2, None))] - f[S(slice(None, -2))]) / f.dtype.type(2.0)
        out[S(0)] = f[S(1)] - f[S(0)]
        out[S(-1)] = f[S(-1)] - f[S(-2)]
        outs.append(out)
    return outs if axis is None else outs[0]


def hessian_matrix_fd(image, sigma=1, mode="constant", cval=0, order="rc"):
    """feature/corner.py:355-384 (use_gaussian_derivatives=False)."""
    image = img_as_float(np.asarray(image))
    image = image.astype(supported_float_type(image.dtype), copy=False)
    ch = -1 if (image.ndim == 3 and image.shape[-1] == 3) else None
    g = sk_gaussian(image, sigma=sigma, mode=mode, cval=cval, channel_axis=ch)
    grads = gradient(g)
    axes = list(range(image.ndim))
    if order == "xy":
        axes = axes[::-1]
    return [gradient(grads[a0], axis=a1) for a0, a1 in combinations_with_replacement(axes, 2)]


def eigvals_sym(elems, sort="descending", abs_sort=False):
    """feature/corner.py:699-755 with the closed forms of :473-527 and :566-647,
    evaluated in float64 (the 3x3 kernel's own precision) and rounded to F."""
    F = elems[0].dtype
    e = [np.asarray(x, dtype=np.float64) for x in elems]
    if len(e) == 3:
        m00, m01, m11 = e
        # the 2x2 kernel keeps its temporaries in F; evaluated on the GPU with
        # every operation rounded on its own (checked on 2 M matrices against
        # the fused alternatives, which differ on 5 % of them)
        t1 = (m01 * m01).astype(F) * F.type(4)
        t2 = (m00 - m11).astype(F)
        t2 = (t2 * t2 + t1).astype(F)
        t2 = (np.sqrt(t2) / F.type(2)).astype(F)
        t1 = ((m00 + m11).astype(F) / F.type(2)).astype(F)
        lo, hi = (t1 - t2).astype(F), (t1 + t2).astype(F)
        l1, l2 = (lo, hi) if sort == "ascending" else (hi, lo)
        if abs_sort:
            sw = (np.abs(l1) > np.abs(l2)) if sort == "ascending" else (np.abs(l1) < np.abs(l2))
            l1, l2 = np.where(sw, l2, l1), np.where(sw, l1, l2)
        return np.stack([l1, l2])
    else:
        a, d, f, b, ee, c = e
        d_sq, e_sq, f_sq = d * d, ee * ee, f * f
        ta, tb, tc = 2 * a - b - c, 2 * b - a - c, 2 * c - a - b
        x2 = -ta * tb * tc + 9 * (tc * d_sq + tb * f_sq + ta * e_sq) - 54 * (d * ee * f)
        x1 = a * a + b * b + c * c - a * b - a * c - b * c + 3 * (d_sq + e_sq + f_sq)
        x1 = np.maximum(x1, 0.0)
        arg = np.maximum(4 * x1 ** 3 - x2 ** 2, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            phi = np.arctan(np.sqrt(arg) / x2)
        phi = np.where(x2 < 0, phi + np.pi, phi)
        phi = np.where(x2 == 0.0, np.pi / 2.0, phi)
        x1t = (2.0 / 3.0) * np.sqrt(x1)
        abc = (a + b + c) / 3.0
        lam = [(abc - x1t * np.cos(phi / 3.0)).astype(F),
               (abc + x1t * np.cos((phi - np.pi) / 3.0)).astype(F),
               (abc + x1t * np.cos((phi + np.pi) / 3.0)).astype(F)]
        # The three compare-and-swap steps of corner.py:607-629. With
        # abs_sort the magnitudes are taken once, before any swap, and the
        # comparisons keep using those original magnitudes.
        keys = [np.abs(v) for v in lam] if abs_sort else None
        order = (0, 1, 2) if sort == "ascending" else (2, 1, 0)
        v1, v2, v3 = order

        def step(i, j):
            ki = keys[i] if abs_sort else lam[i]
            kj = keys[j] if abs_sort else lam[j]
            sw = ki > kj
            lam[i], lam[j] = np.where(sw, lam[j], lam[i]), np.where(sw, lam[i], lam[j])

        step(v1, v2)
        step(v1, v3)
        step(v2, v3)
        return np.stack(lam)


def _by_chunks(fn, arrays):
    """fn(*chunks) over chunks of the inputs' leading axis, in THREADS threads
    (numpy releases the GIL in its loops). fn must be elementwise; its
    results may carry extra leading axes (a stack of eigenvalue images), so
    the chunks are joined along the axis that was the inputs' leading one.
    The result equals fn(*arrays)."""
    n = arrays[0].shape[0]
    nchunk = max(1, min(THREADS, n))
    if nchunk == 1:
        return fn(*arrays)
    from concurrent.futures import ThreadPoolExecutor

    bounds = [(i * n // nchunk, (i + 1) * n // nchunk) for i in range(nchunk)]
    with ThreadPoolExecutor(nchunk) as ex:
        parts = list(ex.map(lambda b: fn(*[a[b[0]:b[1]] for a in arrays]), bounds))
    nd = arrays[0].ndim
    return np.concatenate(parts, axis=parts[0].ndim - nd)


def _frangi_core(ev, alpha_sq, beta_sq, gamma_sq, want_v):
    """r_g and (optionally) the vesselness of one scale from the stacked
    eigenvalues (C core: cuCIM's kernel expressions with the compiler's
    contraction, libm exp)."""
    ev = np.ascontiguousarray(ev)
    F = ev.dtype
    nd = ev.shape[0]
    rg = np.empty(ev.shape[1:], F)
    v = np.empty(ev.shape[1:], F) if want_v else None
    _lib.oracle_frangi_scale(ev[0].ctypes.data, ev[1].ctypes.data, ev[nd - 1].ctypes.data, nd,
                             rg.size, int(F == np.float64), alpha_sq, beta_sq, gamma_sq,
                             rg.ctypes.data, v.ctypes.data if want_v else None)
    return rg, v


def frangi(image, sigmas=range(1, 10, 2), alpha=0.5, beta=0.5, gamma=None,
           black_ridges=True, mode="reflect", cval=0):
    """filters/ridges.py:322-476 with the kernels of :228-319. The eigenvalue
    and vesselness steps are elementwise and run over chunks of the leading
    axis in THREADS threads."""
    image = np.asarray(image)
    image = image.astype(supported_float_type(image.dtype), copy=False)
    if not black_ridges:
        image = -image
    F = image.dtype
    alpha_sq, beta_sq = 2 * alpha * alpha, 2 * beta * beta
    gamma_sq = None if gamma is None else 2 * gamma * gamma
    fmax = None
    for sigma in sigmas:
        H = hessian_matrix_gaussian(image, sigma, mode=mode, cval=cval)
        ev = _by_chunks(lambda *h: eigvals_sym(list(h), sort="ascending", abs_sort=True), H)
        del H
        if gamma_sq is None:
            rg = _by_chunks(lambda *e: _frangi_core(np.stack(e), 1.0, 1.0, 1.0, False)[0],
                            list(ev))
            s_max = float(rg.max())
            g = math.sqrt(s_max) / 2.0
            gamma_sq = 2.0 if s_max == 0 else max(2 * g * g, 1e-10)
        v = _by_chunks(lambda *e: _frangi_core(np.stack(e), alpha_sq, beta_sq, gamma_sq,
                                               True)[1], list(ev))
        fmax = v.copy() if fmax is None else np.maximum(fmax, v)
    return fmax


def fma(a, b, c):
    """Elementwise fused multiply-add in the arrays' float type (C core)."""
    a, b, c = np.broadcast_arrays(*[np.asarray(v) for v in (a, b, c)])
    F = np.result_type(a, b, c)
    a, b, c = (np.ascontiguousarray(v, dtype=F) for v in (a, b, c))
    out = np.empty(a.shape, F)
    _lib.oracle_fma(a.ctypes.data, b.ctypes.data, c.ctypes.data, a.size,
                    int(F == np.float64), out.ctypes.data)
    return out


def _ridge_image(image, black_ridges):
    image = np.asarray(image)
    image = image.astype(supported_float_type(image.dtype), copy=False)
    return -image if not black_ridges else image


def _ridge_eigvals(image, sigma, mode, cval):
    """hessian_matrix_eigvals of the Gaussian-derivative Hessian (descending),
    entries below 1e-12 in magnitude zeroed (ridges.py:112-116)."""
    F = image.dtype
    H = hessian_matrix_gaussian(image, sigma, mode=mode, cval=cval)
    ev = _by_chunks(lambda *h: eigvals_sym(list(h), sort="descending"), H)
    return np.where(np.abs(ev) < F.type(1e-12), F.type(0), ev).astype(F)


def meijering(image, sigmas=range(1, 10, 2), alpha=None, black_ridges=True, mode="reflect",
              cval=0):
    """filters/ridges.py:50-146. The circulant mixing (cupy.tensordot, a
    float GEMM over ndim products) is an ascending multiply-add chain."""
    image = _ridge_image(image, black_ridges)
    F = image.dtype
    if alpha is None:
        alpha = 1 / (image.ndim + 1)
    a = F.type(alpha)
    out = np.zeros_like(image)
    for sigma in sigmas:
        ev = _ridge_eigvals(image, sigma, mode, cval)
        nd = ev.shape[0]
        vals = []
        for r in range(nd):
            v = ((F.type(1) if r == 0 else a) * ev[0]).astype(F)
            for k in range(1, nd):
                v = fma(np.full(v.shape, F.type(1) if r == k else a, F), ev[k], v)
            vals.append(v)
        vals = np.stack(vals)
        v = np.take_along_axis(vals, np.abs(vals).argmax(0)[None], 0)[0]
        v = np.maximum(v, F.type(0))
        mx = v.max()
        if mx > 0:
            v = (v / mx).astype(F)
        out = np.maximum(out, v)
    return out


def sato(image, sigmas=range(1, 10, 2), black_ridges=True, mode="reflect", cval=0):
    """filters/ridges.py:148-225."""
    image = _ridge_image(image, black_ridges)
    if image.ndim not in (2, 3):
        raise ValueError("sato is defined for 2-D and 3-D images")
    F = image.dtype
    out = np.zeros_like(image)
    for sigma in sigmas:
        ev = _ridge_eigvals(image, sigma, mode, cval)[:-1]
        vals = np.prod(np.maximum(ev, F.type(0)), 0).astype(F) ** F.type(1 / len(ev))
        vals = (vals * F.type(sigma ** 2)).astype(F)
        out = np.maximum(out, vals)
    return out


def hessian_ridge(image, sigmas=range(1, 10, 2), alpha=0.5, beta=0.5, gamma=15,
                  black_ridges=True, mode="reflect", cval=0):
    """filters/ridges.py:479-595: frangi, then outputs <= 0 set to 1."""
    out = frangi(image, sigmas=sigmas, alpha=alpha, beta=beta, gamma=gamma,
                 black_ridges=black_ridges, mode=mode, cval=cval)
    out[out <= 0] = 1
    return out


def structure_tensor(image, sigma=1, mode="constant", cval=0, order="rc"):
    """feature/corner.py:48-158 (with feature/util.py:19-24 for the input)."""
    image = np.squeeze(np.asarray(image))
    image = img_as_float(image)
    image = image.astype(supported_float_type(image.dtype), copy=False)
    F = image.dtype
    ders = [sobel(image, i, mode=mode, cval=cval) for i in range(image.ndim)]
    if order == "xy":
        ders = ders[::-1]
    channel_axis = -1 if (image.ndim == 3 and image.shape[-1] == 3) else None
    return [sk_gaussian((d0 * d1).astype(F), sigma=sigma, mode=mode, cval=cval,
                        channel_axis=channel_axis)
            for d0, d1 in combinations_with_replacement(ders, 2)]


def corner_kitchen_rosenfeld(image, mode="constant", cval=0):
    """feature/corner.py:940-1004 (no contraction: compared with a tolerance)."""
    image = np.asarray(image)
    image = image.astype(supported_float_type(image.dtype), copy=False)
    imy, imx = (sobel(image, i, mode=mode, cval=cval) for i in range(2))
    imxy, imxx = (sobel(imx, i, mode=mode, cval=cval) for i in range(2))
    imyy = sobel(imy, 0, mode=mode, cval=cval)
    F = image.dtype
    den = (imx * imx + imy * imy).astype(F)
    num = imxx * (imy * imy) + imyy * (imx * imx) - 2 * imxy * imx * imy
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den == 0, 0, num / np.where(den == 0, 1, den))
    return r.astype(F)


def corner_harris(image, method="k", k=0.05, eps=1e-6, sigma=1):
    """feature/corner.py:1007-1113."""
    Arr, Arc, Acc = structure_tensor(image, sigma)
    F = Arr.dtype
    det = (Arr * Acc - Arc * Arc).astype(F)
    tr = (Arr + Acc).astype(F)
    if method == "k":
        r = det.astype(np.float64) - k * tr.astype(np.float64) * tr
    else:
        r = 2 * det.astype(np.float64) / (tr.astype(np.float64) + eps)
    return r.astype(F)


def corner_shi_tomasi(image, sigma=1):
    """feature/corner.py:1116-1189."""
    Arr, Arc, Acc = structure_tensor(image, sigma)
    F = Arr.dtype
    tmp = ((Arr - Acc) * (Arr - Acc)).astype(F)
    return ((Arr + Acc - np.sqrt(tmp + 4 * Arc * Arc)) / 2.0).astype(F)


def corner_foerstner(image, sigma=1):
    """feature/corner.py:1192-1284."""
    Arr, Arc, Acc = structure_tensor(image, sigma)
    F = Arr.dtype
    det = (Arr * Acc - Arc * Arc).astype(F)
    tr = (Arr + Acc).astype(F)
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(tr == 0, 0, det / tr).astype(F)
        q = np.where(tr == 0, 0, 4 * det / (tr * tr)).astype(F)
    return w, q


def rgb2gray(rgb, channel_axis=-1):
    """color/colorconv.py:1049-1095 (+ _prepare_colorarray :160-183)."""
    rgb = np.moveaxis(np.asarray(rgb), channel_axis, -1)
    if rgb.shape[-1] != 3:
        raise ValueError("the input array must have size 3 along `channel_axis`")
    fdt = supported_float_type(rgb.dtype)
    x = img_as_float(rgb).astype(fdt)
    x = np.ascontiguousarray(x).astype(np.float64)
    g = np.empty(x.shape[:-1], np.float64)
    # the kernel's expression with the CUDA compiler's contraction (C core)
    _lib.oracle_rgb2gray(x.ctypes.data, g.size, g.ctypes.data)
    return g.astype(fdt)


def cast_w(values_w, w64, out_dtype):
    """cast<D>() of a W-typed array alone (CORE:227-244)."""
    src = np.ascontiguousarray(values_w, dtype=np.float64 if w64 else np.float32)
    out = np.empty(src.shape, dtype=out_dtype)
    _lib.oracle_cast(src.ctypes.data, int(w64), out.ctypes.data, ord(out.dtype.char), src.size)
    return out
