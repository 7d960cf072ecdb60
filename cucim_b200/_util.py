"""Argument checks and dtype rules of cuCIM's vendored ndimage, restated.

Paths are relative to python/cucim/src/cucim/skimage in rapidsai/cucim:
UTIL = _vendored/_ndimage_util.py, FLT = _vendored/_ndimage_filters.py,
SEP = filters/_separable_filtering.py.
"""

import math
import operator
from collections.abc import Iterable

import numpy as np

from . import _lib

try:
    from numpy.exceptions import AxisError
except ImportError:  # pragma: no cover
    from numpy import AxisError

_VALID_MODES = (
    "reflect", "constant", "nearest", "mirror", "wrap", "grid-mirror", "grid-wrap",
    "grid-reflect",
)

# per-block shared memory of every CUDA device (bytes); SEP:130-152 compares
# the shared-memory kernel's tile against it
SHARED_BLOCK_BYTES = 49152

_NEW_FLOAT = {
    "f": np.float32, "d": np.float64, "e": np.float32, "b": np.float32,
    "B": np.float32, "h": np.float32, "H": np.float32, "?": np.float32,
}


def supported_float_type(input_dtype, allow_complex=False):
    """_shared/utils.py:1151-1179."""
    if isinstance(input_dtype, Iterable) and not isinstance(input_dtype, str):
        return np.result_type(*(supported_float_type(d) for d in input_dtype))
    dt = np.dtype(input_dtype)
    if not allow_complex and dt.kind == "c":
        raise ValueError("complex valued input is not supported")
    return np.dtype(_NEW_FLOAT.get(dt.char, np.float64))


def weights_dtype(input_dtype, w_dtype):
    """UTIL:35-46 with use_cucim_casting=True: complex64 / complex128 when the
    input or the weights are complex."""
    w_dtype = np.dtype(w_dtype)
    in_dtype = np.dtype(input_dtype)
    if w_dtype.kind == "c" or in_dtype.kind == "c":
        real = in_dtype if in_dtype.kind != "c" else np.empty(0, in_dtype).real.dtype
        return np.promote_types(real, np.complex64)
    if w_dtype.kind in "iub":
        return supported_float_type(w_dtype)
    return np.promote_types(in_dtype, np.float32)


def check_mode(mode):
    """UTIL:95-108. 'grid-reflect' passes cuCIM's name check but has no
    boundary code (UTIL:186-308); it is rejected here up front."""
    if mode not in _VALID_MODES or mode == "grid-reflect":
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
        axes = (operator.index(axes),)
    elif isinstance(axes, Iterable):
        axes = tuple(operator.index(ax) for ax in axes)
        for ax in axes:
            if ax < -ndim or ax > ndim - 1:
                raise AxisError(f"specified axis: {ax} is out of range")
        axes = tuple(ax % ndim if ax < 0 else ax for ax in axes)
    else:
        raise ValueError("axes must be an integer, iterable of integers, or None")
    if len(set(axes)) != len(axes):
        raise ValueError("axes must be unique")
    return axes


def normalize_axis(axis, ndim):
    if axis < -ndim or axis >= ndim:
        raise AxisError(f"axis {axis} is out of bounds for array of dimension {ndim}")
    return axis % ndim


def _smem_bytes(ndim, axis, K, anchor, itemsize):
    """Shared-memory tile of cuCIM's shared-memory kernel (SEP:17-88)."""
    hpn = max(K - anchor, anchor)
    if ndim == 2:
        bx, by, bz = (16, 16, 1) if axis == 1 else (32, 8, 1)
        halo = math.ceil(hpn / (bx if axis == 1 else by))
    elif axis == 2:
        bx, by, bz = 16, 4, 4
        halo = math.ceil(hpn / bx)
    else:
        bx, by, bz = 32, 4, 4
        halo = math.ceil(hpn / (by if axis == 1 else bz))
    ppb = max(4, halo)
    return (ppb + 2 * halo) * bx * by * bz * itemsize


def choose_algorithm(ndim, axis, K, anchor, mode, cval, in_dtype, algorithm=None):
    """Which of cuCIM's two kernels a correlate1d call runs (FLT:271-344).

    The answer decides two details of the arithmetic: how a constant-mode
    fill value is rounded and whether zero taps are skipped.
    """
    in_dtype = np.dtype(in_dtype)
    if algorithm is None:
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
        if mode == "constant" and not np.isfinite(cval):
            return "elementwise"
        if K > 32 and _smem_bytes(ndim, axis, K, anchor, in_dtype.itemsize) > SHARED_BLOCK_BYTES:
            return "elementwise"
    return algorithm


def pass_flags(in_dtype, ndim, axis, K, origin, mode, cval, w_dtype, convolve, algorithm):
    """CIMX_F_* flags for one pass (memoised: a pure function of its
    arguments, called once per pass of every filter call)."""
    try:
        key = (np.dtype(in_dtype).str, ndim, axis, K, origin, mode, float(cval),
               np.dtype(w_dtype).str, bool(convolve), algorithm)
    except (TypeError, ValueError):
        return _pass_flags(in_dtype, ndim, axis, K, origin, mode, cval, w_dtype, convolve,
                           algorithm)
    flags = _PASS_FLAGS.get(key)
    if flags is None:
        flags = _pass_flags(in_dtype, ndim, axis, K, origin, mode, cval, w_dtype, convolve,
                            algorithm)
        if len(_PASS_FLAGS) < 4096:
            _PASS_FLAGS[key] = flags
    return flags


_PASS_FLAGS = {}


def _pass_flags(in_dtype, ndim, axis, K, origin, mode, cval, w_dtype, convolve, algorithm):
    wdt = weights_dtype(in_dtype, w_dtype)
    o = origin
    if convolve:
        o = -o
        if K % 2 == 0:
            o -= 1
    anchor = K // 2 + o
    alg = choose_algorithm(ndim, axis, K, anchor, mode, cval, in_dtype, algorithm)
    flags = 0
    if wdt in (np.float64, np.complex128):
        flags |= _lib.F_W64
    if np.dtype(w_dtype).kind == "c":
        flags |= _lib.F_COMPLEX_TAPS
    if convolve:
        flags |= _lib.F_CONVOLVE
    if alg == "shared_memory":
        flags |= _lib.F_CVAL_AS_INPUT
    else:
        flags |= _lib.F_SKIP_ZERO_TAPS
    return flags
