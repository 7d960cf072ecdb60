"""dtype conversions of cucim.skimage.util (python/cucim/src/cucim/skimage/
util/dtype.py) and _shared/utils.py used on the filtering path."""

import ctypes

import numpy as np

from .. import _arrays, _lib
from .._util import supported_float_type

__all__ = ["img_as_float", "img_as_float32", "img_as_float64", "convert_to_float",
           "supported_float_type"]


def _convert(image, out_dtype, op, force_copy=False):
    x = _arrays.as_tensor(image)
    in_dt = _arrays.np_dtype(x)
    out_dtype = np.dtype(out_dtype)
    if in_dt == out_dtype and op != 2:
        return _arrays.wrap_like(image, x.clone()) if force_copy else image
    if op == 1 and in_dt.kind == "f":
        op = 0  # float -> float is a plain astype (util/dtype.py:301-304)
    if in_dt.kind == "b":
        op = 0  # bool -> float: astype (util/dtype.py:292-297)
    xc = x.contiguous()
    out = _arrays.empty(xc.shape, out_dtype, xc.device)
    a_in, a_out = _arrays.to_cimx(xc), _arrays.to_cimx(out)
    rc = _lib.lib.cimx_convert(ctypes.byref(a_in), ctypes.byref(a_out), op,
                               _arrays.stream_of(xc))
    _lib.check(rc, "convert")
    return _arrays.wrap_like(image, out)


def img_as_float32(image, force_copy=False):
    """util/dtype.py:437-460."""
    return _convert(image, np.float32, 1, force_copy)


def img_as_float64(image, force_copy=False):
    """util/dtype.py:463-486."""
    return _convert(image, np.float64, 1, force_copy)


def img_as_float(image, force_copy=False):
    """util/dtype.py:489-512: float16/float32/<=16-bit integers -> float32,
    everything else -> float64."""
    x = _arrays.as_tensor(image)
    return _convert(image, supported_float_type(_arrays.np_dtype(x)), 1, force_copy)


def astype(image, dtype):
    """Plain dtype conversion on the device (ndarray.astype, copy=False)."""
    return _convert(image, dtype, 0)


def negative_astype(image, dtype):
    """-image.astype(dtype) in one pass."""
    return _convert(image, dtype, 2)


def convert_to_float(image, preserve_range):
    """_shared/utils.py:1019-1052."""
    x = _arrays.as_tensor(image)
    dt = _arrays.np_dtype(x)
    if dt == np.float16:
        return astype(image, np.float32)
    if preserve_range:
        if dt.char not in "df":
            image = astype(image, supported_float_type(dt))
        return image
    return img_as_float(image)
