"""rgb2gray of cucim.skimage.color (python/cucim/src/cucim/skimage/color/
colorconv.py:1038-1095)."""

import ctypes

import numpy as np

from .. import _arrays, _lib
from .._util import supported_float_type
from . import util as _u

__all__ = ["rgb2gray"]


def rgb2gray(rgb, *, channel_axis=-1):
    """Luminance Y = 0.2125 R + 0.7154 G + 0.0721 B (float64 arithmetic,
    stored in the image's float type). uint8 input is scaled by
    float32(1/255) first, in the same kernel."""
    x = _arrays.as_tensor(rgb)
    if not isinstance(channel_axis, int):
        raise TypeError("channel_axis must be an integer")
    if channel_axis < -x.dim() or channel_axis >= x.dim():
        raise np.exceptions.AxisError("channel_axis exceeds array dimensions")
    x = x.movedim(channel_axis, -1)
    if x.shape[-1] != 3:
        raise ValueError(
            f"the input array must have size 3 along `channel_axis`, got {tuple(x.shape)}")
    dt = _arrays.np_dtype(x)
    fdt = supported_float_type(dt)
    if not (dt == np.uint8 and fdt == np.float32) and dt != fdt:
        x = _arrays.as_tensor(_u.img_as_float32(x) if fdt == np.float32 else _u.img_as_float64(x))
    xc = x.contiguous()
    gray = _arrays.empty(xc.shape[:-1], fdt, xc.device)
    a_in, a_out = _arrays.to_cimx(xc), _arrays.to_cimx(gray)
    rc = _lib.lib.cimx_rgb2gray(ctypes.byref(a_in), ctypes.byref(a_out), _arrays.stream_of(xc))
    _lib.check(rc, "rgb2gray")
    return _arrays.wrap_like(rgb, gray)
