"""hessian_matrix and its eigenvalues from cucim.skimage.feature
(python/cucim/src/cucim/skimage/feature/corner.py:161-362, :473-837)."""

import ctypes
import math
from itertools import combinations_with_replacement
from warnings import warn

import numpy as np

from .. import _arrays, _lib
from .. import ndimage as ndi
from .._util import supported_float_type
from . import util as _u

__all__ = ["hessian_matrix", "hessian_matrix_eigvals"]


def _as_float_image(image):
    image = _u.img_as_float(image)
    fdt = supported_float_type(_arrays.np_dtype(_arrays.as_tensor(image)))
    return _u.astype(image, fdt)


def _hessian_matrix_with_gaussian(image, sigma=1, mode="reflect", cval=0, order="rc", *,
                                  algorithm=None):
    """corner.py:161-254: Gaussian-derivative Hessian. sigma is scaled by
    1/sqrt(2) for each of the two first-derivative passes; truncate is 8 when
    every sigma exceeds 1 and 100 otherwise. `algorithm` is passed to
    gaussian_filter ("tensor" runs the float32 passes with 16 taps or more on
    the tensor cores; an addition of this library)."""
    image = _as_float_image(image)
    x = _arrays.as_tensor(image)
    ndim = x.dim()
    if ndim > 2 and order == "xy":
        raise ValueError("Order 'xy' is only supported for 2D images.")
    if order not in ["rc", "xy"]:
        raise ValueError(f"unrecognized order: {order}")
    if np.isscalar(sigma):
        sigma = (sigma,) * ndim
    truncate = 8 if all(s > 1 for s in sigma) else 100
    sq1_2 = 1 / math.sqrt(2)
    sigma_scaled = tuple(sq1_2 * s for s in sigma)
    orders = tuple([0] * d + [1] + [0] * (ndim - d - 1) for d in range(ndim))

    def g(img, o):
        return ndi.gaussian_filter(img, sigma_scaled, order=o, mode=mode, cval=cval,
                                   truncate=truncate, algorithm=algorithm)

    gradients = [g(image, orders[d]) for d in range(ndim)]
    axes = range(ndim)
    if order == "xy":
        axes = reversed(axes)
    return [g(gradients[a0], orders[a1]) for a0, a1 in combinations_with_replacement(axes, 2)]


def _gradient(f, axis):
    x = _arrays.as_tensor(f).contiguous()
    out = _arrays.empty(x.shape, _arrays.np_dtype(x), x.device)
    a_in, a_out = _arrays.to_cimx(x), _arrays.to_cimx(out)
    rc = _lib.lib.cimx_gradient_fd(ctypes.byref(a_in), ctypes.byref(a_out), axis,
                                   _arrays.stream_of(x))
    if rc != 0 and "too small" in _lib.last_error():
        raise ValueError(_lib.last_error())
    _lib.check(rc, "gradient")
    return _arrays.wrap_like(f, out)


def hessian_matrix(image, sigma=1, mode="constant", cval=0, order="rc",
                   use_gaussian_derivatives=None):
    """corner.py:257-384."""
    from .filters import gaussian  # noqa: PLC0415

    image = _as_float_image(image)
    x = _arrays.as_tensor(image)
    if x.dim() > 2 and order == "xy":
        raise ValueError("Order 'xy' is only supported for 2D images.")
    if order not in ["rc", "xy"]:
        raise ValueError(f"unrecognized order: {order}")
    if use_gaussian_derivatives is None:
        use_gaussian_derivatives = False
        warn(
            "use_gaussian_derivatives currently defaults to False, but will "
            "change to True in a future version. Please specify this "
            "argument explicitly to maintain the current behavior",
            category=FutureWarning,
            stacklevel=2,
        )
    if use_gaussian_derivatives:
        return _hessian_matrix_with_gaussian(image, sigma=sigma, mode=mode, cval=cval,
                                             order=order)
    channel_axis = -1 if (x.dim() == 3 and x.shape[-1] == 3) else None
    smoothed = gaussian(image, sigma=sigma, mode=mode, cval=cval, channel_axis=channel_axis)
    ndim = x.dim()
    gradients = [_gradient(smoothed, a) for a in range(ndim)]
    axes = range(ndim)
    if order == "xy":
        axes = reversed(axes)
    return [_gradient(gradients[a0], a1) for a0, a1 in combinations_with_replacement(axes, 2)]


def symmetric_compute_eigenvalues(S_elems, sort="descending", abs_sort=False):
    """corner.py:699-755 for 2-D (3 elements) and 3-D (6 elements)."""
    if sort not in ("ascending", "descending"):
        raise ValueError(f"unknown sort type: {sort}")
    ts = [_arrays.as_tensor(s).contiguous() for s in S_elems]
    if len(ts) not in (3, 6):
        raise NotImplementedError("eigenvalues are implemented for 2-D and 3-D images only")
    dt = _arrays.np_dtype(ts[0])
    if dt.kind != "f":
        raise ValueError("expected real-valued floating point matrices")
    n_out = 2 if len(ts) == 3 else 3
    eigs = _arrays.empty((n_out,) + tuple(ts[0].shape), dt, ts[0].device)
    elems = (_lib.CimxArray * len(ts))(*[_arrays.to_cimx(t) for t in ts])
    outs = (_lib.CimxArray * n_out)(*[_arrays.to_cimx(eigs[i]) for i in range(n_out)])
    rc = _lib.lib.cimx_eigvals_sym(elems, len(ts), outs, 1 if sort == "descending" else 0,
                                   1 if abs_sort else 0, _arrays.stream_of(ts[0]))
    _lib.check(rc, "eigvals")
    return _arrays.wrap_like(S_elems[0], eigs)


def hessian_matrix_eigvals(H_elems):
    """corner.py:824-858: eigenvalues in decreasing order, leading axis."""
    return symmetric_compute_eigenvalues(H_elems)
