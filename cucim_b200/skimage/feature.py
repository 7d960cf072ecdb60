"""hessian_matrix, structure_tensor, their eigenvalues and the corner
measures of cucim.skimage.feature (python/cucim/src/cucim/skimage/feature/
corner.py:21-158, :161-384, :473-858, :940-1284)."""

import ctypes
import math
from itertools import combinations_with_replacement
from warnings import warn

import numpy as np

from .. import _arrays, _lib
from .. import ndimage as ndi
from .._util import supported_float_type
from . import util as _u

__all__ = ["hessian_matrix", "hessian_matrix_eigvals", "structure_tensor",
           "structure_tensor_eigenvalues", "corner_kitchen_rosenfeld", "corner_harris",
           "corner_shi_tomasi", "corner_foerstner"]


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

    axes = list(range(ndim))
    if order == "xy":
        axes = axes[::-1]
    if ndim < 2:
        gradients = [g(image, orders[d]) for d in range(ndim)]
        return [g(gradients[a0], orders[a1]) for a0, a1 in combinations_with_replacement(axes, 2)]

    # Every chain runs its axis-0 pass first and most chains share it: the
    # gradients along axes >= 1 all start with the order-0 pass on the image,
    # and H[a0, a1] for a1 >= 1 all start with the order-0 pass on gradient
    # a0. Each shared pass runs once (a 1-pass call) and the rest of each
    # chain is a call over the remaining axes: the same passes in the same
    # order, so the results are bit-identical (6 axis-0 passes instead of 9
    # in 3-D).
    rest = tuple(range(1, ndim))

    def part(img, o, ax):
        return ndi.gaussian_filter(img, [sigma_scaled[a] for a in ax],
                                   order=[o[a] for a in ax], mode=mode, cval=cval,
                                   truncate=truncate, axes=ax, algorithm=algorithm)

    lead = {}

    def lead_pass(key, img, o0):
        if (key, o0) not in lead:
            lead[(key, o0)] = part(img, [o0] + [0] * (ndim - 1), (0,))
        return lead[(key, o0)]

    gradients = [part(lead_pass("image", image, orders[d][0]), orders[d], rest)
                 for d in range(ndim)]
    lead.clear()
    return [part(lead_pass(a0, gradients[a0], orders[a1][0]), orders[a1], rest)
            for a0, a1 in combinations_with_replacement(axes, 2)]


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


# ------------------------------------------------ structure tensor, corners

def _prepare_grayscale_input_nd(image):
    """feature/util.py:19-24: squeeze, 2-5 dimensions, img_as_float, the
    supported float type."""
    x = _arrays.as_tensor(image)
    x = x.squeeze()
    if x.dim() not in range(2, 6):
        raise ValueError("The parameter `image` must be a 2-, 3-, 4- or 5-dimensional array")
    return _as_float_image(x)


def _compute_derivatives(image, mode="constant", cval=0):
    """corner.py:21-45: the ndimage sobel along every axis."""
    ndim = _arrays.as_tensor(image).dim()
    return [ndi.sobel(image, axis=i, mode=mode, cval=cval) for i in range(ndim)]


def _multiply(a, b):
    ta, tb = _arrays.as_tensor(a).contiguous(), _arrays.as_tensor(b).contiguous()
    out = _arrays.empty(ta.shape, _arrays.np_dtype(ta), ta.device)
    ca, cb, co = _arrays.to_cimx(ta), _arrays.to_cimx(tb), _arrays.to_cimx(out)
    _lib.check(_lib.lib.cimx_multiply(ctypes.byref(ca), ctypes.byref(cb), ctypes.byref(co),
                                      _arrays.stream_of(ta)), "multiply")
    return out


def structure_tensor(image, sigma=1, mode="constant", cval=0, order="rc"):
    """corner.py:48-158: the Gaussian-weighted products of the sobel
    derivatives, upper-triangular elements in combinations_with_replacement
    order (Arr, Arc, Acc for 2-D)."""
    from .filters import gaussian  # noqa: PLC0415

    x = _arrays.as_tensor(image)
    if order == "xy" and x.dim() > 2:
        raise ValueError('Only "rc" order is supported for dim > 2.')
    if order not in ["rc", "xy"]:
        raise ValueError(f'order {order} is invalid. Must be either "rc" or "xy"')
    if not np.isscalar(sigma):
        sigma = tuple(sigma)
        if len(sigma) != x.dim():
            raise ValueError("sigma must have as many elements as image has axes")
    image = _prepare_grayscale_input_nd(image)
    derivatives = _compute_derivatives(image, mode=mode, cval=cval)
    if order == "xy":
        derivatives = list(reversed(derivatives))
    t = _arrays.as_tensor(image)
    channel_axis = -1 if (t.dim() == 3 and t.shape[-1] == 3) else None
    return [gaussian(_multiply(d0, d1), sigma=sigma, mode=mode, cval=cval,
                     channel_axis=channel_axis)
            for d0, d1 in combinations_with_replacement(derivatives, 2)]


def structure_tensor_eigenvalues(A_elems):
    """corner.py:786-821: eigenvalues in decreasing order, leading axis."""
    return symmetric_compute_eigenvalues(A_elems)


def _corner(kind, inputs, n_out=1, param=0.0):
    ts = [_arrays.as_tensor(i).contiguous() for i in inputs]
    outs = [_arrays.empty(ts[0].shape, _arrays.np_dtype(ts[0]), ts[0].device)
            for _ in range(n_out)]
    arr = (_lib.CimxArray * len(ts))(*[_arrays.to_cimx(t) for t in ts])
    co = [_arrays.to_cimx(o) for o in outs]
    rc = _lib.lib.cimx_corner_response(kind, arr, len(ts), ctypes.byref(co[0]),
                                       ctypes.byref(co[1]) if n_out > 1 else None,
                                       float(param), _arrays.stream_of(ts[0]))
    _lib.check(rc, "corner response")
    return [_arrays.wrap_like(inputs[0], o) for o in outs]


def corner_kitchen_rosenfeld(image, mode="constant", cval=0):
    """corner.py:962-1004."""
    fdt = supported_float_type(_arrays.np_dtype(_arrays.as_tensor(image)))
    image = _u.astype(image, fdt)
    imy, imx = _compute_derivatives(image, mode=mode, cval=cval)
    imxy, imxx = _compute_derivatives(imx, mode=mode, cval=cval)
    imyy = ndi.sobel(imy, axis=0, mode=mode, cval=cval)
    return _corner(_lib.CORNER_KITCHEN_ROSENFELD, [imx, imy, imxx, imxy, imyy])[0]


def corner_harris(image, method="k", k=0.05, eps=1e-6, sigma=1):
    """corner.py:1041-1113."""
    Arr, Arc, Acc = structure_tensor(image, sigma, order="rc")
    if method == "k":
        return _corner(_lib.CORNER_HARRIS_K, [Arr, Acc, Arc], param=k)[0]
    return _corner(_lib.CORNER_HARRIS_EPS, [Arr, Acc, Arc], param=eps)[0]


def corner_shi_tomasi(image, sigma=1):
    """corner.py:1131-1189."""
    Arr, Arc, Acc = structure_tensor(image, sigma, order="rc")
    return _corner(_lib.CORNER_SHI_TOMASI, [Arr, Acc, Arc])[0]


def corner_foerstner(image, sigma=1):
    """corner.py:1216-1284: (w, q)."""
    Arr, Arc, Acc = structure_tensor(image, sigma, order="rc")
    w, q = _corner(_lib.CORNER_FOERSTNER, [Arr, Acc, Arc], n_out=2)
    return w, q
