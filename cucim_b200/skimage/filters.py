"""gaussian, sobel, prewitt and the ridge filters (frangi, meijering, sato,
hessian) of cucim.skimage.filters (python/cucim/src/cucim/skimage/
_shared/filters.py:21-166, filters/edges.py:148-330 and :494,
filters/ridges.py:50-595)."""

import ctypes
import math
from collections.abc import Iterable

import numpy as np
import torch

from .. import _arrays, _lib
from .. import ndimage as ndi
from .._util import check_mode, supported_float_type
from . import util as _u
from .feature import _hessian_matrix_with_gaussian, symmetric_compute_eigenvalues

__all__ = ["gaussian", "difference_of_gaussians", "unsharp_mask", "sobel", "sobel_h", "sobel_v",
           "scharr", "scharr_h", "scharr_v", "prewitt", "prewitt_h", "prewitt_v", "farid",
           "farid_h", "farid_v", "frangi", "meijering", "sato", "hessian"]


def gaussian(image, sigma=1, mode="nearest", cval=0, preserve_range=False, truncate=4.0, *,
             channel_axis=None, out=None):
    """_shared/filters.py:21-166."""
    msg = "Sigma values less than zero are not valid"
    if not isinstance(sigma, Iterable):
        if sigma < 0:
            raise ValueError(msg)
    elif any(s < 0 for s in sigma):
        raise ValueError(msg)
    x = _arrays.as_tensor(image)
    if channel_axis is not None:
        axes = tuple(ax for ax in range(x.dim()) if ax != channel_axis % x.dim())
    else:
        axes = tuple(range(x.dim()))
    if x.dtype in (torch.float32, torch.float64):
        # already its own supported float type: convert_to_float and astype
        # leave it as it is
        image_f, fdt = image, x.dtype
    else:
        image_f = _u.convert_to_float(image, preserve_range)
        fdt = supported_float_type(_arrays.np_dtype(_arrays.as_tensor(image_f)))
        image_f = _u.astype(image_f, fdt)
    if out is None:
        return ndi.gaussian_filter(image_f, sigma, output=fdt, mode=mode, cval=cval,
                                   truncate=truncate, axes=axes)
    out_t = _arrays.as_tensor(out)
    if not out_t.dtype.is_floating_point:
        raise ValueError(f"dtype of `out` must be floating point; got {out_t.dtype!r}.")
    ndi.gaussian_filter(image_f, sigma, output=out, mode=mode, cval=cval, truncate=truncate,
                        axes=axes)
    return out


_SOBEL_SMOOTH = np.array([1, 2, 1]) / 4
_PREWITT_SMOOTH = np.full((3,), 1 / 3)
_SCHARR_SMOOTH = np.array([3, 10, 3]) / 16
# Farid & Simoncelli's 5-tap filters (the coefficients of edges.py:60-70)
_FARID_SMOOTH = np.array([0.0376593171958126, 0.249153396177344, 0.426374573253687,
                          0.249153396177344, 0.0376593171958126])
_FARID_EDGE = np.array([0.109603762960254, 0.276690988455557, 0, -0.276690988455557,
                        -0.109603762960254])


def difference_of_gaussians(image, low_sigma, high_sigma=None, *, mode="nearest", cval=0,
                            channel_axis=None, truncate=4.0):
    """filters/_gaussian.py:13-174: img_as_float, then gaussian(low_sigma)
    minus gaussian(high_sigma) (high_sigma defaults to 1.6 low_sigma), the
    subtraction in place in the float dtype (libcimx)."""
    image = _u.img_as_float(image)
    x = _arrays.as_tensor(image)
    spatial_dims = x.dim() - 1 if channel_axis is not None else x.dim()
    if np.isscalar(low_sigma):
        low_sigma = (low_sigma,) * spatial_dims
    low_sigma = tuple(map(float, low_sigma))
    if high_sigma is None:
        high_sigma = tuple(low * 1.6 for low in low_sigma)
    elif np.isscalar(high_sigma):
        high_sigma = (high_sigma,) * spatial_dims
    high_sigma = tuple(map(float, high_sigma))
    if len(low_sigma) != 1 and len(low_sigma) != spatial_dims:
        raise ValueError("low_sigma must have length equal to number of"
                         " spatial dimensions of input")
    if len(high_sigma) != 1 and len(high_sigma) != spatial_dims:
        raise ValueError("high_sigma must have length equal to number of"
                         " spatial dimensions of input")
    if any(s_hi < s_low for s_hi, s_low in zip(high_sigma, low_sigma)):
        raise ValueError("high_sigma must be equal to or larger thanlow_sigma for all axes")
    out = gaussian(image, sigma=low_sigma, mode=mode, cval=cval, channel_axis=channel_axis,
                   truncate=truncate, preserve_range=False)
    high = gaussian(image, sigma=high_sigma, mode=mode, cval=cval, channel_axis=channel_axis,
                    truncate=truncate, preserve_range=False)
    out_t = _arrays.as_tensor(out)
    ndi._combine(out_t, _arrays.as_tensor(high).contiguous(), _lib.COMBINE_SUBTRACT)
    return out


def _unsharp_mask_single_channel(image, radius, amount, vrange):
    """filters/_unsharp_mask.py:12-20: the gaussian blur (mode 'reflect'),
    then image + (image - blurred) * amount and the clip in one kernel."""
    img = _arrays.as_tensor(image).contiguous()
    blurred = _arrays.as_tensor(gaussian(img, sigma=radius, mode="reflect")).contiguous()
    out = torch.empty_like(img)
    a_img, a_bl, a_out = _arrays.to_cimx(img), _arrays.to_cimx(blurred), _arrays.to_cimx(out)
    clip, lo, hi = (0, 0.0, 0.0) if vrange is None else (1, float(vrange[0]), float(vrange[1]))
    rc = _lib.lib.cimx_unsharp(ctypes.byref(a_img), ctypes.byref(a_bl), ctypes.byref(a_out),
                               float(amount), clip, lo, hi, _arrays.stream_of(img))
    _lib.check(rc, "unsharp mask")
    return out


def unsharp_mask(image, radius=1.0, amount=1.0, preserve_range=False, *, channel_axis=None):
    """filters/_unsharp_mask.py:23-160: float conversion (img_as_float unless
    preserve_range), the clip range [-1, 1] or [0, 1] from whether any value
    is negative (a device reduction and one readback, as cp.any is), and the
    per-channel loop for channel_axis."""
    x = _arrays.as_tensor(image)
    float_dtype = supported_float_type(_arrays.np_dtype(x))
    vrange = None
    if preserve_range:
        fimg = _arrays.as_tensor(_u.astype(image, float_dtype))
    else:
        fimg = _arrays.as_tensor(_u.astype(_u.img_as_float(image), float_dtype)).contiguous()
        flag = ctypes.c_int(0)
        a = _arrays.to_cimx(fimg)
        rc = _lib.lib.cimx_any_negative(ctypes.byref(a), ctypes.byref(flag),
                                        _arrays.stream_of(fimg))
        _lib.check(rc, "unsharp mask range")
        vrange = [-1.0, 1.0] if flag.value else [0.0, 1.0]
    if channel_axis is not None:
        result = torch.empty_like(fimg)
        ax = channel_axis % fimg.dim()
        for c in range(fimg.shape[ax]):
            sl = tuple(c if d == ax else slice(None) for d in range(fimg.dim()))
            result[sl] = _unsharp_mask_single_channel(fimg[sl], radius, amount, vrange)
        return _arrays.wrap_like(image, result)
    return _arrays.wrap_like(image, _unsharp_mask_single_channel(fimg, radius, amount, vrange))


def _generic_edge_filter(image, *, smooth_weights, edge_weights=(1, 0, -1), axis=None,
                         mode="reflect", cval=0.0):
    """edges.py:148-241: the edge taps along each requested axis, the
    smoothing taps along every other axis (ascending), all as convolutions
    with float intermediates; with several axes the result is
    sqrt(sum of squares) with the edge taps divided by sqrt(ndim). `cval` is
    accepted and ignored, as in cuCIM."""
    x = _arrays.as_tensor(image)
    ndim = x.dim()
    if axis is None:
        axes = list(range(ndim))
    elif np.isscalar(axis):
        axes = [axis]
    else:
        axes = list(axis)
    magnitude = len(axes) > 1
    dt = _arrays.np_dtype(x)
    if dt.kind == "f":
        fdt = supported_float_type(dt)
        image = _u.astype(image, fdt)
    else:
        image = _u.img_as_float(image)
        fdt = _arrays.np_dtype(_arrays.as_tensor(image))
    ew = np.asarray(edge_weights, dtype=fdt)
    sw = np.asarray(smooth_weights, dtype=fdt)
    if magnitude:
        ew = (ew / fdt.type(math.sqrt(ndim))).astype(fdt)
    if not isinstance(mode, str):
        raise RuntimeError(f"boundary mode not supported (actual: {mode})")
    check_mode(mode)
    chains = []
    for ed in axes:
        ed_n = ed % ndim
        chain = [(ed_n, ew, mode, 0, True)]
        chain += [(sd, sw, mode, 0, True) for sd in sorted(set(range(ndim)) - {ed_n})]
        chains.append(chain)
    if magnitude:
        return ndi._gradient_magnitude(image, chains, fdt, 0.0)
    return ndi._run(image, chains[0], fdt, 0.0)


def _mask_filter_result(result, mask):
    """edges.py:75-85: the mask eroded with the full-connectivity footprint
    (border value 0) multiplies the result in place, on the device."""
    if mask is None:
        return result
    t = _arrays.as_tensor(result)
    m = _arrays.as_tensor(mask).contiguous()
    if tuple(m.shape) != tuple(t.shape):
        raise ValueError("mask must have the shape of the image")
    a_r, a_m = _arrays.to_cimx(t), _arrays.to_cimx(m)
    _lib.check(_lib.lib.cimx_mask_erode_multiply(ctypes.byref(a_r), ctypes.byref(a_m),
                                                 _arrays.stream_of(t)), "mask")
    return result


def _check_2d(image):
    if _arrays.as_tensor(image).dim() != 2:
        raise ValueError("The parameter `image` must be a 2-dimensional array")


def sobel(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """edges.py:244-299."""
    out = _generic_edge_filter(image, smooth_weights=_SOBEL_SMOOTH, axis=axis, mode=mode,
                               cval=cval)
    return _mask_filter_result(out, mask)


def sobel_h(image, mask=None):
    """edges.py:302-329: horizontal edges of a 2-D image."""
    _check_2d(image)
    return sobel(image, mask=mask, axis=0)


def sobel_v(image, mask=None):
    """edges.py:332-359: vertical edges of a 2-D image."""
    _check_2d(image)
    return sobel(image, mask=mask, axis=1)


def scharr(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """edges.py:362-422: smoothing taps [3, 10, 3] / 16."""
    out = _generic_edge_filter(image, smooth_weights=_SCHARR_SMOOTH, axis=axis, mode=mode,
                               cval=cval)
    return _mask_filter_result(out, mask)


def scharr_h(image, mask=None):
    """edges.py:425-457."""
    _check_2d(image)
    return scharr(image, mask=mask, axis=0)


def scharr_v(image, mask=None):
    """edges.py:460-491."""
    _check_2d(image)
    return scharr(image, mask=mask, axis=1)


def prewitt(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """edges.py:494-551."""
    out = _generic_edge_filter(image, smooth_weights=_PREWITT_SMOOTH, axis=axis, mode=mode,
                               cval=cval)
    return _mask_filter_result(out, mask)


def prewitt_h(image, mask=None):
    """edges.py:554-581."""
    _check_2d(image)
    return prewitt(image, mask=mask, axis=0)


def prewitt_v(image, mask=None):
    """edges.py:584-611."""
    _check_2d(image)
    return prewitt(image, mask=mask, axis=1)


def farid(image, mask=None, *, axis=None, mode="reflect", cval=0.0):
    """edges.py:783-850: Farid's 5-tap derivative and smoothing filters."""
    out = _generic_edge_filter(image, smooth_weights=_FARID_SMOOTH, edge_weights=_FARID_EDGE,
                               axis=axis, mode=mode, cval=cval)
    return _mask_filter_result(out, mask)


def farid_h(image, *, mask=None):
    """edges.py:853-890."""
    _check_2d(image)
    return farid(image, mask=mask, axis=0)


def farid_v(image, *, mask=None):
    """edges.py:893-927."""
    _check_2d(image)
    return farid(image, mask=mask, axis=1)


def frangi(image, sigmas=range(1, 10, 2), scale_range=None, scale_step=None, alpha=0.5,
           beta=0.5, gamma=None, black_ridges=True, mode="reflect", cval=0, *,
           algorithm=None):
    """ridges.py:322-476. The automatic gamma (half the largest Hessian norm
    of the first scale) stays on the device: no host synchronisation.
    `algorithm="tensor"` (an addition of this library) runs the Hessian's
    Gaussian-derivative passes with 16 taps or more on the tensor cores
    (TF32x3); the default is cuCIM's float32 arithmetic."""
    if scale_range is not None and scale_step is not None:
        sigmas = np.arange(scale_range[0], scale_range[1], scale_step)
    x = _arrays.as_tensor(image)
    if x.dim() not in (2, 3):
        raise ValueError(
            f"The parameter `image` must be a 2-dimensional or 3-dimensional array")
    fdt = supported_float_type(_arrays.np_dtype(x))
    if black_ridges:
        image = _u.astype(image, fdt)
    else:
        image = _u.negative_astype(image, fdt)
    ndim = x.dim()
    out = _arrays.empty(x.shape, fdt, x.device)
    state = torch.zeros(1, dtype=torch.int64, device=x.device)
    g = float("nan") if gamma is None else float(gamma)
    a_out = _arrays.to_cimx(out)
    for i, sigma in enumerate(sigmas):
        H = [_arrays.as_tensor(h).contiguous() for h in
             _hessian_matrix_with_gaussian(image, sigma, mode=mode, cval=cval,
                                           algorithm=algorithm)]
        # eigenvalues and vesselness in one pass over the Hessian elements
        hs = (_lib.CimxArray * len(H))(*[_arrays.to_cimx(h) for h in H])
        rc = _lib.lib.cimx_frangi_hessian_accumulate(hs, len(H), ctypes.byref(a_out),
                                                     float(alpha), float(beta), g,
                                                     1 if i == 0 else 0,
                                                     ctypes.c_void_p(state.data_ptr()),
                                                     _arrays.stream_of(out))
        _lib.check(rc, "frangi")
    return _arrays.wrap_like(image, out)


def _ridge_image(image, black_ridges, names):
    """image.astype(_supported_float_type), negated for white ridges
    (ridges.py:107-109, :200-202)."""
    x = _arrays.as_tensor(image)
    if x.dim() not in (2, 3):
        raise NotImplementedError(
            f"{names} is implemented here for 2-D and 3-D images (the closed-form eigenvalues)")
    fdt = supported_float_type(_arrays.np_dtype(x))
    img = _u.astype(image, fdt) if black_ridges else _u.negative_astype(image, fdt)
    return img, x.dim(), fdt, x.shape, x.device


def _eig_arrays(H, ndim):
    ev = _arrays.as_tensor(symmetric_compute_eigenvalues(H))  # descending
    return ev, (_lib.CimxArray * ndim)(*[_arrays.to_cimx(ev[k]) for k in range(ndim)])


def meijering(image, sigmas=range(1, 10, 2), alpha=None, black_ridges=True, mode="reflect",
              cval=0):
    """ridges.py:50-146: Meijering neuriteness. Per scale the eigenvalues of
    the Gaussian-derivative Hessian (descending) are mixed by the circulant
    matrix (1 on the diagonal, alpha = 1 / (ndim + 1) by default elsewhere),
    the mixed value of largest magnitude is kept, clipped at 0, normalised by
    its maximum over the image (reduced on the device: no host
    synchronisation) and folded into the maximum over scales."""
    img, ndim, fdt, shape, device = _ridge_image(image, black_ridges, "meijering")
    if alpha is None:
        alpha = 1 / (ndim + 1)
    out = torch.zeros(tuple(shape), dtype=_arrays.torch_dtype(fdt), device=device)
    state = torch.zeros(2, dtype=torch.int64, device=device)
    a_out = _arrays.to_cimx(out)
    for i, sigma in enumerate(sigmas):
        H = _hessian_matrix_with_gaussian(img, sigma, mode=mode, cval=cval)
        ev, eigs = _eig_arrays(H, ndim)
        rc = _lib.lib.cimx_meijering_accumulate(eigs, ndim, ctypes.byref(a_out), float(alpha),
                                                1 if i == 0 else 0,
                                                ctypes.c_void_p(state.data_ptr()),
                                                _arrays.stream_of(out))
        _lib.check(rc, "meijering")
    return _arrays.wrap_like(img, out)


def sato(image, sigmas=range(1, 10, 2), black_ridges=True, mode="reflect", cval=0):
    """ridges.py:148-225: Sato tubeness. Per scale the geometric mean of the
    Hessian eigenvalues but the lowest, clipped at 0, times sigma^2, folded
    into the maximum over scales."""
    img, ndim, fdt, shape, device = _ridge_image(image, black_ridges, "sato")
    out = torch.zeros(tuple(shape), dtype=_arrays.torch_dtype(fdt), device=device)
    a_out = _arrays.to_cimx(out)
    for i, sigma in enumerate(sigmas):
        H = _hessian_matrix_with_gaussian(img, sigma, mode=mode, cval=cval)
        ev, eigs = _eig_arrays(H, ndim)
        rc = _lib.lib.cimx_sato_accumulate(eigs, ndim, ctypes.byref(a_out), float(sigma),
                                           1 if i == 0 else 0, _arrays.stream_of(out))
        _lib.check(rc, "sato")
    return _arrays.wrap_like(img, out)


def hessian(image, sigmas=range(1, 10, 2), scale_range=None, scale_step=None, alpha=0.5,
            beta=0.5, gamma=15, black_ridges=True, mode="reflect", cval=0):
    """ridges.py:479-595: the hybrid Hessian filter, frangi with gamma 15 by
    default and every output <= 0 set to 1."""
    out = frangi(image, sigmas=sigmas, scale_range=scale_range, scale_step=scale_step,
                 alpha=alpha, beta=beta, gamma=gamma, black_ridges=black_ridges, mode=mode,
                 cval=cval)
    t = _arrays.as_tensor(out)
    a = _arrays.to_cimx(t)
    _lib.check(_lib.lib.cimx_nonpositive_to_one(ctypes.byref(a), _arrays.stream_of(t)),
               "hessian")
    return out
