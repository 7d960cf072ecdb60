"""The whole-filter C entry points, called through ctypes alone (no Python
filter wrapper is involved: arrays are described with CimxArray structs
built here from device tensors), against the oracle: gaussian_filter,
uniform_filter, sobel / prewitt, gaussian_gradient_magnitude,
hessian_matrix and the ridge filters. These are what a host without the
Python layer (C, C++, Go over cgo, Java over JNI) calls.

float32 and integer inputs use float32 weights, whose taps the library
generates bit-identical to numpy's once rounded, so those results are
compared bit for bit. float64 inputs use float64 taps, which may differ from
numpy's in the last bits (see cimx_gaussian_taps), hence a tolerance of
1e-13 relative to each output and to the largest output there."""

import ctypes
import math

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = {"reflect": 0, "mirror": 1, "nearest": 2, "wrap": 3, "constant": 4}
NAN = float("nan")


@pytest.fixture(scope="module")
def lib(cuda):
    from cucim_b200 import _lib

    return _lib


def carr(lib, t):
    """CimxArray of a C-contiguous device tensor."""
    a = lib.CimxArray()
    a.data = t.data_ptr()
    a.dtype = ord(np.dtype(str(t.dtype).replace("torch.", "")).char)
    a.ndim = t.dim()
    for d in range(t.dim()):
        a.shape[d] = t.shape[d]
        a.strides[d] = t.stride(d) * t.element_size()
    return a


def ints(vals):
    return (ctypes.c_int * max(1, len(vals)))(*vals)


def dbls(vals):
    return (ctypes.c_double * max(1, len(vals)))(*vals)


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def empty(shape, dtype):
    return torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name), device="cuda")


def check(lib, rc):
    assert rc == 0, lib.last_error()


def compare(got, exp):
    if np.dtype(exp.dtype) == np.float64:
        # outputs that cancel to ~1e-15 of the scale carry the taps' last-bit
        # differences: the floor is relative to the largest output
        np.testing.assert_allclose(got, exp, rtol=1e-13,
                                   atol=1e-13 * float(np.abs(exp).max()))
    else:
        np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("shape,tin,tout", [((37, 53), np.float32, np.float32),
                                            ((9, 30, 41), np.float32, np.float32),
                                            ((9, 30, 41), np.uint16, np.float32),
                                            ((40, 44), np.uint8, np.uint8),
                                            ((12, 20, 24), np.uint16, np.uint16),
                                            ((33, 35), np.float64, np.float64)])
@pytest.mark.parametrize("mode", ["reflect", "mirror", "nearest", "wrap", "constant"])
def test_gaussian_nd(lib, shape, tin, tout, mode):
    rng = np.random.default_rng(1)
    x = (rng.random(shape) * 200).astype(tin)
    nd = len(shape)
    sig = [1.5, 0.7, 2.2][:nd]
    order = [0, 1, 2][:nd] if np.dtype(tout).kind == "f" else [0] * nd
    out = empty(shape, tout)
    check(lib, lib.lib.cimx_gaussian_nd(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                        dbls(sig), ints(order), None, ints([MODES[mode]] * nd),
                                        None, nd, 4.0, 3.0, 0, 0, None))
    torch.cuda.synchronize()
    exp = R.gaussian_filter(x, sig, order=order, mode=mode, cval=3.0, output=tout)
    compare(out.cpu().numpy(), exp)


def test_gaussian_nd_axes_radius_and_copy(lib):
    x = np.random.default_rng(2).random((8, 30, 41)).astype(np.float32)
    out = empty(x.shape, np.float32)
    check(lib, lib.lib.cimx_gaussian_nd(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                        dbls([2.0, 1.0]), None, ints([3, -1]), ints([0, 2]),
                                        ints([-1, 0]), 2, 4.0, 0.0, 0, 0, None))
    torch.cuda.synchronize()
    exp = R.gaussian_filter(x, [2.0, 1.0], mode=["reflect", "nearest"], radius=[3, None],
                            axes=(-1, 0))
    compare(out.cpu().numpy(), exp)
    # every sigma below the threshold: a cast-copy
    out16 = empty(x.shape, np.float64)
    check(lib, lib.lib.cimx_gaussian_nd(ctypes.byref(carr(lib, dev(x))),
                                        ctypes.byref(carr(lib, out16)), dbls([0.0, 0.0, 0.0]),
                                        None, None, ints([0, 0, 0]), None, 3, 4.0, 0.0, 0, 0,
                                        None))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out16.cpu().numpy(), x.astype(np.float64))


@pytest.mark.parametrize("algorithm", [0, 1, 2])
def test_gaussian_nd_algorithm_choice(lib, algorithm):
    """The shared-memory kernel rounds a constant-mode fill value through the
    input type; the elementwise kernel does not: cval 2.7 on uint8 input."""
    x = np.random.default_rng(3).integers(0, 255, (30, 40)).astype(np.uint8)
    out = empty(x.shape, np.float32)
    check(lib, lib.lib.cimx_gaussian_nd(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                        dbls([1.0, 1.0]), None, None, ints([4, 4]), None, 2, 4.0,
                                        2.7, algorithm, 0, None))
    torch.cuda.synchronize()
    alg = [None, "shared_memory", "elementwise"][algorithm]
    exp = R.gaussian_filter(x, 1.0, mode="constant", cval=2.7, output=np.float32, algorithm=alg)
    compare(out.cpu().numpy(), exp)


@pytest.mark.parametrize("shape,tin,tout", [((9, 30, 41), np.uint16, np.uint16),
                                            ((37, 53), np.uint8, np.uint8),
                                            ((9, 30, 41), np.float32, np.float32)])
def test_uniform_nd(lib, shape, tin, tout):
    x = (np.random.default_rng(4).random(shape) * 250).astype(tin)
    nd = len(shape)
    sizes, origins = [5, 3, 4][:nd], [0, 1, -1][:nd]
    out = empty(shape, tout)
    check(lib, lib.lib.cimx_uniform_nd(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                       ints(sizes), ints([1] * nd), ints(origins), None, nd, 0.0,
                                       0, 0, None))
    torch.cuda.synchronize()
    exp = R.uniform_filter(x, sizes, output=tout, mode="mirror", origin=origins)
    compare(out.cpu().numpy(), exp)


@pytest.mark.parametrize("prewitt", [0, 1])
@pytest.mark.parametrize("tin,tout", [(np.uint16, np.float32), (np.uint8, np.uint8),
                                      (np.float32, np.float32)])
def test_sobel_prewitt_nd(lib, prewitt, tin, tout):
    x = (np.random.default_rng(5).random((7, 33, 44)) * 250).astype(tin)
    for axis in (0, 1, -1):
        out = empty(x.shape, tout)
        check(lib, lib.lib.cimx_sobel_nd(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                         axis, ints([0, 0, 0]), 0.0, prewitt, 0, 0, None))
        torch.cuda.synchronize()
        exp = (R.prewitt if prewitt else R.sobel)(x, axis, output=tout)
        compare(out.cpu().numpy(), exp)


def test_gaussian_gradient_magnitude_nd(lib):
    x = np.random.default_rng(6).random((10, 31, 40)).astype(np.float32)
    out = empty(x.shape, np.float32)
    check(lib, lib.lib.cimx_gaussian_gradient_magnitude_nd(
        ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)), dbls([1.0, 2.0, 1.5]),
        ints([0, 1, 2]), 4.0, 0.0, 0, None))
    torch.cuda.synchronize()
    exp = R.gaussian_gradient_magnitude(x, [1.0, 2.0, 1.5], mode=["reflect", "mirror", "nearest"])
    compare(out.cpu().numpy(), exp)


@pytest.mark.parametrize("shape,dtype", [((30, 34), np.float32), ((12, 14, 16), np.float32),
                                         ((24, 26), np.uint8), ((10, 12, 14), np.float64)])
@pytest.mark.parametrize("sigma", [1.0, 2.5])
def test_hessian_gaussian_derivatives(lib, shape, dtype, sigma):
    x = (np.random.default_rng(7).random(shape) * 100).astype(dtype)
    nd = len(shape)
    F = R.supported_float_type(dtype)
    ne = nd * (nd + 1) // 2
    outs = [empty(shape, F) for _ in range(ne)]
    arr = (lib.CimxArray * ne)(*[carr(lib, o) for o in outs])
    check(lib, lib.lib.cimx_hessian(ctypes.byref(carr(lib, dev(x))), arr, ne, dbls([sigma] * nd),
                                    0, 0.0, 1, 0, 0, None))
    torch.cuda.synchronize()
    exp = R.hessian_matrix_gaussian(x, sigma, mode="reflect")
    for o, e in zip(outs, exp):
        compare(o.cpu().numpy(), e)


def test_hessian_finite_differences(lib):
    x = np.random.default_rng(8).random((26, 30)).astype(np.float32)
    outs = [empty(x.shape, np.float32) for _ in range(3)]
    arr = (lib.CimxArray * 3)(*[carr(lib, o) for o in outs])
    check(lib, lib.lib.cimx_hessian(ctypes.byref(carr(lib, dev(x))), arr, 3, dbls([1.5, 1.5]), 4,
                                    0.0, 0, 0, 0, None))
    torch.cuda.synchronize()
    exp = R.hessian_matrix_fd(x, 1.5, mode="constant")
    for o, e in zip(outs, exp):
        compare(o.cpu().numpy(), e)


@pytest.mark.parametrize("kind,name", [(0, "frangi"), (1, "meijering"), (2, "sato"),
                                       (3, "hessian")])
@pytest.mark.parametrize("shape", [(36, 40), (14, 16, 18)])
@pytest.mark.parametrize("black", [True, False])
def test_ridge_filter_matches_python_api(lib, kind, name, shape, black):
    """The C entry and the Python filter run the same kernels on the same
    float32 taps: bit-identical outputs."""
    from cucim_b200.skimage import filters

    x = np.random.default_rng(9).random(shape).astype(np.float32)
    xd = dev(x)
    out = empty(shape, np.float32)
    sig = [1.0, 2.0]
    check(lib, lib.lib.cimx_ridge_filter(ctypes.byref(carr(lib, xd)), ctypes.byref(carr(lib, out)),
                                         kind, dbls(sig), 2, 0.5 if kind != 1 else NAN, 0.5, NAN,
                                         1 if black else 0, 0, 0.0, 0, None))
    torch.cuda.synchronize()
    ref = getattr(filters, name)(xd, sigmas=sig, black_ridges=black)
    np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())


def test_frangi_uint8_input_converts_without_rescaling(lib):
    x = np.random.default_rng(10).integers(0, 255, (30, 32)).astype(np.uint8)
    out = empty(x.shape, np.float32)
    check(lib, lib.lib.cimx_frangi(ctypes.byref(carr(lib, dev(x))), ctypes.byref(carr(lib, out)),
                                   dbls([1.0, 2.0]), 2, 0.5, 0.5, NAN, 0, 0, 0.0, 0, None))
    torch.cuda.synchronize()
    exp = R.frangi(x, sigmas=[1.0, 2.0], black_ridges=False)
    got = out.cpu().numpy()
    big = np.abs(exp) >= 1e-3 * np.abs(exp).max()
    np.testing.assert_array_equal(got[big], exp[big])
    assert np.abs(got - exp).max() <= 1e-9 * np.abs(exp).max()
