"""The generic row and column kernels and lone passes along the last axis
(correlate1d / convolve1d /
gaussian_filter1d / uniform_filter1d along axis -1, and filters whose only
pass besides the last axis is a leading one). Over float32 data the slab
kernel takes such a pass behind an identity y pass; every other pair runs
on the generic row kernel (typed or runtime-typed loads, outputs stored
straight or through the row buffer by their width). Either way the result
must equal the oracle bit for bit (cuCIM's
_vendored/_ndimage_filters.py:109-134 per pass) and the one-launch-per-pass
generic schedule."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]
SHAPES = [(33, 128), (7, 9, 244), (5, 70), (3, 4, 37), (17, 8), (2, 1, 100), (1, 3)]
PAIRS = [(np.float32, np.float32), (np.uint16, np.float32), (np.uint16, np.uint16),
         (np.uint8, np.uint8), (np.uint8, np.float32), (np.uint8, np.uint16),
         (np.float64, np.float64), (np.int16, np.float32), (np.float16, np.float32),
         (np.int32, np.float64)]


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def _input(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt.kind == "f":
        return (rng.standard_normal(shape) * 50).astype(dt)
    info = np.iinfo(dt)
    return rng.integers(max(info.min, -30000), min(info.max, 60000) + 1, shape).astype(dt)


def _same_bits(got, exp):
    assert got.dtype == exp.dtype, (got.dtype, exp.dtype)
    if got.dtype.kind == "f":
        nan = np.isnan(exp)
        assert np.array_equal(np.isnan(got), nan)
        u = {2: np.uint16, 4: np.uint32, 8: np.uint64}[got.dtype.itemsize]
        np.testing.assert_array_equal(got.view(u)[~nan], exp.view(u)[~nan])
    else:
        np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("tin,tout", PAIRS)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("mode", MODES)
def test_gaussian_last_axis(ndi, tin, tout, shape, mode):
    x = _input(shape, tin, 1)
    xd = dev(x)
    for sigma in (1.5, 4.0):  # 13 and 33 taps
        got = host(ndi.gaussian_filter1d(xd, sigma, axis=-1, mode=mode, cval=3.5, output=tout))
        _same_bits(got, R.gaussian_filter1d(x, sigma, axis=-1, mode=mode, cval=3.5,
                                            output=tout))
        with ndi.pass_by_pass():
            generic = host(ndi.gaussian_filter1d(xd, sigma, axis=-1, mode=mode, cval=3.5,
                                                 output=tout))
        _same_bits(got, generic)


@pytest.mark.parametrize("tin,tout", PAIRS[:6])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("algorithm", ["shared_memory", "elementwise"])
def test_correlate_last_axis_zero_taps(ndi, tin, tout, mode, algorithm):
    """Zero taps inside and at both ends (skipped by the elementwise rule),
    an origin, and both kernels' fill-value rules."""
    x = _input((6, 11, 52), tin, 2)
    w = np.array([0.0, 0.3, 0.0, -0.2, 0.5, 0.0])
    for convolve in (False, True):
        f = ndi.convolve1d if convolve else ndi.correlate1d
        g = R.convolve1d if convolve else R.correlate1d
        got = host(f(dev(x), w, axis=-1, mode=mode, cval=-1.25, origin=1, output=tout,
                     algorithm=algorithm))
        _same_bits(got, g(x, w, axis=-1, mode=mode, cval=-1.25, origin=1, output=tout,
                          algorithm=algorithm))


@pytest.mark.parametrize("tin,tout", PAIRS[:5])
@pytest.mark.parametrize("size", [1, 2, 5, 40])
def test_uniform_last_axis(ndi, tin, tout, size):
    x = _input((9, 30, 64), tin, 3)
    got = host(ndi.uniform_filter1d(dev(x), size, axis=-1, output=tout, mode="mirror"))
    _same_bits(got, R.uniform_filter1d(x, size, axis=-1, output=tout, mode="mirror"))


@pytest.mark.parametrize("tin,tout", PAIRS[:5])
@pytest.mark.parametrize("sigma", [(1.0, 0, 2.0), (0, 0, 1.5), (2.0, 0.0, 0.7)])
def test_leading_pass_then_last_axis(ndi, tin, tout, sigma):
    """A z pass (stream kernel) followed by the last axis alone."""
    x = _input((12, 20, 72), tin, 4)
    xd = dev(x)
    got = host(ndi.gaussian_filter(xd, sigma, mode="reflect", output=tout))
    _same_bits(got, R.gaussian_filter(x, sigma, mode="reflect", output=tout))
    with ndi.pass_by_pass():
        _same_bits(got, host(ndi.gaussian_filter(xd, sigma, mode="reflect", output=tout)))


def test_last_axis_non_finite_and_signed_zero(ndi):
    x = _input((8, 40), np.float32, 5)
    x[1, 3] = np.nan
    x[2, 0] = np.inf
    x[3, 39] = -np.inf
    x[4, :] = -0.0
    x[5, 10:20] = -0.0
    w = np.array([0.25, 0.5, 0.25])
    for mode in MODES:
        got = host(ndi.correlate1d(dev(x), w, axis=-1, mode=mode, cval=-0.0))
        _same_bits(got, R.correlate1d(x, w, axis=-1, mode=mode, cval=-0.0))


def test_last_axis_large_rows(ndi):
    """Rows longer than one slab tile and many slabs per CTA."""
    x = _input((40, 24, 3000), np.uint16, 6)
    xd = dev(x)
    got = host(ndi.gaussian_filter1d(xd, 2.0, axis=-1, output=np.float32))
    _same_bits(got, R.gaussian_filter1d(x, 2.0, axis=-1, output=np.float32))


@pytest.mark.parametrize("tin,tout", [(np.float64, np.float64), (np.float32, np.float32),
                                      (np.int16, np.float32), (np.int32, np.int32),
                                      (np.uint16, np.uint16), (np.float64, np.float32),
                                      (np.uint8, np.uint8), (np.uint8, np.float32),
                                      (np.uint16, np.float32), (np.float16, np.float16),
                                      (np.float16, np.float32), (np.int8, np.int8),
                                      (np.uint32, np.uint32), (np.int16, np.int16)])
@pytest.mark.parametrize("mode", MODES)
def test_strided_axes_generic(ndi, tin, tout, mode):
    """The generic strided-axis kernel: lines long enough for tiles inside
    the line (walked, typed loads for float32 / uint16 / uint8 / float64) and tiles past
    either end (the row table), every mode, through pass_by_pass so that no
    fused kernel takes the fast pairs."""
    x = _input((3, 300, 40), tin, 7)
    xd = dev(x)
    for axis, sigma in ((0, 1.0), (1, 1.5), (1, 6.0)):
        exp = R.gaussian_filter1d(x, sigma, axis=axis, mode=mode, cval=2.5, output=tout)
        with ndi.pass_by_pass():
            got = host(ndi.gaussian_filter1d(xd, sigma, axis=axis, mode=mode, cval=2.5,
                                              output=tout))
        _same_bits(got, exp)


@pytest.mark.parametrize("tin,tout", [(np.uint16, np.uint16), (np.uint16, np.float32),
                                      (np.uint8, np.uint8), (np.uint8, np.float32),
                                      (np.uint8, np.uint16)])
@pytest.mark.parametrize("ymode,xmode", [("reflect", "constant"), ("constant", "mirror"),
                                         ("constant", "constant"), ("wrap", "nearest"),
                                         ("mirror", "reflect"), ("nearest", "wrap")])
def test_integer_slab_modes(ndi, tin, tout, ymode, xmode):
    """The (y, x) slab kernel on 8/16-bit input with TMA-eligible rows (a
    multiple of 16 bytes): tiles inside the array and tiles past every edge,
    one mode per axis, a fill value that does not fit the input dtype; the
    y pass reads the raw tile directly except where rows outside take a
    constant fill."""
    x = _input((2, 70, 272), tin, 8)
    xd = dev(x)
    for sigma in ((0, 0.7, 1.2), (0, 2.0, 4.0), (0, 5.0, 1.0)):
        kw = dict(mode=("reflect", ymode, xmode), cval=3.5, output=tout)
        got = host(ndi.gaussian_filter(xd, sigma, **kw))
        _same_bits(got, R.gaussian_filter(x, sigma, **kw))
        with ndi.pass_by_pass():
            _same_bits(got, host(ndi.gaussian_filter(xd, sigma, **kw)))
