"""The fused kernels of the plain path on rows of a multiple of 4 elements
(the vector kernels' condition): the single-launch 3-D kernel (3 or 5 taps
on each of the last three axes: z, y and x passes in one launch) and the
(y, x) slab kernel with 9 or 17 taps. Their outputs must be bit-identical
to the oracle and to the pass-by-pass schedule (one launch per pass through
a scratch volume). The shapes cover partial tiles in y and x, short and
chunked z, a leading batch axis and rows of only 8 elements."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]
SHAPES = [(9, 70, 128), (7, 33, 244), (3, 9, 8), (2, 3, 19, 36), (130, 20, 16), (1, 66, 40)]


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def _ints(shape, dtype, seed, hi=250):
    return np.random.default_rng(seed).integers(0, hi, shape).astype(dtype)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("func", ["sobel", "prewitt"])
@pytest.mark.parametrize("tin,tout", [(np.uint16, np.float32), (np.uint8, np.uint8),
                                      (np.float32, np.float32), (np.uint8, np.float32),
                                      (np.uint8, np.uint16)])
def test_volume_sobel_prewitt(ndi, shape, func, tin, tout):
    x = _ints(shape, tin, 3)
    xd = dev(x)
    for axis in (-3, -2, -1):
        got = host(getattr(ndi, func)(xd, axis, output=tout))
        exp = getattr(R, func)(x, axis, output=tout)
        np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("size", [3, 5])
@pytest.mark.parametrize("shape", [(9, 70, 128), (7, 33, 244), (2, 3, 19, 36)])
def test_volume_uniform_u16_exact(ndi, mode, size, shape):
    x = _ints(shape, np.uint16, 1, hi=65536)
    got = host(ndi.uniform_filter(dev(x), size, output=np.uint16, mode=mode, cval=7))
    exp = R.uniform_filter(x, size, output=np.uint16, mode=mode, cval=7)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("tin,tout", [(np.uint8, np.uint8), (np.uint8, np.uint16),
                                      (np.uint16, np.uint16)])
def test_volume_integer_smoothing(ndi, mode, tin, tout):
    # non-negative taps on integer data: the truncating kernels
    hi = 256 if tin == np.uint8 else 65536
    x = _ints((7, 45, 132), tin, 4, hi=hi)
    xd = dev(x)
    for cval in (0.0, 200.0):
        got = host(ndi.gaussian_filter(xd, 0.5, mode=mode, cval=cval, output=tout))
        np.testing.assert_array_equal(got, R.gaussian_filter(x, 0.5, mode=mode, cval=cval,
                                                             output=tout))
        got = host(ndi.uniform_filter(xd, 3, mode=mode, cval=cval, output=tout))
        np.testing.assert_array_equal(got, R.uniform_filter(x, 3, mode=mode, cval=cval,
                                                            output=tout))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", [(9, 70, 128), (130, 20, 16), (3, 9, 8)])
def test_volume_float_modes(ndi, mode, shape):
    x = np.random.default_rng(5).standard_normal(shape).astype(np.float32)
    xd = dev(x)
    for got, exp in [
        (ndi.gaussian_filter(xd, 0.5, mode=mode, cval=-0.5),
         R.gaussian_filter(x, 0.5, mode=mode, cval=-0.5)),
        (ndi.uniform_filter(xd, 3, mode=mode, cval=1.25),
         R.uniform_filter(x, 3, mode=mode, cval=1.25)),
        (ndi.sobel(xd, 1, mode=mode, cval=2.0), R.sobel(x, 1, mode=mode, cval=2.0)),
    ]:
        np.testing.assert_array_equal(host(got), exp)


def test_volume_mixed_modes_and_origins(ndi):
    x = np.random.default_rng(6).standard_normal((11, 45, 132)).astype(np.float32)
    xd = dev(x)
    for mode, origin in [(("constant", "mirror", "nearest"), 0),
                         (("reflect", "constant", "constant"), 0),
                         (("mirror", "nearest", "constant"), (1, -1, 0)),
                         (("wrap", "wrap", "reflect"), 0),
                         ("nearest", (0, 0, 1))]:
        got = host(ndi.uniform_filter(xd, 3, mode=mode, cval=0.75, origin=origin))
        exp = R.uniform_filter(x, 3, mode=mode, cval=0.75, origin=origin)
        np.testing.assert_array_equal(got, exp)


def test_volume_batch_axis(ndi):
    # passes over the last three axes of a 4-D array: the batch loop
    x = _ints((3, 5, 21, 40), np.uint16, 8, hi=65536)
    got = host(ndi.uniform_filter(dev(x), 5, output=np.uint16, axes=(1, 2, 3), mode="mirror"))
    exp = R.uniform_filter(x, 5, output=np.uint16, axes=(1, 2, 3), mode="mirror")
    np.testing.assert_array_equal(got, exp)


def test_volume_nonfinite_and_zero_taps(ndi):
    # the derivative's zero tap is skipped: inf and nan do not leak through it
    x = np.random.default_rng(7).standard_normal((6, 20, 64)).astype(np.float32)
    x[2, 5, 10] = np.inf
    x[4, 11, 40] = np.nan
    xd = dev(x)
    for axis in range(3):
        np.testing.assert_array_equal(host(ndi.sobel(xd, axis)), R.sobel(x, axis))


@pytest.mark.parametrize("dtype", [np.float32, np.uint16])
def test_volume_matches_pass_by_pass(ndi, dtype):
    """At a larger size: the single launch against one launch per pass."""
    shape = (40, 300, 1000)
    if dtype == np.uint16:
        x = _ints(shape, dtype, 9, hi=65536)
        out = np.float32
    else:
        x = np.random.default_rng(9).random(shape, dtype=np.float32)
        out = np.float32
    xd = dev(x)
    calls = [lambda: ndi.sobel(xd, 0, output=out), lambda: ndi.sobel(xd, 2, output=out),
             lambda: ndi.uniform_filter(xd, 5, output=dtype),
             lambda: ndi.prewitt(xd, 1, output=out, mode="constant", cval=3.0)]
    for call in calls:
        got = call()
        with ndi.pass_by_pass():
            exp = call()
        assert torch.equal(got, exp)


@pytest.mark.parametrize("shape", [(64, 128), (40, 96), (7, 50, 72), (300, 260)])
@pytest.mark.parametrize("tout", [np.uint16, np.uint8])
def test_narrowed_intermediates_2d(ndi, shape, tout):
    """Sobel of uint8 into uint8 / uint16: the first pass's negative and
    out-of-range values are narrowed as cast<D>() stores them (wrap for
    negatives, saturation above the range) before the next pass reads them,
    also where the intermediate never leaves the chip (row-streaming and
    slab kernels)."""
    x = _ints(shape, np.uint8, 11, hi=256)
    xd = dev(x)
    for axis in range(len(shape)):
        got = host(ndi.sobel(xd, axis, output=tout))
        np.testing.assert_array_equal(got, R.sobel(x, axis, output=tout))
    got = host(ndi.uniform_filter(xd, 5, output=tout))
    np.testing.assert_array_equal(got, R.uniform_filter(x, 5, output=tout))


@pytest.mark.parametrize("tout", [np.uint16, np.uint8])
def test_narrowed_outputs_pass_by_pass(ndi, tout):
    """The one-launch-per-pass kernels narrow out-of-range results the same
    way (saturation for uint16, int16 saturation then the low 8 bits for
    uint8)."""
    x = _ints((9, 70, 128), np.uint8, 12, hi=256)
    xd = dev(x)
    with ndi.pass_by_pass():
        for axis in range(3):
            got = host(ndi.sobel(xd, axis, output=tout))
            np.testing.assert_array_equal(got, R.sobel(x, axis, output=tout))


@pytest.mark.parametrize("dtype,cval", [(np.uint8, 300.0), (np.uint8, -5.0), (np.uint16, 70000.0),
                                        (np.uint16, -3.0), (np.int16, 40000.0)])
@pytest.mark.parametrize("shape", [(40, 96), (6, 20, 64)])
def test_out_of_range_fill_values(ndi, dtype, cval, shape):
    # constant mode with a fill value outside the dtype's range: the
    # shared-memory kernel's rule converts it to the input dtype first
    x = _ints(shape, dtype, 13, hi=200)
    got = host(ndi.uniform_filter(dev(x), 3, mode="constant", cval=cval))
    np.testing.assert_array_equal(got, R.uniform_filter(x, 3, mode="constant", cval=cval))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", [(300, 1000), (7, 130, 232), (5, 9, 8), (2, 3, 150, 116)])
@pytest.mark.parametrize("sigma", [1.0, 2.0])
def test_slab_long_taps_gaussian(ndi, mode, shape, sigma):
    # 9 or 17 taps on the last two axes, with partial tiles in x and y,
    # rows shorter than the taps and a batch axis
    x = np.random.default_rng(21).standard_normal(shape).astype(np.float32)
    axes = tuple(range(len(shape)))[-2:]
    got = host(ndi.gaussian_filter(dev(x), sigma, mode=mode, cval=0.25, axes=axes))
    exp = R.gaussian_filter(x, sigma, mode=mode, cval=0.25, axes=axes)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("tin,tout", [(np.uint16, np.float32), (np.uint8, np.uint8),
                                      (np.uint16, np.uint16), (np.uint8, np.float32)])
def test_slab_long_taps_dtypes(ndi, tin, tout):
    x = _ints((3, 200, 360), tin, 22, hi=256 if tin == np.uint8 else 65536)
    xd = dev(x)
    for sigma, order in [((0, 2, 2), 0), ((0, 1, 1), 0), ((0, 2, 2), (0, 1, 0))]:
        got = host(ndi.gaussian_filter(xd, sigma, order=order, mode="mirror", output=tout))
        exp = R.gaussian_filter(x, sigma, order=order, mode="mirror", output=tout)
        np.testing.assert_array_equal(got, exp)


def test_slab_long_taps_match_pass_by_pass(ndi):
    x = torch.rand((24, 1024, 1024), device="cuda")
    got = ndi.gaussian_filter(x, (1, 2, 2), mode="mirror")
    with ndi.pass_by_pass():
        exp = ndi.gaussian_filter(x, (1, 2, 2), mode="mirror")
    assert torch.equal(got, exp)


@pytest.mark.parametrize("mode", ["mirror", "constant", "wrap"])
def test_long_leading_pass_then_slab(ndi, mode):
    # the z pass is longer than the stream kernel takes (25 taps): it runs on
    # the generic kernel, the (y, x) passes still as one slab launch
    x = np.random.default_rng(23).standard_normal((30, 70, 136)).astype(np.float32)
    xd = dev(x)
    got = ndi.gaussian_filter(xd, (3.0, 2.0, 1.5), mode=mode, cval=0.5)
    np.testing.assert_array_equal(host(got), R.gaussian_filter(x, (3.0, 2.0, 1.5), mode=mode,
                                                               cval=0.5))
    with ndi.pass_by_pass():
        exp = ndi.gaussian_filter(xd, (3.0, 2.0, 1.5), mode=mode, cval=0.5)
    assert torch.equal(got, exp)


def test_volume_status_clean(ndi):
    from cucim_b200 import _lib

    ndi.sobel(dev(np.ones((8, 16, 32), np.float32)), 0)
    torch.cuda.synchronize()
    assert _lib.lib.cimx_device_status(1) == 0


@pytest.mark.parametrize("axes", [(2, 0, 1), (1, 0, 2), (2, 1, 0), (1, 2), (2, 0)])
@pytest.mark.parametrize("tin,tout", [(np.uint16, np.uint16), (np.uint16, np.float32),
                                      (np.float32, np.float32), (np.uint8, np.uint8)])
def test_passes_out_of_axis_order(ndi, axes, tin, tout):
    """Axes in the caller's order (cuCIM keeps it, and each pass rounds
    through the output dtype, so the order matters): the fused kernels need
    ascending axes, so such lists run pass by pass, each pass on the fastest
    single-pass kernel that covers it. Bit for bit against the oracle and
    against the generic kernels one pass at a time."""
    shape = (20, 48, 64)
    x = _ints(shape, tin, 31) if np.dtype(tin).kind in "iu" else \
        np.random.default_rng(31).standard_normal(shape).astype(tin)
    xd = dev(x)
    calls = [
        (lambda f, a, o: f.gaussian_filter(a, 1.5, mode="mirror", output=o, axes=axes)),
        (lambda f, a, o: f.uniform_filter(a, 5, mode="reflect", output=o, axes=axes)),
    ]
    for call in calls:
        exp = call(R, x, np.empty(shape, tout))
        got = host(call(ndi, xd, torch.empty(shape, dtype=getattr(torch, np.dtype(tout).name),
                                             device="cuda")))
        np.testing.assert_array_equal(got, exp)
        with ndi.pass_by_pass():
            again = host(call(ndi, xd, torch.empty(shape,
                                                   dtype=getattr(torch, np.dtype(tout).name),
                                                   device="cuda")))
        np.testing.assert_array_equal(again, exp)


@pytest.mark.parametrize("taps", [3, 5, 7, 9, 11, 13, 15, 17, 19, 21, 23, 25])
@pytest.mark.parametrize("tin,tout", [(np.uint16, np.float32), (np.uint16, np.uint16),
                                      (np.float32, np.float32), (np.uint8, np.uint8)])
@pytest.mark.parametrize("mode", MODES)
def test_stream_tap_counts(ndi, taps, tin, tout, mode):
    """A pass along a leading axis at every tap count the stream kernel is
    instantiated for (19 and above: the generic kernel), uneven
    taps with an origin, against the oracle and the generic schedule."""
    x = _ints((23, 6, 40), tin, 30 + taps, hi=250)
    w = np.linspace(-0.4, 0.9, taps)
    origin = (taps - 1) // 2 - taps // 3
    xd = dev(x)
    kw = dict(axis=0, mode=mode, cval=2.5, origin=origin, output=tout)
    got = host(ndi.correlate1d(xd, w, **kw))
    np.testing.assert_array_equal(got, R.correlate1d(x, w, **kw))
    with ndi.pass_by_pass():
        np.testing.assert_array_equal(got, host(ndi.correlate1d(xd, w, **kw)))
