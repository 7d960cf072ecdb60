"""The rest of the separable family: laplace, gaussian_laplace,
generic_laplace (FLT:806-1009), minimum_filter1d / maximum_filter1d
(FLT:1362-1497) and skimage's difference_of_gaussians
(filters/_gaussian.py:13-174) and unsharp_mask (filters/_unsharp_mask.py:
12-160): bit for bit against the oracle (per-axis chains of the separable
kernels, summed in the output dtype: integers wrap; the unsharp combination
rounded operation by operation; min / max folded in double)."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


@pytest.fixture(scope="module")
def ski(cuda):
    from cucim_b200 import skimage

    return skimage


def _data(shape, dtype, seed=31):
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        return rng.integers(0, 200, shape).astype(dt)
    return rng.standard_normal(shape).astype(dt)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint8, np.uint16, np.int16])
@pytest.mark.parametrize("shape", [(40, 57), (9, 20, 24), (300,)])
def test_laplace(ndi, mode, dtype, shape):
    x = _data(shape, dtype)
    got = host(ndi.laplace(dev(x), mode=mode, cval=3.0))
    np.testing.assert_array_equal(got, R.laplace(x, mode=mode, cval=3.0))


def test_laplace_axes_output_and_empty_axes(ndi):
    x = _data((12, 18, 20), np.uint8)
    xd = dev(x)
    got = host(ndi.laplace(xd, output=np.float32, axes=(0, 2), mode=("mirror", "nearest")))
    exp = R.laplace(x, output=np.float32, axes=(0, 2), mode=("mirror", "nearest"))
    np.testing.assert_array_equal(got, exp)
    got = host(ndi.laplace(xd, output=np.uint16, axes=()))
    np.testing.assert_array_equal(got, R.laplace(x, output=np.uint16, axes=()))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("sigma", [1.0, (0.8, 2.0, 1.3), 3.0])
def test_gaussian_laplace(ndi, mode, sigma):
    x = _data((14, 33, 40), np.float32)
    got = host(ndi.gaussian_laplace(dev(x), sigma, mode=mode, cval=-1.0))
    np.testing.assert_array_equal(got, R.gaussian_laplace(x, sigma, mode=mode, cval=-1.0))


def test_gaussian_laplace_axes_dtypes_kwargs(ndi):
    x = _data((10, 30, 36), np.uint16)
    xd = dev(x)
    got = host(ndi.gaussian_laplace(xd, (1.5, 2.0), axes=(1, 2), output=np.float32,
                                    truncate=3.0))
    exp = R.gaussian_laplace(x, (1.5, 2.0), axes=(1, 2), output=np.float32, truncate=3.0)
    np.testing.assert_array_equal(got, exp)
    got = host(ndi.gaussian_laplace(xd, 1.0, output=np.int16))
    np.testing.assert_array_equal(got, R.gaussian_laplace(x, 1.0, output=np.int16))


def test_generic_laplace_user_callable(ndi):
    x = _data((25, 31), np.float32)
    w = np.array([0.5, -1.25, 0.75], dtype=np.float32)

    def d2(inp, axis, out, mode, cval, scale=1.0):
        return ndi.correlate1d(inp, w * scale, axis, out, mode, cval)

    def d2_ref(inp, axis, out, mode, cval, scale=1.0):
        return R.correlate1d(inp, w * scale, axis, out, mode, cval)

    got = host(ndi.generic_laplace(dev(x), d2, mode="nearest", extra_keywords={"scale": 2.0}))
    exp = R.generic_laplace(x, d2_ref, mode="nearest", extra_keywords={"scale": 2.0})
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.float64])
def test_difference_of_gaussians(ski, dtype):
    x = _data((48, 64), dtype)
    got = host(ski.filters.difference_of_gaussians(dev(x), 1.5))
    np.testing.assert_array_equal(got, R.difference_of_gaussians(x, 1.5))
    got = host(ski.filters.difference_of_gaussians(dev(x), (1.0, 2.0), (2.0, 5.0),
                                                   mode="reflect"))
    exp = R.difference_of_gaussians(x, (1.0, 2.0), (2.0, 5.0), mode="reflect")
    np.testing.assert_array_equal(got, exp)


def test_difference_of_gaussians_channels_and_errors(ski):
    x = _data((30, 40, 3), np.uint8)
    got = host(ski.filters.difference_of_gaussians(dev(x), 1.0, channel_axis=-1))
    np.testing.assert_array_equal(got, R.difference_of_gaussians(x, 1.0, channel_axis=-1))
    with pytest.raises(ValueError):
        ski.filters.difference_of_gaussians(dev(x), 2.0, 1.0, channel_axis=-1)


@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.float64, np.int16])
@pytest.mark.parametrize("radius,amount", [(1.0, 1.0), (2.5, 0.7), (0.5, 3.0)])
def test_unsharp_mask(ski, dtype, radius, amount):
    x = _data((40, 52), dtype)
    got = host(ski.filters.unsharp_mask(dev(x), radius, amount))
    np.testing.assert_array_equal(got, R.unsharp_mask(x, radius, amount))


def test_unsharp_mask_preserve_range_and_channels(ski):
    x = _data((24, 30, 3), np.uint8)
    got = host(ski.filters.unsharp_mask(dev(x), 2.0, 1.5, channel_axis=-1))
    np.testing.assert_array_equal(got, R.unsharp_mask(x, 2.0, 1.5, channel_axis=-1))
    got = host(ski.filters.unsharp_mask(dev(x), 1.0, 2.0, preserve_range=True))
    np.testing.assert_array_equal(got, R.unsharp_mask(x, 1.0, 2.0, preserve_range=True))
    xf = _data((24, 30), np.float32)  # negative values: clip to [-1, 1]
    got = host(ski.filters.unsharp_mask(dev(xf), 1.0, 1.0))
    np.testing.assert_array_equal(got, R.unsharp_mask(xf, 1.0, 1.0))



@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("dtype", [np.float32, np.uint8, np.uint16, np.int16, np.float64])
@pytest.mark.parametrize("shape", [(33, 47), (6, 20, 25), (500,)])
def test_min_max_filter1d(ndi, mode, dtype, shape):
    x = _data(shape, dtype)
    xd = dev(x)
    for axis in range(len(shape)):
        for size, origin in [(1, 0), (3, 0), (4, 1), (9, -3), (40, 2)]:
            for name in ("minimum_filter1d", "maximum_filter1d"):
                got = host(getattr(ndi, name)(xd, size, axis, mode=mode, cval=5.0,
                                              origin=origin))
                exp = getattr(R, name)(x, size, axis, mode=mode, cval=5.0, origin=origin)
                np.testing.assert_array_equal(got, exp)


def test_min_max_filter1d_nan_outputs_and_errors(ndi):
    x = _data((20, 30), np.float32)
    x[3, 4] = np.nan
    x[10, :] = np.nan  # a row of nan: nan survives only where the window is all nan
    xd = dev(x)
    for name in ("minimum_filter1d", "maximum_filter1d"):
        for axis in (0, 1):
            got = host(getattr(ndi, name)(xd, 5, axis))
            np.testing.assert_array_equal(got, getattr(R, name)(x, 5, axis))
        got = host(getattr(ndi, name)(dev(_data((20, 30), np.uint8)), 4, 0, output=np.int16,
                                      mode="constant", cval=300.0))
        exp = getattr(R, name)(_data((20, 30), np.uint8), 4, 0, output=np.int16,
                               mode="constant", cval=300.0)
        np.testing.assert_array_equal(got, exp)
    with pytest.raises(RuntimeError):
        ndi.minimum_filter1d(xd, 0)
    with pytest.raises(ValueError):
        ndi.minimum_filter1d(xd, 3, origin=2)



@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_generic_gradient_magnitude_user_callable(ndi, dtype):
    # FLT:1012-1097 with a user derivative: squares, sums and sqrt in libcimx
    x = _data((14, 30, 36), dtype)
    got = host(ndi.generic_gradient_magnitude(dev(x), ndi.sobel, mode="nearest"))
    exp = R.generic_gradient_magnitude(x, R.sobel, mode="nearest")
    np.testing.assert_array_equal(got, exp)
    got = host(ndi.generic_gradient_magnitude(dev(x), ndi.prewitt, axes=(0, 2),
                                              mode=("mirror", "constant"), cval=2.0))
    exp = R.generic_gradient_magnitude(x, R.prewitt, axes=(0, 2), mode=("mirror", "constant"),
                                       cval=2.0)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint16, np.int16])
@pytest.mark.parametrize("mode", ["reflect", "constant", "wrap"])
def test_min_max_filter1d_tiles(ndi, dtype, mode):
    """The shared-memory tiles: rows longer than one 1024-output segment,
    columns over several 32 x 64 tiles, windows from 2 to 80 elements;
    signed zeros and nan runs in the float inputs (the fold keeps the
    element-first, tap-ordered fmin / fmax of the reference kernel)."""
    x = _data((2, 90, 1100), dtype)
    if np.dtype(dtype).kind == "f":
        x[0, 5, 100:140] = -0.0
        x[0, 6, 100:140] = 0.0
        x[1, 7, 1000:1010] = np.nan
        x[1, 20:40, 33] = np.nan
    xd = dev(x)
    for axis in (2, 1, 0):
        for size, origin in [(2, 0), (15, 3), (80, -30)]:
            for name in ("minimum_filter1d", "maximum_filter1d"):
                got = host(getattr(ndi, name)(xd, size, axis, mode=mode, cval=-1.5,
                                              origin=origin))
                exp = getattr(R, name)(x, size, axis, mode=mode, cval=-1.5, origin=origin)
                assert got.dtype == exp.dtype
                if got.dtype.kind == "f":
                    u = np.uint32 if got.dtype.itemsize == 4 else np.uint64
                    nan = np.isnan(exp)
                    assert np.array_equal(np.isnan(got), nan)
                    np.testing.assert_array_equal(got.view(u)[~nan], exp.view(u)[~nan])
                else:
                    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype,cval", [(np.float32, 0.1), (np.float32, 2.5), (np.float16, 0.1),
                                        (np.float16, -7.0), (np.int32, 3.0)])
def test_min_max_filter1d_fold_precision(ndi, dtype, cval):
    """The fold runs in float32 when every value it sees is exact there
    (8/16-bit and float16/float32 inputs, a fill value float32 holds) and in
    float64 otherwise (a fill value like 0.1, 32-bit integer inputs); both
    give the reference's float64 fold."""
    x = _data((40, 1100), dtype)
    xd = dev(x)
    for axis in (0, 1):
        for name in ("minimum_filter1d", "maximum_filter1d"):
            for output in (None, np.float64):
                got = host(getattr(ndi, name)(xd, 7, axis, mode="constant", cval=cval,
                                              output=output))
                exp = getattr(R, name)(x, 7, axis, mode="constant", cval=cval, output=output)
                assert got.dtype == exp.dtype
                np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("mode", ["reflect", "mirror", "nearest", "wrap", "constant"])
@pytest.mark.parametrize("shape,axes", [((9, 70, 300), None), ((9, 70, 300), (2, 0)),
                                        ((40, 1000), None), ((40, 1000), (1,)), ((777,), None)])
def test_laplace_modes_axes_in_place(ndi, mode, shape, axes):
    """float32 laplace over every mode, axis subsets and orders, 1-D to 3-D,
    signed zeros: bit for bit the oracle (one pass per axis into the output
    and a temporary, added in place), also with the output overlapping the
    input."""
    x = _data(shape, np.float32)
    x.flat[::97] = -0.0
    xd = dev(x)
    got = host(ndi.laplace(xd, mode=mode, cval=1.25, axes=axes))
    exp = R.laplace(x, mode=mode, cval=1.25, axes=axes)
    np.testing.assert_array_equal(got.view(np.uint32), exp.view(np.uint32))
    y = xd.clone()
    ndi.laplace(y, output=y, mode=mode, cval=1.25, axes=axes)
    np.testing.assert_array_equal(host(y).view(np.uint32), exp.view(np.uint32))
