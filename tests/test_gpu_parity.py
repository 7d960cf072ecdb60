"""GPU parity: libcimx's kernels against the oracle on the same seeded inputs.

Separable filters are compared bit for bit (integer and float outputs alike:
the kernels run the oracle's exact fused multiply-add chain). Composite
operations with float64 transcendental functions (eigenvalues, frangi) are
compared within a stated tolerance.
"""

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


def _rand(shape, dtype, seed=123):
    rng = np.random.default_rng(seed)
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        return rng.integers(0, 128, shape).astype(dt)
    return rng.standard_normal(shape).astype(dt)


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


@pytest.fixture(scope="module")
def ski(cuda):
    from cucim_b200 import skimage

    return skimage


# ----------------------------------------------------------- correlate1d

@pytest.mark.parametrize("shape", [(64, 57), (1000, 50), (5, 500), (1500, 5), (1, 1), (7,),
                                   (6, 9, 11), (3, 4, 5, 6)])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K", [1, 2, 3, 4, 9, 16, 17, 33])
def test_correlate1d_f32(ndi, shape, mode, K):
    x = _rand(shape, np.float32, seed=K)
    w = np.random.default_rng(K + 1).standard_normal(K).astype(np.float32)
    xd = dev(x)
    for axis in range(len(shape)):
        for origin in sorted({-(K // 2), 0, (K - 1) // 2 - (1 - K % 2)}):
            if K // 2 + origin < 0 or K // 2 + origin >= K:
                continue
            got = host(ndi.correlate1d(xd, w, axis, mode=mode, cval=0.5, origin=origin))
            exp = R.correlate1d(x, w, axis, mode=mode, cval=0.5, origin=origin)
            np.testing.assert_array_equal(got, exp, err_msg=f"axis={axis} origin={origin}")


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K", [3, 4, 7])
def test_convolve1d_f32(ndi, mode, K):
    x = _rand((33, 40), np.float32)
    w = np.random.default_rng(2).standard_normal(K).astype(np.float32)
    xd = dev(x)
    for axis in (0, 1):
        for origin in (-(K // 2), 0):
            got = host(ndi.convolve1d(xd, w, axis, mode=mode, origin=origin))
            exp = R.convolve1d(x, w, axis, mode=mode, origin=origin)
            np.testing.assert_array_equal(got, exp)


DTYPE_PAIRS = [
    (np.uint8, np.uint8), (np.uint8, np.float32), (np.int8, np.int8), (np.uint16, np.uint16),
    (np.uint16, np.float32), (np.int16, np.int16), (np.int16, np.float64),
    (np.uint32, np.uint32), (np.int32, np.int32), (np.int32, np.float32), (np.int64, np.int64),
    (np.uint64, np.float64), (np.float16, np.float16), (np.float16, np.float32),
    (np.float32, np.float32), (np.float32, np.uint16), (np.float64, np.float64),
    (np.float64, np.float32),
]


@pytest.mark.parametrize("tin,tout", DTYPE_PAIRS)
@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("mode,cval", [("reflect", 0.0), ("constant", 1.5),
                                       ("constant", -2.25)])
def test_correlate1d_dtypes(ndi, tin, tout, ndim, mode, cval):
    shape = (31, 44) if ndim == 2 else (9, 13, 17)
    x = _rand(shape, tin, seed=5)
    xd = dev(x)
    for w in (np.array([0.25, 0.5, 0.25, 0.125, 0.0625], np.float32),
              np.array([-1.0, 0.0, 1.0], np.float64), np.array([1, 2, 1], np.int64)):
        for axis in range(ndim):
            got = host(ndi.correlate1d(xd, w, axis, output=tout, mode=mode, cval=cval))
            exp = R.correlate1d(x, w, axis, output=tout, mode=mode, cval=cval)
            assert got.dtype == exp.dtype
            np.testing.assert_array_equal(got, exp, err_msg=f"w={w} axis={axis}")


@pytest.mark.parametrize("algorithm", [None, "shared_memory", "elementwise"])
def test_algorithm_kwarg(ndi, algorithm):
    x = _rand((40, 30), np.uint16)
    w = np.array([0.5, 0.0, 0.5], np.float32)
    xd = dev(x)
    got = host(ndi.correlate1d(xd, w, 0, output=np.float32, mode="constant", cval=3.7,
                               algorithm=algorithm))
    exp = R.correlate1d(x, w, 0, output=np.float32, mode="constant", cval=3.7,
                        algorithm=algorithm)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("K", [65, 129, 257, 601, 2049])
@pytest.mark.parametrize("shape", [(300, 200), (5, 40, 37)])
def test_long_kernels(ndi, K, shape):
    x = _rand(shape, np.float32)
    w = np.random.default_rng(K).random(K).astype(np.float32)
    xd = dev(x)
    for axis in range(len(shape)):
        got = host(ndi.correlate1d(xd, w, axis, mode="nearest"))
        exp = R.correlate1d(x, w, axis, mode="nearest")
        np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype", [np.float32, np.uint16])
def test_very_long_kernel_short_rows(ndi, dtype):
    """8001 taps on 100-sample rows: the row kernel packs 8 rows per CTA and
    would need more shared memory than a CTA has, so the pass runs on the
    per-output kernel; along axis 0 the column kernels take it."""
    x = _rand((16, 100), dtype, seed=8)
    w = np.random.default_rng(8001).random(8001).astype(np.float32) / 8001
    xd = dev(x)
    for axis in (0, 1):
        for mode in ("nearest", "mirror", "constant"):
            got = host(ndi.correlate1d(xd, w, axis, mode=mode, cval=2.0, output=np.float32))
            exp = R.correlate1d(x, w, axis, mode=mode, cval=2.0, output=np.float32)
            np.testing.assert_array_equal(got, exp, err_msg=f"axis={axis} mode={mode}")


def test_nonfinite_inputs_and_zero_taps(ndi):
    """Zero taps are skipped by the elementwise kernel (3-D) but not by the
    shared-memory kernel (2-D): an inf under a zero tap differs."""
    for shape in [(12, 13), (3, 12, 13)]:
        x = _rand(shape, np.float32)
        x.flat[40] = np.inf
        x.flat[77] = np.nan
        xd = dev(x)
        for axis in range(len(shape)):
            got = host(ndi.sobel(xd, axis))
            exp = R.sobel(x, axis)
            np.testing.assert_array_equal(got, exp)


def test_empty_arrays(ndi):
    for shape in [(0,), (0, 5), (4, 0, 3)]:
        x = dev(np.zeros(shape, np.float32))
        assert tuple(ndi.gaussian_filter(x, 2.0).shape) == shape
        assert tuple(ndi.uniform_filter(x, 3).shape) == shape


# ------------------------------------------------------- filter family

@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", [(64, 57), (1000, 50), (8, 9, 10), (2, 3, 4, 5)])
def test_uniform_u16_exact(ndi, mode, shape):
    x = np.random.default_rng(1).integers(0, 65536, shape).astype(np.uint16)
    got = host(ndi.uniform_filter(dev(x), 5, output=np.uint16, mode=mode, cval=7))
    exp = R.uniform_filter(x, 5, output=np.uint16, mode=mode, cval=7)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("size", [2, 3, (3, 1, 4), 8, 63])
def test_uniform_sizes(ndi, size):
    x = _rand((20, 30, 25), np.float32)
    got = host(ndi.uniform_filter(dev(x), size, mode="mirror"))
    exp = R.uniform_filter(x, size, mode="mirror")
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("sigma", [0.5, 1.0, (1, 2, 2), 3.3])
@pytest.mark.parametrize("order", [0, 1, (0, 2, 1)])
@pytest.mark.parametrize("mode", MODES)
def test_gaussian_filter(ndi, sigma, order, mode):
    x = _rand((12, 21, 19), np.float32)
    got = host(ndi.gaussian_filter(dev(x), sigma, order=order, mode=mode, cval=-0.5))
    exp = R.gaussian_filter(x, sigma, order=order, mode=mode, cval=-0.5)
    np.testing.assert_array_equal(got, exp)


def test_gaussian_filter_u16_to_f32_mirror(ndi):
    """The 3-D stack workload at small size: uint16 in, float32 out."""
    from cucim_b200 import synthetic

    x = synthetic.smooth_volume_u16((16, 40, 48), seed=1)
    got = host(ndi.gaussian_filter(dev(x), (1, 2, 2), mode="mirror", output=np.float32))
    exp = R.gaussian_filter(x, (1, 2, 2), mode="mirror", output=np.float32)
    np.testing.assert_array_equal(got, exp)


def test_gaussian_axes_and_radius(ndi):
    x = _rand((15, 16, 17), np.float64)
    got = host(ndi.gaussian_filter(dev(x), (1.5, 2.0), axes=(2, 0), radius=(3, 2),
                                   mode=("wrap", "nearest")))
    exp = R.gaussian_filter(x, (1.5, 2.0), axes=(2, 0), radius=(3, 2), mode=("wrap", "nearest"))
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("func", ["sobel", "prewitt"])
@pytest.mark.parametrize("tin,tout", [(np.uint16, np.float32), (np.uint8, np.uint8),
                                      (np.float32, np.float32), (np.int16, np.int16)])
def test_sobel_prewitt(ndi, func, tin, tout):
    x = np.random.default_rng(3).integers(0, 250, (10, 17, 19)).astype(tin)
    xd = dev(x)
    for axis in range(3):
        got = host(getattr(ndi, func)(xd, axis, output=tout))
        exp = getattr(R, func)(x, axis, output=tout)
        np.testing.assert_array_equal(got, exp)


def test_uint8_cast_wraps_like_the_gpu(ndi):
    """Out-of-range results stored to uint8: sobel of a uint8 step reaches
    +-1020; cast<uint8>() of those is what the oracle's cast table says."""
    x = np.zeros((8, 16), np.uint8)
    x[:, 8:] = 255
    for axis in (0, 1):
        got = host(ndi.sobel(dev(x), axis))
        exp = R.sobel(x, axis)
        np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gaussian_gradient_magnitude(ndi, dtype):
    x = _rand((23, 31, 17), dtype)
    got = host(ndi.gaussian_gradient_magnitude(dev(x), 1.3, mode="reflect"))
    exp = R.gaussian_gradient_magnitude(x, 1.3, mode="reflect")
    np.testing.assert_array_equal(got, exp)


# ------------------------------------------------------------ skimage layer

@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float16, np.float32, np.float64])
def test_sk_gaussian(ski, dtype):
    x = _rand((40, 50), dtype)
    got = host(ski.filters.gaussian(dev(x), sigma=2.0))
    exp = R.sk_gaussian(x, sigma=2.0)
    assert got.dtype == exp.dtype
    np.testing.assert_array_equal(got, exp)


def test_sk_gaussian_channel_axis(ski):
    x = _rand((30, 20, 3), np.float32)
    got = host(ski.filters.gaussian(dev(x), sigma=1.5, channel_axis=-1, mode="reflect"))
    exp = R.sk_gaussian(x, sigma=1.5, channel_axis=-1, mode="reflect")
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("func", ["sobel", "prewitt"])
@pytest.mark.parametrize("axis", [None, 0, 1, (0, 1)])
@pytest.mark.parametrize("dtype", [np.uint8, np.float32])
def test_sk_edges(ski, func, axis, dtype):
    x = _rand((33, 47), dtype)
    got = host(getattr(ski.filters, func)(dev(x), axis=axis))
    exp = getattr(R, "sk_" + func)(x, axis=axis)
    np.testing.assert_array_equal(got, exp)


def test_sk_edges_3d(ski):
    x = _rand((9, 13, 15), np.float32)
    got = host(ski.filters.sobel(dev(x)))
    exp = R.sk_sobel(x)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("shape", [(25, 27), (9, 12, 14)])
@pytest.mark.parametrize("sigma", [0.7, 1.0, 2.5])
def test_hessian_gaussian_derivatives(ski, shape, sigma):
    x = _rand(shape, np.float32)
    got = ski.feature.hessian_matrix(dev(x), sigma, mode="reflect", use_gaussian_derivatives=True)
    exp = R.hessian_matrix_gaussian(x, sigma, mode="reflect")
    for g, e in zip(got, exp):
        np.testing.assert_array_equal(host(g), e)


def test_hessian_fd_known_answer(ski):
    sq = np.zeros((5, 5), np.float32)
    sq[2, 2] = 4
    got = ski.feature.hessian_matrix(dev(sq), sigma=0.1, use_gaussian_derivatives=False)
    exp = R.hessian_matrix_fd(sq, sigma=0.1)
    for g, e in zip(got, exp):
        np.testing.assert_array_equal(host(g), e)
    ev = host(ski.feature.hessian_matrix_eigvals(got))
    np.testing.assert_allclose(ev, R.eigvals_sym(exp), atol=1e-6)


@pytest.mark.parametrize("n", [3, 6])
@pytest.mark.parametrize("sort,abs_sort", [("ascending", True), ("descending", False),
                                           ("ascending", False), ("descending", True)])
def test_eigvals(ski, n, sort, abs_sort):
    from cucim_b200.skimage.feature import symmetric_compute_eigenvalues

    H = [_rand((40, 50), np.float32, seed=i) for i in range(n)]
    got = host(symmetric_compute_eigenvalues([dev(h) for h in H], sort=sort, abs_sort=abs_sort))
    exp = R.eigvals_sym(H, sort=sort, abs_sort=abs_sort)
    np.testing.assert_allclose(got, exp, rtol=2e-6, atol=2e-6)


@pytest.mark.parametrize("shape,black", [((40, 44), True), ((18, 20, 22), False)])
def test_frangi(ski, shape, black):
    """Bit-identical wherever the output is at least 1e-3 of its maximum,
    within 1e-9 of the maximum elsewhere (see tests/test_gpu_ridges.py)."""
    x = _rand(shape, np.float32)
    got = host(ski.filters.frangi(dev(x), sigmas=[1, 2], black_ridges=black))
    exp = R.frangi(x, sigmas=[1, 2], black_ridges=black)
    big = np.abs(exp) >= 1e-3 * np.abs(exp).max()
    np.testing.assert_array_equal(got[big], exp[big])
    assert np.abs(got.astype(np.float64) - exp).max() <= 1e-9 * np.abs(exp).max()


@pytest.mark.parametrize("dtype", [np.uint8, np.float32, np.float64])
def test_rgb2gray(ski, dtype):
    """Bit for bit: the oracle evaluates the kernel's expression with the
    CUDA compiler's contraction (oracle/cimx_oracle.c)."""
    rgb = np.random.default_rng(0).integers(0, 256, (257, 301, 3)).astype(np.uint8)
    if dtype != np.uint8:
        rgb = (rgb / 255 + np.random.default_rng(1).random(rgb.shape) * 1e-3).astype(dtype)
    got = host(ski.color.rgb2gray(dev(rgb)))
    exp = R.rgb2gray(rgb)
    assert got.dtype == exp.dtype
    np.testing.assert_array_equal(got, exp)
