"""The oracle pinned against cuCIM's own known answers and against
scipy.ndimage in float64 (CPU only)."""

import json
import os

import numpy as np
import pytest
import scipy.ndimage as sndi

from oracle import restate as R

HERE = os.path.dirname(os.path.abspath(__file__))
KA = json.load(open(os.path.join(HERE, "golden", "known_answers.json")))

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


# ------------------------------------------------------ cuCIM known answers

def test_gaussian_docstring_values():
    """_shared/filters.py:100-117: 3x3 delta at sigma 0.4 / 1 (nearest) and
    sigma 1 (reflect), float64."""
    delta, s04, s1, s1r = [np.array(a) for a in KA["gaussian_delta_docstring"]["arrays"]]
    np.testing.assert_array_almost_equal(R.sk_gaussian(delta, sigma=0.4), s04, decimal=8)
    np.testing.assert_array_almost_equal(R.sk_gaussian(delta, sigma=1), s1, decimal=8)
    np.testing.assert_array_almost_equal(R.sk_gaussian(delta, sigma=1, mode="reflect"), s1r,
                                         decimal=8)


@pytest.mark.parametrize("dtype", [np.float16, np.float32, np.float64])
def test_hessian_matrix_5x5(dtype):
    """feature/tests/test_corner.py:136-170."""
    sq = np.zeros((5, 5), dtype=dtype)
    sq[2, 2] = 4
    H = R.hessian_matrix_fd(sq, sigma=0.1, order="rc")
    exp = [np.array(a) for a in KA["hessian_5x5_fd"]["arrays"]]
    assert all(h.dtype == R.supported_float_type(dtype) for h in H)
    for h, e in zip(H, exp):
        np.testing.assert_array_almost_equal(h, e)


def test_hessian_matrix_3d_slice():
    """feature/tests/test_corner.py:195-213."""
    cube = np.zeros((5, 5, 5))
    cube[2, 2, 2] = 4
    Hs = R.hessian_matrix_fd(cube, sigma=0.1, order="rc")
    assert len(Hs) == 6
    np.testing.assert_array_almost_equal(Hs[2][:, 2, :],
                                         np.array(KA["hessian_3d_fd_slice"]["arrays"][0]))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_hessian_eigvals_5x5(dtype):
    """feature/tests/test_corner.py:284-307."""
    sq = np.zeros((5, 5), dtype=dtype)
    sq[2, 2] = 4
    H = R.hessian_matrix_fd(sq, sigma=0.1, order="rc")
    l1, l2 = R.eigvals_sym(H)
    e1, e2 = [np.array(a) for a in KA["hessian_eigvals_5x5_fd"]["arrays"]]
    np.testing.assert_array_almost_equal(l1, e1)
    np.testing.assert_array_almost_equal(l2, e2)


def test_hessian_order_xy_is_reversed():
    """feature/tests/test_corner.py:171-192 (gaussian-derivative branch)."""
    sq = np.zeros((5, 5))
    sq[2, 2] = 4
    hxx, hxy, hyy = R.hessian_matrix_gaussian(sq, sigma=0.1, order="xy")
    hrr, hrc, hcc = R.hessian_matrix_gaussian(sq, sigma=0.1, order="rc")
    np.testing.assert_allclose(hxx, hcc, atol=1e-30)
    np.testing.assert_allclose(hxy, hrc, atol=1e-30)
    np.testing.assert_allclose(hyy, hrr, atol=1e-30)


def test_sobel_horizontal_vertical_edges():
    """filters/tests/test_edges.py:88-107."""
    i, j = np.mgrid[-5:6, -5:6]
    img = (i >= 0).astype(float)
    r = R.sk_sobel(img) * np.sqrt(2)
    np.testing.assert_allclose(r[i == 0], 1)
    np.testing.assert_allclose(r[np.abs(i) > 1], 0)
    img = (j >= 0).astype(float)
    r = R.sk_sobel(img) * np.sqrt(2)
    np.testing.assert_allclose(r[j == 0], 1)
    assert np.all(r[np.abs(j) > 1] == 0)


def test_eig33_matches_eigvalsh():
    """feature/tests/test_corner.py:345-356 (closed form vs eigvalsh)."""
    rng = np.random.default_rng(5)
    H = [rng.normal(size=(8, 16, 24)) for _ in range(6)]
    ev = R.eigvals_sym(H)  # descending
    a, d, f, b, e, c = H
    M = np.stack([np.stack([a, d, f], -1), np.stack([d, b, e], -1), np.stack([f, e, c], -1)], -2)
    ref = np.linalg.eigvalsh(M)[..., ::-1]
    np.testing.assert_allclose(np.moveaxis(ref, -1, 0), ev, atol=1e-10)


def test_eig33_abs_sort_keeps_original_magnitudes():
    """corner.py:607-629: with abs_sort the magnitudes are read before the
    swaps and not updated. diag(-3, 1, -2): the closed form yields
    (min, max, mid) = (-3, 1, -2) with magnitudes (3, 1, 2); the three steps
    leave (-2, -3, 1), which is not sorted by magnitude."""
    Hd = [np.array([v]) for v in (-3.0, 0.0, 0.0, 1.0, 0.0, -2.0)]
    ev = R.eigvals_sym(Hd, sort="ascending", abs_sort=True)
    np.testing.assert_allclose(ev[:, 0], [-2.0, -3.0, 1.0], atol=1e-12)


# --------------------------------------------------- float64 vs scipy

@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", [(64, 57), (7, 5, 9), (1, 1), (5, 500), (300, 5)])
def test_gaussian_vs_scipy_f64(mode, shape):
    x = np.random.default_rng(123).standard_normal(shape)
    a = R.gaussian_filter(x, 2.3, mode=mode, cval=0.7)
    b = sndi.gaussian_filter(x, 2.3, mode=mode, cval=0.7)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_gaussian_derivative_vs_scipy_f64(mode, order):
    x = np.random.default_rng(1).standard_normal((40, 33))
    a = R.gaussian_filter(x, (1.5, 0.8), order=order, mode=mode)
    b = sndi.gaussian_filter(x, (1.5, 0.8), order=order, mode=mode)
    np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("size", [1, 2, 3, 4, 7, 20])
@pytest.mark.parametrize("origin", [-1, 0, 1])
def test_uniform_vs_scipy_f64(mode, size, origin):
    x = np.random.default_rng(7).standard_normal((23, 31))
    if size > 1 and (size // 2 + origin < 0 or size // 2 + origin >= size):
        with pytest.raises(ValueError):
            R.uniform_filter(x, size, mode=mode, origin=origin)
        return
    a = R.uniform_filter(x, size, mode=mode, origin=origin)
    if size == 1:  # the axis is skipped (weights None), origin never checked
        np.testing.assert_array_equal(a, x)
        return
    b = sndi.uniform_filter(x, size, mode=mode, origin=origin)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K", [1, 2, 5, 16, 31])
@pytest.mark.parametrize("convolve", [False, True])
def test_correlate1d_vs_scipy_f64(mode, K, convolve):
    rng = np.random.default_rng(K)
    x = rng.standard_normal((9, 12, 10))
    w = rng.standard_normal(K)
    origin = -(K // 2) if K > 1 else 0
    for axis in range(3):
        if convolve:
            a = R.convolve1d(x, w, axis, mode=mode, origin=origin)
            b = sndi.convolve1d(x, w, axis, mode=mode, origin=origin)
        else:
            a = R.correlate1d(x, w, axis, mode=mode, origin=origin)
            b = sndi.correlate1d(x, w, axis, mode=mode, origin=origin)
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("wkind", ["real", "complex"])
@pytest.mark.parametrize("convolve", [False, True])
def test_complex_correlate1d_vs_scipy_c128(mode, wkind, convolve):
    """The complex restatement (complex128: W = complex<double>) against
    scipy's complex correlate1d, including correlate's conjugated weights,
    convolve's flip and K > n."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((7, 9, 11)) + 1j * rng.standard_normal((7, 9, 11))
    w = rng.standard_normal(13)
    if wkind == "complex":
        w = w + 1j * rng.standard_normal(13)
    f, g = (R.convolve1d, sndi.convolve1d) if convolve else (R.correlate1d, sndi.correlate1d)
    for axis in range(3):
        a = f(x, w, axis, mode=mode, cval=-0.5, origin=1)
        b = g(x, w, axis, mode=mode, cval=-0.5, origin=1)
        assert a.dtype == np.complex128
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_complex_real_input_complex_weights_vs_scipy():
    rng = np.random.default_rng(12)
    x = rng.standard_normal((20, 30)).astype(np.float32)
    w = np.array([0.2 + 0.1j, 0.5 - 0.3j, 0.1 + 0.05j])
    a = R.correlate1d(x, w, 1)
    assert a.dtype == np.complex64
    np.testing.assert_allclose(a, sndi.correlate1d(x.astype(np.float64), w, 1), rtol=0,
                               atol=4e-7)


@pytest.mark.parametrize("mode", MODES)
def test_kernel_longer_than_axis_vs_scipy(mode):
    """Multi-period reflection when K > n (UTIL:186-308)."""
    x = np.random.default_rng(3).standard_normal((3, 4))
    w = np.random.default_rng(4).standard_normal(15)
    for axis in (0, 1):
        a = R.correlate1d(x, w, axis, mode=mode, cval=-1.5)
        b = sndi.correlate1d(x, w, axis, mode=mode, cval=-1.5)
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("func", ["sobel", "prewitt"])
@pytest.mark.parametrize("mode", MODES)
def test_sobel_prewitt_vs_scipy(func, mode):
    x = np.random.default_rng(9).standard_normal((17, 13, 11))
    for axis in range(3):
        a = getattr(R, func)(x, axis, mode=mode)
        b = getattr(sndi, func)(x, axis, mode=mode)
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_gaussian_gradient_magnitude_vs_scipy():
    x = np.random.default_rng(11).standard_normal((20, 30))
    a = R.gaussian_gradient_magnitude(x, 1.7)
    b = sndi.gaussian_gradient_magnitude(x, 1.7)
    np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-12)


def test_gaussian_taps_equal_scipy_weights():
    """_gaussian_kernel1d (FLT:689-717) reproduces scipy's weights exactly."""
    from scipy.ndimage._filters import _gaussian_kernel1d as sp_kernel

    for sigma in (0.5, 1.0, 2.0, 3.7, 16.0):
        for order in (0, 1, 2):
            r = int(4 * sigma + 0.5)
            a = R.gaussian_kernel1d(sigma, order, r)
            b = sp_kernel(sigma, order, r)
            if order == 0:
                np.testing.assert_array_equal(a, b)
            else:
                np.testing.assert_array_equal(a, b[::-1])


# ------------------------------------------------ exact float32 FMA chain

def _emulated_pass(x, taps32, axis, mode, cval32, origin=0):
    """Independent model of one float32 pass: the exact fused chain via
    float64 (exact for integer data of <= 16 bits)."""
    K = taps32.size
    anchor = K // 2 + origin
    pad_mode = {"reflect": "symmetric", "mirror": "reflect", "nearest": "edge",
                "wrap": "wrap", "constant": "constant"}[mode]
    pads = [(0, 0)] * x.ndim
    pads[axis] = (anchor, K - 1 - anchor)
    kw = {"constant_values": cval32} if mode == "constant" else {}
    xp = np.pad(x.astype(np.float64), pads, mode=pad_mode, **kw)
    s = np.zeros(x.shape, np.float32)
    n = x.shape[axis]
    for k in range(K):
        sl = [slice(None)] * x.ndim
        sl[axis] = slice(k, k + n)
        s = (xp[tuple(sl)] * np.float64(taps32[k]) + s.astype(np.float64)).astype(np.float32)
    return s


@pytest.mark.parametrize("mode", MODES)
def test_uint16_uniform_chain_is_exact(mode):
    """uint16 -> uint16 uniform_filter(size=5): per-axis exact chain and
    truncating cast, intermediates truncated to uint16 (CORE:124-163)."""
    x = np.random.default_rng(1).integers(0, 65536, (6, 9, 11)).astype(np.uint16)
    got = R.uniform_filter(x, 5, output=np.uint16, mode=mode, cval=3)
    taps = np.full(5, 1 / 5, np.float32)
    cur = x
    for ax in range(3):  # 3-D: elementwise kernel, fill value (float)cval
        s = _emulated_pass(cur, taps, ax, mode, np.float32(3))
        cur = s.astype(np.uint16)  # s >= 0, in range
    np.testing.assert_array_equal(got, cur)


def test_path_choice_rules():
    from oracle.restate import choose_path

    assert choose_path(2, 0, 33, 16, "reflect", 0.0, np.float32) == "shared_memory"
    assert choose_path(3, 0, 33, 16, "reflect", 0.0, np.float32) == "elementwise"
    assert choose_path(2, 0, 257, 128, "reflect", 0.0, np.float32) == "elementwise"
    assert choose_path(2, 0, 9, 4, "constant", -1.0, np.uint16) == "elementwise"
    assert choose_path(2, 0, 9, 4, "constant", -1.0, np.int16) == "shared_memory"
    assert choose_path(2, 0, 9, 4, "constant", np.nan, np.float32) == "elementwise"
    # float64 with a long kernel along axis 0 overflows the 48 KiB tile
    assert choose_path(2, 0, 201, 100, "reflect", 0.0, np.float64) == "elementwise"
    assert choose_path(2, 1, 201, 100, "reflect", 0.0, np.float64) == "shared_memory"


def test_cval_rounding_depends_on_path():
    """2-D: the shared-memory kernel rounds the fill value to the input type
    first (SEP:219-223); 3-D uses (W)cval (CORE:334-348)."""
    x2 = np.full((4, 4), 10, np.uint16)
    r2 = R.correlate1d(x2, np.array([1.0, 0, 0], np.float32), 0, output=np.float32,
                       mode="constant", cval=2.7)
    assert r2[0, 0] == 2.0
    x3 = np.full((2, 4, 4), 10, np.uint16)
    r3 = R.correlate1d(x3, np.array([1.0, 0, 0], np.float32), 1, output=np.float32,
                       mode="constant", cval=2.7)
    assert r3[0, 0, 0] == np.float32(2.7)


def test_cast_rule():
    """cast<D>() of CORE:227-244 with the GPU's saturating conversion."""
    v = np.array([-5.0, 70000.0, np.nan, 3.9, -0.5], np.float32)
    np.testing.assert_array_equal(R.cast_w(v, 0, np.uint16), [65531, 65535, 0, 3, 0])
    np.testing.assert_array_equal(R.cast_w(v, 0, np.int16), [-5, 32767, 0, 3, 0])
    np.testing.assert_array_equal(R.cast_w(np.array([300.0, -2.0], np.float32), 0, np.uint8),
                                  [44, 254])


def test_nonfinite_cval_integer_output_raises():
    x = np.zeros((3, 4, 5), np.uint8)
    with pytest.raises(NotImplementedError):
        R.correlate1d(x, np.ones(3), 0, mode="constant", cval=np.nan)


def test_rgb2gray_weights():
    rgb = np.random.default_rng(0).integers(0, 256, (5, 7, 3)).astype(np.uint8)
    g = R.rgb2gray(rgb)
    x = (rgb.astype(np.float32) * np.float32(1 / 255)).astype(np.float64)
    ref = 0.2125 * x[..., 0] + 0.7154 * x[..., 1] + 0.0721 * x[..., 2]
    np.testing.assert_allclose(g, ref.astype(np.float32), rtol=1e-7)


def test_frangi_small_oracle_properties():
    """filters/tests/test_ridges.py invariants on the oracle: null image gives
    zeros, output in [0, 1]."""
    z = np.zeros((12, 13))
    np.testing.assert_array_equal(R.frangi(z, sigmas=[1, 2]), 0)
    v = R.frangi(np.random.default_rng(2).random((20, 21)).astype(np.float32), sigmas=[1, 2])
    assert v.dtype == np.float32 and np.all((v >= 0) & (v <= 1))


@pytest.mark.parametrize("mode", ["reflect", "mirror", "nearest", "constant", "wrap"])
def test_laplace_family_matches_scipy_float64(mode):
    # the oracle's laplace and gaussian_laplace (FLT:806-1009) in float64
    # agree with scipy.ndimage up to the order of the final sums
    import scipy.ndimage as sndi

    x = np.random.default_rng(5).standard_normal((16, 21, 19))
    np.testing.assert_allclose(R.laplace(x, mode=mode, cval=0.5),
                               sndi.laplace(x, mode=mode, cval=0.5), rtol=0, atol=1e-12)
    np.testing.assert_allclose(R.gaussian_laplace(x, (1.5, 0.7, 2.0), mode=mode, cval=0.5),
                               sndi.gaussian_laplace(x, (1.5, 0.7, 2.0), mode=mode, cval=0.5),
                               rtol=0, atol=1e-12)


@pytest.mark.parametrize("mode", ["reflect", "mirror", "nearest", "constant", "wrap"])
def test_min_max_filter1d_matches_scipy(mode):
    # min / max are exact: the oracle's restatement of cuCIM's kernel (the
    # element itself, then the window folded with fmin / fmax in double)
    # agrees with scipy.ndimage bit for bit on finite data
    x = np.random.default_rng(6).standard_normal((7, 40, 33)).astype(np.float32)
    for axis in range(3):
        for size, origin in [(1, 0), (3, 0), (4, 1), (7, -2), (50, 3)]:
            for ours, ref in [(R.minimum_filter1d, sndi.minimum_filter1d),
                              (R.maximum_filter1d, sndi.maximum_filter1d)]:
                np.testing.assert_array_equal(
                    ours(x, size, axis, mode=mode, cval=0.25, origin=origin),
                    ref(x, size, axis, mode=mode, cval=0.25, origin=origin))
    xi = np.random.default_rng(7).integers(0, 255, (30, 50)).astype(np.uint8)
    np.testing.assert_array_equal(R.maximum_filter1d(xi, 5, 0, mode=mode, cval=17),
                                  sndi.maximum_filter1d(xi, 5, 0, mode=mode, cval=17))


def test_min_max_fold_is_minimum_number():
    """The oracle's min / max fold is IEEE 754-2019 minimumNumber /
    maximumNumber (CUDA's fmin / fmax on the GPU): nan ignored unless every
    value is nan, and -0 below +0 in either order. Windows of two along a
    length-2 axis, so both operand orders occur."""
    pz, nz, nan = 0.0, -0.0, np.nan
    x = np.array([[pz, nz], [nz, pz], [nan, 1.0], [1.0, nan], [nan, nan]], np.float64)
    mn = R.minimum_filter1d(x, 2, axis=1, mode="wrap")
    mx = R.maximum_filter1d(x, 2, axis=1, mode="wrap")
    assert np.all(np.signbit(mn[:2])) and not np.any(np.signbit(mx[:2]))
    assert np.array_equal(mn[2:4], [[1.0, 1.0], [1.0, 1.0]])
    assert np.array_equal(mx[2:4], [[1.0, 1.0], [1.0, 1.0]])
    assert np.all(np.isnan(mn[4])) and np.all(np.isnan(mx[4]))
