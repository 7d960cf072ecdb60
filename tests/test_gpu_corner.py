"""structure_tensor, its eigenvalues and the corner measures on the GPU path
against the oracle.

structure_tensor is bit-exact (sobel passes, exactly rounded products,
gaussian passes). The corner responses evaluate cuCIM's kernel expressions,
which the CUDA compiler contracts into fused multiply-adds as NVRTC does for
cuCIM; the oracle evaluates them without contraction. Their difference is
bounded by a few float32 roundings of the terms that cancel (det = Arr*Acc -
Arc*Arc and the like), so each response is compared with a tolerance of
1e-6 times the magnitude of those terms."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def feature(cuda):
    from cucim_b200.skimage import feature as f

    return f


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def _square_image():
    img = np.zeros((40, 48), np.float32)
    img[10:30, 12:36] = 1
    return img + np.random.default_rng(0).random(img.shape).astype(np.float32) * 0.1


@pytest.mark.parametrize("shape,dtype", [((40, 48), np.float32), ((12, 14, 16), np.float32),
                                         ((30, 32), np.uint8), ((20, 22, 3), np.float32),
                                         ((24, 26), np.float64)])
@pytest.mark.parametrize("mode", ["constant", "reflect", "nearest"])
def test_structure_tensor(feature, shape, dtype, mode):
    x = (np.random.default_rng(1).random(shape) * 200).astype(dtype)
    got = feature.structure_tensor(dev(x), sigma=1.5, mode=mode)
    exp = R.structure_tensor(x, sigma=1.5, mode=mode)
    assert len(got) == len(exp)
    for g, e in zip(got, exp):
        np.testing.assert_array_equal(host(g), e)


def test_structure_tensor_order_and_sigma_checks(feature):
    x = _square_image()
    got = feature.structure_tensor(dev(x), sigma=(1.0, 2.0), order="xy")
    exp = R.structure_tensor(x, sigma=(1.0, 2.0), order="xy")
    for g, e in zip(got, exp):
        np.testing.assert_array_equal(host(g), e)
    with pytest.raises(ValueError):
        feature.structure_tensor(dev(np.zeros((4, 5, 6), np.float32)), order="xy")
    with pytest.raises(ValueError):
        feature.structure_tensor(dev(x), sigma=(1, 2, 3))


def test_structure_tensor_eigenvalues(feature):
    x = _square_image()
    A = feature.structure_tensor(dev(x), sigma=1.0)
    got = host(feature.structure_tensor_eigenvalues(A))
    exp = R.eigvals_sym(R.structure_tensor(x, sigma=1.0), sort="descending")
    np.testing.assert_array_equal(got, exp)


def _tol(terms):
    return 1e-6 * sum(np.abs(t.astype(np.float64)) for t in terms) + 1e-30


@pytest.mark.parametrize("method", ["k", "eps"])
def test_corner_harris(feature, method):
    x = _square_image()
    got = host(feature.corner_harris(dev(x), method=method, sigma=1.2))
    exp = R.corner_harris(x, method=method, sigma=1.2)
    Arr, Arc, Acc = R.structure_tensor(x, 1.2)
    tr = Arr.astype(np.float64) + Acc
    scale = Arr * Acc + Arc * Arc + 0.05 * tr * tr
    if method == "eps":
        scale = scale / np.abs(tr + 1e-6)
    assert np.all(np.abs(got - exp) <= _tol([scale]))
    assert got.dtype == np.float32


def test_corner_shi_tomasi_and_foerstner(feature):
    x = _square_image()
    Arr, Arc, Acc = R.structure_tensor(x, 1.0)
    got = host(feature.corner_shi_tomasi(dev(x), sigma=1.0))
    exp = R.corner_shi_tomasi(x, sigma=1.0)
    assert np.all(np.abs(got - exp) <= _tol([Arr, Acc, 2 * Arc]))
    w, q = feature.corner_foerstner(dev(x), sigma=1.0)
    ew, eq = R.corner_foerstner(x, sigma=1.0)
    tr = np.abs(Arr.astype(np.float64) + Acc) + 1e-30
    det_scale = np.abs(Arr * Acc.astype(np.float64)) + Arc.astype(np.float64) ** 2
    assert np.all(np.abs(host(w) - ew) <= _tol([det_scale / tr]))
    assert np.all(np.abs(host(q) - eq) <= _tol([4 * det_scale / tr ** 2]))


@pytest.mark.parametrize("mode", ["constant", "reflect"])
def test_corner_kitchen_rosenfeld(feature, mode):
    x = _square_image()
    got = host(feature.corner_kitchen_rosenfeld(dev(x), mode=mode))
    exp = R.corner_kitchen_rosenfeld(x, mode=mode)
    imy, imx = (R.sobel(x, i, mode=mode) for i in range(2))
    imxy, imxx = (R.sobel(imx, i, mode=mode) for i in range(2))
    imyy = R.sobel(imy, 0, mode=mode)
    den = imx.astype(np.float64) ** 2 + imy.astype(np.float64) ** 2
    num_scale = (np.abs(imxx * imy.astype(np.float64) ** 2) + np.abs(imyy * imx.astype(np.float64) ** 2)
                 + np.abs(2 * imxy * imx.astype(np.float64) * imy))
    bound = np.where(den > 0, _tol([num_scale]) / np.where(den > 0, den, 1), 0)
    assert np.all(np.abs(got.astype(np.float64) - exp) <= bound + 1e-6 * np.abs(exp))


def test_corner_known_answer(feature):
    """corner.py:1063-1100: the Harris peaks of a white square sit near its
    four corners."""
    sq = np.zeros((10, 10), np.float32)
    sq[2:8, 2:8] = 1
    r = host(feature.corner_harris(dev(sq)))
    exp = R.corner_harris(sq)
    assert np.all(np.abs(r - exp) <= 1e-6 * np.abs(exp).max())
    top = set(map(tuple, np.argwhere(r == r.max())))
    assert top <= {(2, 2), (2, 7), (7, 2), (7, 7), (3, 3), (3, 6), (6, 3), (6, 6)}
