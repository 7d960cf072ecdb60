"""The split-precision tensor-core path (algorithm="tensor"): BF16x3 banded
Toeplitz products on tcgen05 with float32 accumulation. Not bit-identical to
the float32 chain; checked against scipy.ndimage in float64 with the error
bound written below (relative to the largest output magnitude)."""

import numpy as np
import pytest
import scipy.ndimage as sndi
import torch

pytestmark = pytest.mark.gpu

# max |tensor - float64| / max |float64|
REL_BOUND = 2e-5
MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def _check(got, ref):
    err = np.abs(got.astype(np.float64) - ref)
    scale = max(np.abs(ref).max(), 1e-30)
    assert np.isfinite(got).all()
    assert err.max() / scale < REL_BOUND, (err.max() / scale, err.mean() / scale)


@pytest.mark.parametrize("shape", [(300, 257), (128, 64), (1, 700), (700, 3), (5, 130, 90)])
@pytest.mark.parametrize("sigma", [4.0, 16.0])
@pytest.mark.parametrize("mode", MODES)
def test_tensor_gaussian(ndi, shape, sigma, mode):
    x = np.random.default_rng(2).random(shape, dtype=np.float32)
    got = ndi.gaussian_filter(dev(x), sigma, mode=mode, cval=0.5, algorithm="tensor")
    ref = sndi.gaussian_filter(x.astype(np.float64), sigma, mode=mode, cval=0.5)
    _check(got.cpu().numpy(), ref)


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("K", [16, 63, 257, 385])
def test_tensor_correlate_axes(ndi, axis, K):
    x = np.random.default_rng(K).standard_normal((517, 333)).astype(np.float32)
    w = np.random.default_rng(K + 1).random(K).astype(np.float32)
    got = ndi.correlate1d(dev(x), w, axis, mode="nearest", algorithm="tensor")
    ref = sndi.correlate1d(x.astype(np.float64), w.astype(np.float64), axis, mode="nearest")
    _check(got.cpu().numpy(), ref)


def test_tensor_uniform_and_derivative(ndi):
    x = np.random.default_rng(3).random((400, 380), dtype=np.float32)
    got = ndi.uniform_filter(dev(x), 63, mode="nearest", algorithm="tensor")
    _check(got.cpu().numpy(), sndi.uniform_filter(x.astype(np.float64), 63, mode="nearest"))
    got = ndi.gaussian_filter(dev(x), 6.0, order=1, algorithm="tensor")
    _check(got.cpu().numpy(), sndi.gaussian_filter(x.astype(np.float64), 6.0, order=1))
