"""The persistent warp-specialised slab kernel (k_slabw, float32 (y, x)
passes with up to 48 taps) against the one-tile-per-CTA slab kernel
(forced with CIMX_L_NO_SLABW) and the oracle, bit for bit: every mode,
tap counts up to 48, origins, zero taps skipped (derivative taps), shapes
that are not multiples of the 64 x 128 tile, slabs enough that each CTA
walks many tiles through both input stages, and a status word that shows
no bounded wait ran out."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


@pytest.fixture(scope="module")
def mods(cuda):
    from cucim_b200 import _lib
    from cucim_b200 import ndimage as ndi

    return ndi, _lib


def _f32(shape, seed):
    return np.random.default_rng(seed).random(shape, dtype=np.float32)


def _check(ndi, lib, x, call):
    xd = torch.as_tensor(x).cuda()
    lib.lib.cimx_device_status(1)
    got = call(ndi, xd).cpu().numpy()
    with ndi.schedule(lib.L_NO_SLABW):
        old = call(ndi, xd).cpu().numpy()
    exp = call(R, x)
    np.testing.assert_array_equal(got, old)
    np.testing.assert_array_equal(got, exp)
    assert lib.lib.cimx_device_status(0) == 0


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("sigma", [1.1, 2.0, 2.8, 4.0, 4.4, 5.5])  # 9 .. 45 taps
@pytest.mark.parametrize("shape", [(3, 130, 260), (1, 64, 128), (2, 67, 132), (5, 200, 36)])
def test_gaussian_yx(mods, mode, sigma, shape):
    ndi, lib = mods
    _check(ndi, lib, _f32(shape, 1),
           lambda f, x: f.gaussian_filter(x, sigma, mode=mode, cval=0.5, axes=(1, 2)))


@pytest.mark.parametrize("order", [(1, 0), (0, 1), (1, 1), (2, 0)])
def test_derivative_taps(mods, order):
    ndi, lib = mods
    # 3-D: the elementwise rule, zero taps skipped inside the chains
    _check(ndi, lib, _f32((4, 150, 140), 2),
           lambda f, x: f.gaussian_filter(x, [3.0, 2.5], order=list(order), axes=(1, 2)))


@pytest.mark.parametrize("size,origin", [((40, 33), (3, -5)), ((48, 8), (0, 2)), ((17, 46), (-2, 0))])
@pytest.mark.parametrize("mode", ["reflect", "constant", "wrap"])
def test_uniform_origins(mods, size, origin, mode):
    ndi, lib = mods
    _check(ndi, lib, _f32((3, 140, 300), 3),
           lambda f, x: f.uniform_filter(x, size, mode=mode, cval=2.0, origin=origin,
                                         axes=(1, 2)))


def test_many_tiles_per_cta(mods):
    ndi, lib = mods
    _check(ndi, lib, _f32((64, 256, 260), 4),
           lambda f, x: f.gaussian_filter(x, 4.0, mode="mirror", axes=(1, 2)))


def test_2d_and_tiny(mods):
    ndi, lib = mods
    for shape in [(2048, 2048), (1, 4), (5, 8), (64, 4), (300, 12)]:
        _check(ndi, lib, _f32(shape, 5), lambda f, x: f.gaussian_filter(x, 4.0, mode="reflect"))
