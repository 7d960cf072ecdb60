"""skimage edge filters on the GPU path against the oracle, bit for bit:
sobel, scharr, prewitt and farid (magnitude and per axis, 2-D and 3-D), the
2-D _h / _v variants, and the `mask=` argument (the mask eroded with the
full-connectivity footprint, border value 0, multiplying the result;
filters/edges.py:75-85) with bool, integer and float masks, including masks
that touch the border and the known answer of cuCIM's test_edges.py:88-107
masked case (only the interior of an eroded square survives)."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

FILTERS = {"sobel": R.sk_sobel, "scharr": R.sk_scharr, "prewitt": R.sk_prewitt,
           "farid": R.sk_farid}


@pytest.fixture(scope="module")
def filters(cuda):
    from cucim_b200.skimage import filters as f

    return f


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def _mask(shape, kind, seed):
    rng = np.random.default_rng(seed)
    m = np.zeros(shape, bool)
    sl = tuple(slice(1, n - 2) for n in shape)
    m[sl] = True
    m &= rng.random(shape) > 0.05
    m[(0,) * len(shape)] = True  # a border element: eroded away
    if kind == "bool":
        return m
    if kind == "uint8":
        return (m * rng.integers(1, 200, shape)).astype(np.uint8)
    return np.where(m, rng.random(shape) + 0.5, 0.0).astype(np.float32)


@pytest.mark.parametrize("name", sorted(FILTERS))
@pytest.mark.parametrize("shape", [(47, 53), (9, 21, 26)])
@pytest.mark.parametrize("axis", [None, 0, -1])
@pytest.mark.parametrize("mask_kind", [None, "bool", "uint8", "float32"])
def test_edge_filters_with_masks(filters, name, shape, axis, mask_kind):
    x = np.random.default_rng(1).random(shape).astype(np.float32)
    mask = None if mask_kind is None else _mask(shape, mask_kind, 2)
    got = host(getattr(filters, name)(dev(x), None if mask is None else dev(mask), axis=axis))
    exp = FILTERS[name](x, mask, axis=axis)
    assert got.dtype == exp.dtype
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float64])
def test_edge_filters_dtypes(filters, dtype):
    x = (np.random.default_rng(3).random((40, 44)) * 200).astype(dtype)
    m = _mask(x.shape, "bool", 4)
    for name, ref in FILTERS.items():
        got = host(getattr(filters, name)(dev(x), dev(m)))
        np.testing.assert_array_equal(got, ref(x, m))


@pytest.mark.parametrize("base", ["sobel", "scharr", "prewitt"])
def test_h_v_variants(filters, base):
    x = np.random.default_rng(5).random((30, 34)).astype(np.float32)
    m = _mask(x.shape, "bool", 6)
    for suffix, axis in (("_h", 0), ("_v", 1)):
        got = host(getattr(filters, base + suffix)(dev(x), dev(m)))
        np.testing.assert_array_equal(got, FILTERS[base](x, m, axis=axis))
    got = host(filters.farid_h(dev(x), mask=dev(m)))
    np.testing.assert_array_equal(got, R.sk_farid(x, m, axis=0))
    with pytest.raises(ValueError):
        getattr(filters, base + "_h")(dev(np.zeros((3, 4, 5), np.float32)))


def test_mask_known_answer(filters):
    """test_edges.py:88-107 style: a vertical step image and a square mask;
    outside the eroded square the result is exactly zero, inside it equals
    the unmasked result."""
    image = np.zeros((12, 12), np.float32)
    image[:, 6:] = 1
    mask = np.zeros((12, 12), bool)
    mask[2:10, 2:10] = True
    got = host(filters.sobel(dev(image), dev(mask)))
    free = host(filters.sobel(dev(image)))
    inner = np.zeros_like(mask)
    inner[3:9, 3:9] = True
    np.testing.assert_array_equal(got[~inner], 0)
    np.testing.assert_array_equal(got[inner], free[inner])
    assert got[inner].max() > 0


def test_mask_shape_mismatch(filters):
    with pytest.raises(ValueError):
        filters.sobel(dev(np.zeros((8, 9), np.float32)), dev(np.ones((8, 8), bool)))
