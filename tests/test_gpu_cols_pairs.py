"""GPU parity of the column-pair pass (float32 input along a strided axis of
lines longer than 64 samples): bit for bit against the oracle at the tile
edges (lines of 65, 128, 129 and 257 samples), with an odd number of
columns (the last pair has one column), two columns, several outer slabs,
every boundary mode, integer and float64 outputs, and zero taps inside the
kernel with inf and nan in the input."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def _run(ndi, x, w, axis, **kw):
    xd = torch.as_tensor(np.ascontiguousarray(x)).cuda()
    got = ndi.correlate1d(xd, w, axis, **kw).cpu().numpy()
    exp = R.correlate1d(x, w, axis, **kw)
    assert got.dtype == exp.dtype
    np.testing.assert_array_equal(got, exp, err_msg=f"axis={axis} {kw}")


@pytest.mark.parametrize("shape", [(65, 33), (128, 2), (129, 35), (257, 31), (3, 200, 9)])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K", [23, 57, 143])
def test_cols_pairs_modes(ndi, shape, mode, K):
    rng = np.random.default_rng(K + len(shape))
    x = rng.standard_normal(shape).astype(np.float32)
    w = rng.standard_normal(K).astype(np.float32)
    axis = len(shape) - 2
    for origin in (0, -(K // 2), K // 2):
        _run(ndi, x, w, axis, mode=mode, cval=0.75, origin=origin)


@pytest.mark.parametrize("output", [np.float64, np.uint16, np.int16, np.uint8])
def test_cols_pairs_output_dtypes(ndi, output):
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((300, 41)) * 40 + 60).astype(np.float32)
    w = rng.random(29).astype(np.float32) / 10
    _run(ndi, x, w, 0, output=output, mode="reflect")


def test_cols_pairs_zero_taps_and_nonfinite(ndi):
    x = np.random.default_rng(9).standard_normal((200, 3, 37)).astype(np.float32)
    x[50, 1, 7] = np.inf
    x[120, 2, 36] = np.nan
    w = np.random.default_rng(10).standard_normal(31).astype(np.float32)
    w[[3, 15, 16, 28]] = 0
    _run(ndi, x, w, 0, mode="mirror")


def test_cols_pairs_matches_single_columns(ndi):
    """The same pass with the line stored as the last axis (row kernel)
    gives the transposed result."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((400, 64)).astype(np.float32)
    w = rng.standard_normal(47).astype(np.float32)
    xd = torch.as_tensor(x).cuda()
    a = ndi.correlate1d(xd, w, 0, mode="nearest").cpu().numpy()
    b = ndi.correlate1d(xd.T.contiguous(), w, 1, mode="nearest").cpu().numpy().T
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dtype", [np.uint16, np.uint8])
@pytest.mark.parametrize("shape", [(65, 33), (129, 35), (3, 200, 9)])
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("K", [23, 57])
def test_cols_pairs_integer_input(ndi, dtype, shape, mode, K):
    """uint16 / uint8 input on the same lines (the typed column kernel),
    with the input dtype and float32 as outputs and a fill value that does
    not fit the input dtype."""
    rng = np.random.default_rng(K + len(shape) + 7)
    hi = np.iinfo(dtype).max
    x = rng.integers(0, hi + 1, shape).astype(dtype)
    w = rng.standard_normal(K).astype(np.float32) / 8
    axis = len(shape) - 2
    for output in (dtype, np.float32):
        for origin in (0, K // 2):
            _run(ndi, x, w, axis, mode=mode, cval=-3.25, origin=origin, output=output)
