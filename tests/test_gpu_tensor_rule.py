"""Which passes algorithm="tensor" sends to the tensor cores by default:
only those along lines of at least 2048 samples (where the tensor-core
kernels measured faster). Shorter lines run the plain kernels, so the result
equals the plain float32 chain bit for bit; longer lines take the TF32x3
path, close to but not identical with it."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def test_short_lines_stay_plain(ndi):
    x = torch.as_tensor(np.random.default_rng(1).random((24, 256, 256), dtype=np.float32)).cuda()
    plain = ndi.gaussian_filter(x, 4.0)
    assert torch.equal(ndi.gaussian_filter(x, 4.0, algorithm="tensor"), plain)
    with ndi.tensor_cores_everywhere():
        forced = ndi.gaussian_filter(x, 4.0, algorithm="tensor")
    assert not torch.equal(forced, plain)
    assert float((forced - plain).abs().max()) < 1e-5


def test_long_lines_use_tensor_cores(ndi):
    x = torch.as_tensor(np.random.default_rng(2).random((64, 4096), dtype=np.float32)).cuda()
    plain = ndi.gaussian_filter1d(x, 16.0, axis=1)
    tensor = ndi.gaussian_filter1d(x, 16.0, axis=1, algorithm="tensor")
    assert not torch.equal(tensor, plain)
    assert float((tensor - plain).abs().max()) < 1e-5
