"""Batched tiles (rgb2gray -> gaussian(sigma per tile) -> sobel magnitude in
one launch): bit-identical to the three per-tile calls, which the oracle
pins; also under CUDA graph replay."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _tiles(shapes, seed):
    rng = np.random.default_rng(seed)
    means = np.array([60.0, 150.0, 220.0])
    out = []
    for h, w in shapes:
        comp = rng.integers(0, 3, size=(h, w, 3))
        vals = np.clip(np.rint(rng.normal(means[comp], 20.0)), 0, 255).astype(np.uint8)
        out.append(torch.as_tensor(vals).cuda())
    return out


SHAPES = [(1, 1), (3, 70), (64, 64), (65, 129), (200, 37), (130, 130), (7, 300), (257, 66)]
SIGMAS = [0.5, 8.0, 1.0, 3.7, 2.2, 8.0, 0.8, 5.5]


def test_batch_matches_per_tile(cuda):
    from cucim_b200 import batch

    tiles = _tiles(SHAPES, 3)
    b = batch.TileBatch(tiles, SIGMAS)
    got = b.run()
    ref = batch.gray_gauss_sobel_per_tile(tiles, SIGMAS)
    torch.cuda.synchronize()
    for g, r, s in zip(got, ref, SHAPES):
        assert g.shape == r.shape == s
        assert torch.equal(g, r), (s, (g - r).abs().max().item())


def test_batch_graph_replay(cuda):
    from cucim_b200 import batch

    tiles = _tiles(SHAPES[:5], 4)
    b = batch.TileBatch(tiles, SIGMAS[:5])
    first = [o.clone() for o in b.run()]
    for o in b.outputs:
        o.zero_()
    g = b.graph()
    for o in b.outputs:
        o.zero_()
    g.replay()
    torch.cuda.synchronize()
    for a, o in zip(first, b.outputs):
        assert torch.equal(a, o)


def test_batch_one_tile_against_oracle(cuda):
    from cucim_b200 import batch
    from oracle import restate as R

    tiles = _tiles([(96, 70)], 5)
    b = batch.TileBatch(tiles, [2.5])
    got = b.run()[0].cpu().numpy()
    x = tiles[0].cpu().numpy()
    gray = R.rgb2gray(x)
    sm = R.sk_gaussian(gray, 2.5)
    ref = R.sk_sobel(sm)
    np.testing.assert_array_equal(got, ref)


def test_batch_rejects_long_filters(cuda):
    from cucim_b200 import batch

    tiles = _tiles([(16, 16)], 6)
    with pytest.raises(ValueError):
        batch.TileBatch(tiles, [20.0])  # 161 taps
