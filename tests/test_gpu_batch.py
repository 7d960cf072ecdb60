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


def test_batch_from_slide_regions(cuda):
    """Tiles taken as regions of one slide image on the device (views with
    the slide's row pitch, no copies), written into their own outputs and
    into the matching regions of a slide-sized output: bit-identical to the
    per-tile calls on copies of the regions."""
    from cucim_b200 import batch

    slide = _tiles([(700, 900)], 8)[0]
    regions = [(0, 0, 64, 64), (10, 600, 300, 299), (650, 850, 50, 50), (100, 0, 1, 900),
               (333, 444, 77, 3)]
    sigmas = [1.0, 3.3, 0.6, 2.0, 7.5]
    b = batch.TileBatch.from_regions(slide, regions, sigmas)
    got = b.run()
    copies = [slide[y:y + h, x:x + w].contiguous() for y, x, h, w in regions]
    ref = batch.gray_gauss_sobel_per_tile(copies, sigmas)
    torch.cuda.synchronize()
    for g, r in zip(got, ref):
        assert torch.equal(g, r)
    # into one slide-sized output (non-overlapping regions)
    out_slide = torch.full((700, 900), -1.0, device="cuda")
    regions2 = [(0, 0, 64, 64), (10, 600, 300, 299), (650, 850, 50, 50)]
    b2 = batch.TileBatch.from_regions(slide, regions2, sigmas[:3], out_slide=out_slide)
    b2.run()
    torch.cuda.synchronize()
    for (y, x, h, w), r in zip(regions2, ref[:3]):
        assert torch.equal(out_slide[y:y + h, x:x + w], r)
    untouched = torch.ones_like(out_slide, dtype=torch.bool)
    for y, x, h, w in regions2:
        untouched[y:y + h, x:x + w] = False
    assert bool((out_slide[untouched] == -1.0).all())
    with pytest.raises(ValueError):
        batch.TileBatch.from_regions(slide, [(690, 0, 20, 20)], [1.0])


def test_region_stream_from_host_slide(cuda):
    """Regions of a slide in host memory through RegionStream, in chunks small
    enough that both buffer sets are reused several times: bit-identical to
    TileBatch on the same slide held on the device, again on a second run,
    and to the oracle on a few regions."""
    from cucim_b200 import batch
    from oracle import restate as R

    rng = np.random.default_rng(11)
    slide = rng.integers(0, 256, (700, 900, 3), dtype=np.uint8)
    regions = [(int(rng.integers(0, 600)), int(rng.integers(0, 800)), int(rng.integers(1, 100)),
                int(rng.integers(1, 100))) for _ in range(40)] + [(0, 0, 700, 900), (3, 5, 1, 1)]
    sigmas = [float(v) for v in rng.uniform(0.5, 6.0, len(regions))]
    rs = batch.RegionStream.from_regions(slide, regions, sigmas, chunk_pixels=60_000)
    assert len(rs.chunks) > 3
    got = rs.run()
    ref = batch.TileBatch.from_regions(torch.as_tensor(slide).cuda(), regions, sigmas).run()
    assert len(got) == len(regions)
    for g, r in zip(got, ref):
        assert g.dtype == np.float32 and np.array_equal(g, r.cpu().numpy())
    again = rs.run()
    assert all(np.array_equal(a, b) for a, b in zip(got, again))
    for k in (0, 7, len(regions) - 2, len(regions) - 1):
        y, x, h, w = regions[k]
        exp = R.sk_sobel(R.sk_gaussian(R.rgb2gray(slide[y:y + h, x:x + w]), sigmas[k]))
        assert np.array_equal(got[k], exp), k


def test_region_stream_rejects_bad_input(cuda):
    from cucim_b200 import batch

    with pytest.raises(ValueError):
        batch.RegionStream([np.zeros((4, 4, 3), np.float32)], [1.0])
    with pytest.raises(ValueError):
        batch.RegionStream.from_regions(np.zeros((10, 10, 3), np.uint8), [(5, 5, 6, 2)], [1.0])
