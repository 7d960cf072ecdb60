"""Many uneven tiles in one launch: rgb2gray -> gaussian(sigma per tile) ->
sobel magnitude, the pipeline a whole-slide tile loader feeds (an addition of
this library; cuCIM runs `color.rgb2gray`, `filters.gaussian` and
`filters.sobel` once per tile).

    batch = TileBatch(rgb_tiles, sigmas)     # prepares the device tables once
    batch.run()                              # one persistent launch
    g = batch.graph(); g.replay()            # the same launch in a CUDA graph
    batch.outputs                            # float32 tiles, bit-identical to
                                             # sobel(gaussian(rgb2gray(t), s))

Each tile is an (H, W, 3) uint8 CUDA tensor whose pixels are contiguous
within a row (a C-contiguous tile, or a region view of a larger slide: rows
may be any pitch apart); its output is (H, W) float32 (C-contiguous or a
region view). `TileBatch.from_regions(slide, regions, sigmas)` builds the
batch straight from regions of a whole-slide image held on the device, the
way a slide reader's read_region results feed it, without copying tiles.
The gaussian uses mode 'nearest' and truncate 4 (the defaults of
`skimage.filters.gaussian`), the sobel mode 'reflect'; every tile is
filtered as an image of its own, exactly as the per-tile calls would.
"""

import ctypes
import math

import numpy as np

from . import _arrays, _lib
from .ndimage import _gaussian_kernel1d

BLOCK = 64
MAX_TAPS = 129


def sobel_taps(ndim=2):
    """Correlation taps of the sobel magnitude passes for float32 images:
    the edge taps [1, 0, -1] / sqrt(ndim) and the smoothing taps
    [1, 2, 1] / 4, rounded as filters/edges.py:148-241 rounds them, reversed
    by the convolution."""
    ew = np.asarray([1, 0, -1], dtype=np.float32)
    ew = (ew / np.float32(math.sqrt(ndim))).astype(np.float32)
    sw = np.asarray(np.array([1, 2, 1]) / 4, dtype=np.float32)
    return np.ascontiguousarray(ew[::-1]), np.ascontiguousarray(sw[::-1])


def gaussian_taps(sigma, truncate=4.0):
    """float32 taps of skimage.filters.gaussian for one sigma."""
    r = int(float(truncate) * float(sigma) + 0.5)
    if r <= 0:
        return np.ones(1, dtype=np.float32)
    return np.asarray(_gaussian_kernel1d(float(sigma), 0, r), dtype=np.float32)


class TileBatch:
    """Device tables for one batch of tiles and the launch over them."""

    def __init__(self, rgb_tiles, sigmas, outputs=None, truncate=4.0):
        import torch

        if len(rgb_tiles) != len(sigmas):
            raise ValueError("one sigma per tile")
        self.device = rgb_tiles[0].device if rgb_tiles else torch.device("cuda")
        self.tiles = [_arrays.as_tensor(t) for t in rgb_tiles]
        for t in self.tiles:
            if (t.dtype != torch.uint8 or t.dim() != 3 or t.shape[-1] != 3
                    or t.stride(2) != 1 or t.stride(1) != 3 or t.stride(0) < 3 * t.shape[1]):
                raise ValueError("tiles must be (H, W, 3) uint8 CUDA tensors with contiguous "
                                 "pixels in each row")
        if outputs is None:
            outputs = [torch.empty(t.shape[:2], dtype=torch.float32, device=t.device)
                       for t in self.tiles]
        self.outputs = outputs
        cache, taps, offsets, ntaps = {}, [], [], []
        pos = 0
        for s in sigmas:
            key = float(s)
            if key not in cache:
                w = gaussian_taps(key, truncate)
                if w.size > MAX_TAPS:
                    raise ValueError(f"sigma {s}: {w.size} taps, at most {MAX_TAPS}")
                cache[key] = (pos, w)
                taps.append(w)
                pos += w.size
            off, w = cache[key]
            offsets.append(off)
            ntaps.append(w.size)
        self.max_taps = max(ntaps) if ntaps else 1
        self.taps = torch.as_tensor(np.concatenate(taps) if taps else np.ones(1, np.float32),
                                    device=self.device)
        table = (_lib.CimxBatchTile * max(1, len(self.tiles)))()
        first = 0
        for i, (t, o) in enumerate(zip(self.tiles, outputs)):
            h, w = int(t.shape[0]), int(t.shape[1])
            if (tuple(o.shape) != (h, w) or o.dtype != torch.float32 or o.stride(1) != 1
                    or o.stride(0) < w):
                raise ValueError("outputs must be (H, W) float32 tensors with contiguous rows")
            table[i] = _lib.CimxBatchTile(t.data_ptr(), o.data_ptr(), h, w, ntaps[i], offsets[i],
                                          first, t.stride(0), o.stride(0))
            first += ((h + BLOCK - 1) // BLOCK) * ((w + BLOCK - 1) // BLOCK)
        self.nblocks = first
        raw = np.frombuffer(bytes(table), dtype=np.uint8).copy()
        self.table = torch.as_tensor(raw, device=self.device)
        ew, sw = sobel_taps(2)
        self._edge = (ctypes.c_float * 3)(*ew.tolist())
        self._smooth = (ctypes.c_float * 3)(*sw.tolist())
        self.npixels = sum(int(t.shape[0]) * int(t.shape[1]) for t in self.tiles)

    @classmethod
    def from_regions(cls, slide, regions, sigmas, out_slide=None, truncate=4.0):
        """A batch over regions (y, x, height, width) of one (H, W, 3) uint8
        slide on the device: the tiles are views into the slide (no copies).
        With `out_slide` ((H, W) float32), each region's result is written
        into the same region of it (regions must then not overlap); else
        every region gets its own (height, width) output."""
        import torch

        s = _arrays.as_tensor(slide)
        if s.dim() != 3 or s.shape[-1] != 3 or s.dtype != torch.uint8:
            raise ValueError("the slide must be an (H, W, 3) uint8 array")
        H, W = int(s.shape[0]), int(s.shape[1])
        tiles, outs = [], None if out_slide is None else []
        o_all = None if out_slide is None else _arrays.as_tensor(out_slide)
        if o_all is not None and tuple(o_all.shape) != (H, W):
            raise ValueError("out_slide must have the slide's (H, W) shape")
        for (y, x, h, w) in regions:
            if not (0 <= y and 0 <= x and h >= 1 and w >= 1 and y + h <= H and x + w <= W):
                raise ValueError(f"region {(y, x, h, w)} is outside the {H} x {W} slide")
            tiles.append(s[y:y + h, x:x + w])
            if o_all is not None:
                outs.append(o_all[y:y + h, x:x + w])
        return cls(tiles, sigmas, outputs=outs, truncate=truncate)

    def run(self, stream=None):
        import torch

        st = torch.cuda.current_stream(self.device).cuda_stream if stream is None else stream
        rc = _lib.lib.cimx_batch_gray_gauss_sobel(
            self.table.data_ptr(), len(self.tiles), self.nblocks, self.taps.data_ptr(),
            self.max_taps, self._edge, self._smooth, ctypes.c_void_p(st))
        _lib.check(rc, "batched tiles")
        return self.outputs

    def graph(self):
        """A CUDA graph holding the launch (replay() re-runs the batch)."""
        import torch

        self.run()  # first call outside capture (function attributes, module load)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run()
        return g


def gray_gauss_sobel_per_tile(rgb_tiles, sigmas, outputs=None):
    """The same pipeline as three public calls per tile (the unbatched
    path)."""
    from .skimage import color, filters

    outs = []
    for i, (t, s) in enumerate(zip(rgb_tiles, sigmas)):
        g = filters.gaussian(color.rgb2gray(t), sigma=float(s))
        o = filters.sobel(g)
        if outputs is not None:
            outputs[i].copy_(o)
            o = outputs[i]
        outs.append(o)
    return outs
