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
way a slide reader's read_region results feed it, without copying tiles;
`RegionStream` takes tiles (or slide regions) held in host memory through
the same launch chunk by chunk, its copies overlapped with the filtering.
The gaussian uses mode 'nearest' and truncate 4 (the defaults of
`skimage.filters.gaussian`), the sobel mode 'reflect'; every tile is
filtered as an image of its own, exactly as the per-tile calls would.
"""

import ctypes
import math
import os

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


class RegionStream:
    """Tiles held in host memory through the batched launch, with the copies
    overlapped: the ingest side of a whole-slide pipeline, where a reader
    (cuCIM's read_region, a TIFF decoder) leaves tiles in host memory.

        rs = RegionStream(host_tiles, sigmas)          # or .from_regions(host_slide, regions, sigmas)
        results = rs.run()                             # float32 numpy arrays, input order

    The tiles go in chunks of about `chunk_pixels` pixels through two sets
    of buffers: while chunk i is filtered, host threads gather chunk i + 1
    into pinned memory and its copy to the device runs on its own stream,
    and chunk i - 1's results come back on a third stream; events order the
    reuse of every buffer. Each chunk is one `TileBatch` launch (tables
    prepared once, here), so the results are bit-identical to `TileBatch`
    on the same tiles."""

    def __init__(self, host_tiles, sigmas, chunk_pixels=1 << 26, device=None, truncate=4.0,
                 threads=None):
        import torch

        if len(host_tiles) != len(sigmas):
            raise ValueError("one sigma per tile")
        self.device = torch.device("cuda") if device is None else torch.device(device)
        self.host = [np.asarray(t) for t in host_tiles]
        for t in self.host:
            if t.dtype != np.uint8 or t.ndim != 3 or t.shape[2] != 3 or 0 in t.shape:
                raise ValueError("tiles must be non-empty (H, W, 3) uint8 host arrays")
        self.sigmas = [float(v) for v in sigmas]
        self.threads = threads or min(16, os.cpu_count() or 1)
        # chunks of consecutive tiles, each at most chunk_pixels (or one tile)
        self.chunks, cur, npx = [], [], 0
        for i, t in enumerate(self.host):
            n = t.shape[0] * t.shape[1]
            if cur and npx + n > chunk_pixels:
                self.chunks.append(cur)
                cur, npx = [], 0
            cur.append(i)
            npx += n
        if cur:
            self.chunks.append(cur)
        cap = max((sum(self.host[i].shape[0] * self.host[i].shape[1] for i in c)
                   for c in self.chunks), default=1)
        dev = self.device
        self._pin_in = [torch.empty(3 * cap, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self._pin_out = [torch.empty(cap, dtype=torch.float32).pin_memory() for _ in range(2)]
        self._dev_in = [torch.empty(3 * cap, dtype=torch.uint8, device=dev) for _ in range(2)]
        self._dev_out = [torch.empty(cap, dtype=torch.float32, device=dev) for _ in range(2)]
        # per chunk: each tile's pixel offset and its batch over buffer set c % 2
        self._layout, self._batches = [], []
        for c, chunk in enumerate(self.chunks):
            offs, pos = [], 0
            for i in chunk:
                offs.append(pos)
                pos += self.host[i].shape[0] * self.host[i].shape[1]
            self._layout.append((offs, pos))
            din, dout = self._dev_in[c % 2], self._dev_out[c % 2]
            tiles, outs = [], []
            for i, o in zip(chunk, offs):
                h, w = self.host[i].shape[:2]
                tiles.append(din.narrow(0, 3 * o, 3 * h * w).view(h, w, 3))
                outs.append(dout.narrow(0, o, h * w).view(h, w))
            self._batches.append(TileBatch(tiles, [self.sigmas[i] for i in chunk], outputs=outs,
                                           truncate=truncate))
        self.npixels = sum(t.shape[0] * t.shape[1] for t in self.host)

    @classmethod
    def from_regions(cls, slide, regions, sigmas, **kw):
        """Regions (y, x, height, width) of one (H, W, 3) uint8 slide in host
        memory (views: a region is read once, by the gather of its chunk)."""
        s = np.asarray(slide)
        if s.ndim != 3 or s.shape[2] != 3 or s.dtype != np.uint8:
            raise ValueError("the slide must be an (H, W, 3) uint8 array")
        H, W = s.shape[:2]
        tiles = []
        for (y, x, h, w) in regions:
            if not (0 <= y and 0 <= x and h >= 1 and w >= 1 and y + h <= H and x + w <= W):
                raise ValueError(f"region {(y, x, h, w)} is outside the {H} x {W} slide")
            tiles.append(s[y:y + h, x:x + w])
        return cls(tiles, sigmas, **kw)

    def _gather(self, pool, c):
        """Chunk c's tiles into pinned buffer set c % 2 (host threads)."""
        offs, n = self._layout[c]
        buf = self._pin_in[c % 2].numpy()

        def one(k):
            t = self.host[self.chunks[c][k]]
            h, w = t.shape[:2]
            buf[3 * offs[k]:3 * (offs[k] + h * w)].reshape(h, w, 3)[...] = t
        list(pool.map(one, range(len(self.chunks[c]))))
        return n

    def _collect(self, pool, c, results):
        """Chunk c's results out of pinned buffer set c % 2 (after its copy),
        by host threads."""
        offs, _ = self._layout[c]
        buf = self._pin_out[c % 2].numpy()

        def one(k):
            i = self.chunks[c][k]
            h, w = self.host[i].shape[:2]
            results[i] = buf[offs[k]:offs[k] + h * w].reshape(h, w).copy()
        list(pool.map(one, range(len(self.chunks[c]))))

    def run(self):
        import concurrent.futures as cf

        import torch

        dev = self.device
        cs, ks, ds = (torch.cuda.Stream(dev) for _ in range(3))
        ev_h2d, ev_kernel, ev_d2h = [None, None], [None, None], [None, None]
        pending = [None, None]  # chunk whose results sit in (or are coming to) pinned set s
        results = [None] * len(self.host)
        with cf.ThreadPoolExecutor(self.threads) as pool:
            for c in range(len(self.chunks)):
                s = c % 2
                if ev_h2d[s] is not None:
                    ev_h2d[s].synchronize()  # pinned input set s is read by its copy
                n = self._gather(pool, c)
                with torch.cuda.stream(cs):
                    if ev_kernel[s] is not None:
                        cs.wait_event(ev_kernel[s])  # device input set s is read by its kernel
                    self._dev_in[s][:3 * n].copy_(self._pin_in[s][:3 * n], non_blocking=True)
                    ev_h2d[s] = torch.cuda.Event()
                    ev_h2d[s].record(cs)
                ks.wait_event(ev_h2d[s])
                if ev_d2h[s] is not None:
                    ks.wait_event(ev_d2h[s])  # device output set s is read by its copy back
                self._batches[c].run(stream=ks.cuda_stream)
                ev_kernel[s] = torch.cuda.Event()
                ev_kernel[s].record(ks)
                if pending[s] is not None:
                    ev_d2h[s].synchronize()  # pinned output set s: take the previous results
                    self._collect(pool, pending[s], results)
                with torch.cuda.stream(ds):
                    ds.wait_event(ev_kernel[s])
                    self._pin_out[s][:n].copy_(self._dev_out[s][:n], non_blocking=True)
                    ev_d2h[s] = torch.cuda.Event()
                    ev_d2h[s].record(ds)
                pending[s] = c
            for s in range(2):
                if pending[s] is not None:
                    ev_d2h[s].synchronize()
                    self._collect(pool, pending[s], results)
        return results


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
