"""Seeded synthetic inputs for the filtering workloads.

No public dataset is involved; these generators produce images with the
shapes, dtypes and value distributions of the standard workloads:

- ``uniform_image``: float32 i.i.d. uniform [0, 1) (2-D gaussian workload);
- ``smooth_volume_u16``: uint16 stack made by smoothing normal noise
  (sigma 3), rescaling to [0, 65535] and adding Poisson shot noise;
- ``stack_noise`` / ``stack_shot`` / ``stack_window``: the same recipe drawn
  slice by slice (every z-slice has its own seeded generators and the
  rescaling is a fixed affine map), so that any z-window of the
  512 x 1024 x 1024 stack can be regenerated exactly on its own;
- ``rectangles_image``: float32 uniform [0, 1) plus axis-aligned rectangles
  of constant value in [0, 10) (large-kernel precision workload);
- ``rgb_tiles``: uint8 RGB tiles of random sizes with per-channel
  three-component Gaussian-mixture values, plus a sigma per tile;
- ``segments_volume``: float32 volume of random line segments with Gaussian
  cross-sections on N(0, 0.05) noise (vesselness workload).
"""

import math

import numpy as np


def uniform_image(shape=(2048, 2048), seed=0):
    return np.random.default_rng(seed).random(shape, dtype=np.float32)


def smooth_volume_u16(shape=(512, 1024, 1024), seed=1, smooth=None):
    """`smooth(x, sigma)` smooths a float32 array (default: scipy.ndimage,
    mode 'reflect'); pass the GPU filter for large volumes."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape, dtype=np.float32)
    if smooth is None:
        import scipy.ndimage as sndi  # noqa: PLC0415

        sm = sndi.gaussian_filter(noise, 3.0, mode="reflect")
    else:
        sm = np.asarray(smooth(noise, 3.0), dtype=np.float32)
    lo, hi = float(sm.min()), float(sm.max())
    scaled = (sm - lo) * (65535.0 / max(hi - lo, 1e-30))
    shot = rng.poisson(np.clip(scaled, 0, None).astype(np.float64))
    return np.clip(shot, 0, 65535).astype(np.uint16)


# ---------------------------------------------------------------- 3-D stack
#
# The stack is built slice by slice so that a CPU baseline can regenerate a
# z-window of it without making the whole volume: slice z's noise comes from
# default_rng([seed, 0, z]) and its shot noise from default_rng([seed, 1, z]).
# The smoothing (sigma 3, truncate 4, mode 'reflect', float32) is done by the
# caller's gaussian_filter: on the device for the whole stack, or by the
# oracle on a window with its z halo; both compute the same float32 chain, so
# the smoothed values, and the stack, are identical. Instead of the volume's
# min/max (which a window cannot know), the smoothed noise is mapped to
# [0, 65535] by the fixed affine map that sends -5 and +5 standard deviations
# to 0 and 65535 (values beyond are clipped: about 3e-7 of them).

STACK_SIGMA = 3.0
STACK_TRUNCATE = 4.0


def stack_halo():
    """z-slices of noise needed on each side of a window (the radius of the
    sigma-3 smoothing)."""
    return int(STACK_TRUNCATE * STACK_SIGMA + 0.5)


def stack_noise(z_indices, yx, seed=1, threads=None):
    """float32 N(0, 1) noise of the listed z-slices, shape (len(z), Y, X)."""
    from concurrent.futures import ThreadPoolExecutor

    out = np.empty((len(z_indices),) + tuple(yx), dtype=np.float32)

    def one(i):
        out[i] = np.random.default_rng([seed, 0, int(z_indices[i])]).standard_normal(
            tuple(yx), dtype=np.float32)

    with ThreadPoolExecutor(threads or _threads()) as ex:
        list(ex.map(one, range(len(z_indices))))
    return out


def stack_noise_std():
    """Standard deviation of the smoothed noise: the product over the three
    axes of the root sum of squares of the normalised float64 gaussian taps."""
    r = stack_halo()
    x = np.arange(-r, r + 1, dtype=np.float64)
    w = np.exp(-0.5 / (STACK_SIGMA * STACK_SIGMA) * x * x)
    w /= w.sum()
    return float(np.sum(w * w)) ** 1.5


def stack_shot(smoothed, z_indices, seed=1, threads=None):
    """uint16 slices: smoothed noise (float32) mapped to [0, 65535] by the
    fixed affine map, then Poisson shot noise, clipped."""
    from concurrent.futures import ThreadPoolExecutor

    std = stack_noise_std()
    scale = 65535.0 / (10.0 * std)
    out = np.empty(smoothed.shape, dtype=np.uint16)

    def one(i):
        lam = np.clip((smoothed[i].astype(np.float64) + 5.0 * std) * scale, 0.0, 65535.0)
        shot = np.random.default_rng([seed, 1, int(z_indices[i])]).poisson(lam)
        out[i] = np.clip(shot, 0, 65535).astype(np.uint16)

    with ThreadPoolExecutor(threads or _threads()) as ex:
        list(ex.map(one, range(len(z_indices))))
    return out


def _reflect_index(i, n):
    """'reflect' boundary index (d c b a | a b c d | d c b a) for any i."""
    if n == 1:
        return 0
    period = 2 * n
    i %= period
    return i if i < n else period - 1 - i


def stack_window(z0, z1, shape, gaussian_filter, seed=1, threads=None):
    """Slices [z0, z1) of the stack of `shape`, made from a noise window with
    `stack_halo()` extra slices on each side (reflected at the stack's ends)
    smoothed by `gaussian_filter(noise, sigma, mode=..., truncate=...)`;
    only the centre slices, whose z taps stay inside the window, are kept."""
    h = stack_halo()
    zs = [_reflect_index(z, shape[0]) for z in range(z0 - h, z1 + h)]
    noise = stack_noise(zs, shape[1:], seed, threads)
    sm = np.asarray(gaussian_filter(noise, STACK_SIGMA, mode="reflect",
                                    truncate=STACK_TRUNCATE), dtype=np.float32)
    return stack_shot(np.ascontiguousarray(sm[h:h + (z1 - z0)]), list(range(z0, z1)), seed,
                      threads)


def _threads():
    import os

    return max(1, min(32, os.cpu_count() or 1))


def rectangles_image(shape=(8192, 8192), n_rect=64, seed=2):
    rng = np.random.default_rng(seed)
    img = rng.random(shape, dtype=np.float32)
    for _ in range(n_rect):
        y = np.sort(rng.integers(0, shape[0], 2))
        x = np.sort(rng.integers(0, shape[1], 2))
        img[y[0]:y[1] + 1, x[0]:x[1] + 1] = np.float32(rng.uniform(0, 10))
    return img


def rgb_tiles(n_tiles=4096, side_range=(64, 1024), seed=3, sigma_range=(0.5, 8.0)):
    """List of (H, W, 3) uint8 tiles and a float sigma per tile."""
    rng = np.random.default_rng(seed)
    means = np.array([60.0, 150.0, 220.0])
    tiles, sigmas = [], []
    for _ in range(n_tiles):
        h, w = rng.integers(side_range[0], side_range[1] + 1, 2)
        comp = rng.integers(0, 3, size=(h, w, 3))
        vals = rng.normal(means[comp], 20.0)
        tiles.append(np.clip(np.rint(vals), 0, 255).astype(np.uint8))
        sigmas.append(float(rng.uniform(*sigma_range)))
    return tiles, sigmas


def rgb_tiles_device(device, n_tiles=4096, side_range=(64, 1024), seed=3, sigma_range=(0.5, 8.0)):
    """rgb_tiles generated on the device: the same tile sides and sigmas as
    rgb_tiles (numpy, seed 3), pixel values from the same 3-component mixture
    (means 60 / 150 / 220, sd 20, equal weights, rounded, clipped to
    [0, 255]) drawn with a seeded torch generator."""
    import torch

    rng = np.random.default_rng(seed)
    sides = [rng.integers(side_range[0], side_range[1] + 1, 2) for _ in range(n_tiles)]
    sigmas = [float(rng.uniform(*sigma_range)) for _ in range(n_tiles)]
    g = torch.Generator(device=device).manual_seed(seed)
    means = torch.tensor([60.0, 150.0, 220.0], device=device)
    tiles = []
    for h, w in sides:
        comp = torch.randint(0, 3, (int(h), int(w), 3), generator=g, device=device)
        vals = torch.randn((int(h), int(w), 3), generator=g, device=device) * 20.0 + means[comp]
        tiles.append(vals.round_().clamp_(0, 255).to(torch.uint8))
    return tiles, sigmas


def segments_volume(shape=(256, 256, 256), n_segments=200, seed=4,
                    length_range=(20, 120), radius_range=(1.0, 4.0)):
    rng = np.random.default_rng(seed)
    vol = rng.normal(0.0, 0.05, size=shape).astype(np.float32)
    dims = np.array(shape)
    for _ in range(n_segments):
        p0 = rng.uniform(0, dims)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        length = rng.uniform(*length_range)
        sig = rng.uniform(*radius_range)
        p1 = p0 + d * length
        reach = 4 * sig
        lo = np.maximum(np.floor(np.minimum(p0, p1) - reach).astype(int), 0)
        hi = np.minimum(np.ceil(np.maximum(p0, p1) + reach).astype(int) + 1, dims)
        if np.any(hi <= lo):
            continue
        zz, yy, xx = np.meshgrid(*[np.arange(lo[i], hi[i]) for i in range(3)], indexing="ij")
        pts = np.stack([zz, yy, xx], -1).astype(np.float64)
        t = np.clip(((pts - p0) @ d) / length, 0.0, 1.0)
        closest = p0 + (t[..., None] * length) * d
        d2 = ((pts - closest) ** 2).sum(-1)
        vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += np.exp(
            -d2 / (2 * sig * sig)).astype(np.float32)
    return vol


def gaussian_radius(sigma, truncate=4.0):
    return int(truncate * float(sigma) + 0.5)


def taps_count(sigma, truncate=4.0):
    return 2 * gaussian_radius(sigma, truncate) + 1


__all__ = [
    "uniform_image", "smooth_volume_u16", "stack_noise", "stack_shot", "stack_window",
    "stack_halo", "stack_noise_std", "rectangles_image", "rgb_tiles", "segments_volume",
    "gaussian_radius", "taps_count", "math",
]
