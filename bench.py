"""Benchmark of the separable filtering path on B200.

Workload (one step): the 512 x 1024 x 1024 uint16 stack (smoothed noise with
Poisson shot noise, seed 1; drawn slice by slice so that the CPU arm can
regenerate any z-window of it exactly) filtered by
  - ndimage.gaussian_filter(sigma=(1, 2, 2), mode='mirror', output=float32),
  - ndimage.sobel(axis=a, output=float32) for a = 0, 1, 2,
  - ndimage.uniform_filter(size=5, output=uint16)  (bit-exact integer path),
into preallocated outputs. `value` = voxels filtered per second (the stack's
voxel count per step / step time), whole job over all ranks. The stack is
1 GiB in and 9 GiB out, far above the 126 MB L2, so no flush is needed.

Precision path (reported beside the headline, in `precision_path`): the
8192 x 8192 float32 image of uniform noise plus 64 constant rectangles
(seed 2) filtered by gaussian_filter(sigma=16 and 32, mode='nearest') and
uniform_filter(size=63, mode='nearest'), once with the plain float32 kernels
and once on the tensor cores (algorithm='tensor', TF32x3). For each filter:
device time, Gpx/s, the speed-up, and the max / mean error relative to the
largest output magnitude against a float64 scipy.ndimage reference on a
2048 x 2048 crop (4.2 Mpx; the full image would take minutes on the CPU).
The 256 MiB image alone is above L2; every timed repetition reads it from HBM.

Plain 2-D gaussian (reported in `plain_2d_gaussian`): gaussian sigma 4,
truncate 4, mode 'reflect' on float32 2048 x 2048 uniform images (seed 0),
16 distinct images per repetition so that the inputs exceed L2. The kernel
rate (GB/s at 8 bytes per pixel, fraction of the measured HBM copy
bandwidth) comes from one call over the 16 images as a stack; the per-call
times of ndimage.gaussian_filter and skimage.filters.gaussian, one image per
call, are reported beside it.

Frangi (reported in `frangi`): skimage.filters.frangi(sigmas=1..5,
alpha=beta=0.5, gamma=None, black_ridges=False) on the 256^3 float32
segments volume (seed 4), with the plain float32 passes, with
algorithm="tensor" (tensor cores only on lines of >= 2048 samples, so all
plain here), and with the tensor cores forced on every pass; each with its
largest difference from the plain result.

Batched tiles (reported in `batched_tiles`): 4096 uint8 RGB tiles with
sides drawn from 64..1024 (seed 3; about 1.2 Gpx), each filtered by
rgb2gray -> gaussian(its own sigma in [0.5, 8]) -> sobel magnitude, once as
three public calls per tile and once as one persistent launch replayed from
a CUDA graph; the ratio of the two times, and a bit-for-bit comparison of
the two outputs on a sample of tiles.

Parity (reported in `parity`): after timing, the step's outputs are checked
against the oracle on three 16-slice z-windows of the stack (first, middle,
last; the oracle filters each window with its z halo), bit for bit; the
first 8 slices of the stack are compared with the CPU arm's regeneration of
them; the 2-D gaussian of the 2048 x 2048 image is checked bit for bit; the
precision-path errors are pointwise over the full 8192 x 8192 image; the
frangi output on the 256^3 volume is compared with the oracle's.

--impl reference times the CPU restatement of cuCIM's arithmetic (the
oracle; cuCIM itself needs CuPy and has no CPU implementation) on the host
cores, on the first 8 z-slices of the same stack (regenerated on the CPU by
the same generator), with the same `config`. It imports nothing from the
cucim_b200 package: the generators are loaded from their file.

Multi-GPU: the path has no exchange step; N ranks run N independent replicas
of the step (weak scaling) and the time is the max over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gvox/s gaussian & frangi: tensor-core vs plain FP32 kernel at ≤2e-6 max rel err"
SHAPE = (512, 1024, 1024)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--shape", default=None, help="override the stack shape, e.g. 64,256,256")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-precision", action="store_true", help="skip the precision-path report")
    p.add_argument("--precision-size", type=int, default=8192)
    p.add_argument("--skip-main", action="store_true",
                   help="run only the precision path and the batched tiles (for profiling)")
    p.add_argument("--no-tiles", action="store_true", help="skip the batched-tiles report")
    p.add_argument("--no-sksobel", action="store_true",
                   help="skip the skimage sobel(axis) variant of the stack")
    p.add_argument("--tiles", type=int, default=4096, help="tiles in the batched-tiles report")
    p.add_argument("--no-frangi", action="store_true", help="skip the frangi report")
    p.add_argument("--no-plain2d", action="store_true", help="skip the 2-D gaussian report")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the oracle checks of the outputs (parity field)")
    return p.parse_args()


# ------------------------------------------------------------------ inputs

def load_synthetic():
    """The input generators (numpy only), loaded from their file so that the
    CPU arm never runs cucim_b200/__init__.py, which loads libcimx.so."""
    import importlib.util

    path = os.path.join(ROOT, "cucim_b200", "synthetic.py")
    spec = importlib.util.spec_from_file_location("cimx_bench_synthetic", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_stack(shape, device):
    """The seed-1 stack: per-slice normal noise (host), smoothed on the device
    by gaussian_filter(sigma 3, reflect), mapped to [0, 65535] with Poisson
    shot noise per slice (host), uploaded as uint16."""
    import torch

    from cucim_b200 import ndimage as ndi

    S = load_synthetic()
    noise = torch.from_numpy(S.stack_noise(range(shape[0]), shape[1:])).to(device)
    sm = ndi.gaussian_filter(noise, S.STACK_SIGMA, mode="reflect", truncate=S.STACK_TRUNCATE)
    del noise
    smh = sm.cpu().numpy()
    del sm
    return torch.from_numpy(S.stack_shot(smh, range(shape[0]))).to(device)


def stack_config(shape, world):
    """The `config` of both arms (the CPU arm states its sample separately)."""
    return {"workload": "3-D uint16 stack (seed 1): gaussian(sigma=(1,2,2), mirror)->f32, "
                        "sobel(axis=0,1,2)->f32, uniform(size=5)->u16 (bit-exact)",
            "shape": list(shape), "voxels_per_step": int(np.prod(shape)),
            "l2": "inputs 1 GiB > L2 (126 MB), no flush", "parallelism": f"replicas x{world}"}


# --------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start; wait for its first sample
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.rows.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------------- ours

# the five filters of a step, in order, each writing one output
STEP_OPS = (
    lambda ndi, x, o: ndi.gaussian_filter(x, (1, 2, 2), mode="mirror", output=o),
    lambda ndi, x, o: ndi.sobel(x, 0, output=o),
    lambda ndi, x, o: ndi.sobel(x, 1, output=o),
    lambda ndi, x, o: ndi.sobel(x, 2, output=o),
    lambda ndi, x, o: ndi.uniform_filter(x, 5, output=o),
)


def step_ops(ndi, x, outs):
    for op, o in zip(STEP_OPS, outs):
        op(ndi, x, o)


# gaussian: one streamed z pass + one fused (y, x) launch; each sobel and the
# uniform filter: one launch of the volume kernel
LAUNCHES_PER_STEP = 6

# DRAM bytes per launch measured by ncu on a smaller stack: (bytes, slices of
# that stack, profile file)
TRAFFIC = {
    "slab f32->f32 gaussian y,x K=17,17": (201.404672e6 + 162.276608e6, 48,
                                           "k_slab_f32_gaussian_yx_48x1024x1024_and_2048x2048.md"),
    "volume u16->f32 sobel K=3,3,3": (135.097344e6 + 212.728064e6, 64,
                                      "k_vol_u16_f32_sobel_64x1024x1024.md"),
}


def reduce_step_time(ms, world, device, dist, torch):
    """Max over ranks of the per-step device time (ms): the job is as slow as
    its slowest replica."""
    if world <= 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(nvox, world, ms):
    """Whole-job throughput in Gvox/s: every rank filters its own stack."""
    return nvox * world / (ms * 1e-3) / 1e9


def time_kernel(fn, reps, torch):
    """Average device time of fn() (one launch) with events on the current stream."""
    fn()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from cucim_b200 import ndimage as ndi

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    x = make_stack(shape, dev)
    nvox = x.numel()
    f32 = lambda: torch.empty(shape, dtype=torch.float32, device=dev)  # noqa: E731
    outs = [f32(), f32(), f32(), f32(), torch.empty(shape, dtype=torch.uint16, device=dev)]
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    # the first warm-up step times every schedule of each filter's signature
    # (the autotuner); the timed steps run the recorded fastest ones
    from cucim_b200 import tune

    prev_mode = tune.mode(tune.ON)
    step_ops(ndi, x, outs)
    tune.mode(tune.USE)
    for _ in range(args.warmup):
        step_ops(ndi, x, outs)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        t0.record()
        for _ in range(args.steps):
            step_ops(ndi, x, outs)
        t1.record()
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = reduce_step_time(t0.elapsed_time(t1) / args.steps, world, dev, dist, torch)
    value = aggregate_value(nvox, world, ms)

    # per-kernel timing: each call below is exactly one launch of the kernel
    # that runs inside the step (same shapes, same dtypes)
    tmp = outs[0]
    # (call, algorithmic bytes per launch, launches per step)
    kt = {
        "volume u16->f32 sobel K=3,3,3": (
            lambda: ndi.sobel(x, 0, output=outs[1]), 6 * nvox, 3),
        "slab f32->f32 gaussian y,x K=17,17": (
            lambda: ndi.gaussian_filter(tmp, (0, 2, 2), mode="mirror", output=outs[1]),
            8 * nvox, 1),
        "volume u16->u16 uniform K=5,5,5": (
            lambda: ndi.uniform_filter(x, 5, output=outs[4]), 4 * nvox, 1),
        "stream u16->f32 gaussian z K=9": (
            lambda: ndi.gaussian_filter1d(x, 1.0, axis=0, mode="mirror", output=outs[1]),
            6 * nvox, 1),
    }
    kres = {}
    for name, (fn, nbytes, per_step) in kt.items():
        kms = time_kernel(fn, 5, torch)
        kres[name] = {"ms": kms, "bytes": nbytes, "gbs": nbytes / (kms * 1e-3) / 1e9,
                      "launches_per_step": per_step}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(ndi, torch, x, shape, outs, args, world)

    parity = None
    if rank == 0 and not args.no_parity:
        step_ops(ndi, x, outs)  # the per-kernel timing above rewrote some outputs
        torch.cuda.synchronize()
        parity = stack_parity(x, outs)

    sks = None
    if rank == 0 and not args.no_sksobel:
        sks = run_sk_sobel(torch, x)
    x_host = x.cpu() if rank == 0 else None
    prec = None
    if rank == 0 and not args.no_precision:
        del outs, tmp
        torch.cuda.empty_cache()
        prec = run_precision(torch, ndi, dev, size=args.precision_size,
                             tf32_peak=_peaks().get("bf16_tflops", 1590.0) / 2)
    tiles = None
    if rank == 0 and not args.no_tiles:
        torch.cuda.empty_cache()
        tiles = run_tiles(torch, dev, n_tiles=args.tiles)
    fr = None
    if rank == 0 and not args.no_frangi:
        torch.cuda.empty_cache()
        fr = run_frangi(torch, dev)
    p2 = None
    if rank == 0 and not args.no_plain2d:
        p2 = run_plain2d(torch, dev, hbm_gbs=_peaks().get("hbm_gbs"))

    tune.mode(prev_mode)
    return {"value": value, "ms": ms, "nvox": nvox, "kernels": kres, "clocks": clk.summary(),
            "e2e": e2e, "x": x_host, "parity": parity, "autotune": tune.entries(), "precision": prec, "tiles": tiles, "frangi": fr,
            "plain2d": p2, "sk_sobel": sks}


# the z radius of the step's filters: gaussian sigma 1 (4), sobel (1), uniform 5 (2)
STEP_Z_HALO = 4
ORACLE_STEP = (
    lambda R, x: R.gaussian_filter(x, (1, 2, 2), mode="mirror", output=np.float32),
    lambda R, x: R.sobel(x, 0, output=np.float32),
    lambda R, x: R.sobel(x, 1, output=np.float32),
    lambda R, x: R.sobel(x, 2, output=np.float32),
    lambda R, x: R.uniform_filter(x, 5, output=np.uint16),
)
STEP_NAMES = ("gaussian_f32", "sobel0_f32", "sobel1_f32", "sobel2_f32", "uniform5_u16")


def stack_parity(x, outs, win=16, sample=8):
    """The step's outputs against the oracle on the first, middle and last
    `win` z-slices of the stack: the oracle filters each window with
    STEP_Z_HALO extra slices on each side (none beyond the stack's ends,
    where the boundary mode applies as on the full stack) and the window's
    own slices are compared bit for bit. Also: the first `sample` slices of
    the stack against the CPU arm's regeneration of them."""
    from oracle import restate as R

    R.THREADS = os.cpu_count() or 1
    Z = x.shape[0]
    t0 = time.perf_counter()
    windows = []
    for z0 in sorted({0, max(0, Z // 2 - win // 2), max(0, Z - win)}):
        z1 = min(Z, z0 + win)
        a, b = max(0, z0 - STEP_Z_HALO), min(Z, z1 + STEP_Z_HALO)
        xs = x[a:b].cpu().numpy()
        row = {"z": [z0, z1]}
        for name, op, o in zip(STEP_NAMES, ORACLE_STEP, outs):
            exp = op(R, xs)[z0 - a:z1 - a]
            got = o[z0:z1].cpu().numpy()
            row[name] = bool(np.array_equal(got, exp))
        windows.append(row)
    S = load_synthetic()
    regen = S.stack_window(0, sample, tuple(x.shape), R.gaussian_filter)
    same_input = bool(np.array_equal(regen, x[:sample].cpu().numpy()))
    return {"check": f"oracle bit for bit on {len(windows)} z-windows of {win} slices "
                     f"(each with a {STEP_Z_HALO}-slice halo), all five filters",
            "windows": windows,
            "bit_exact": all(all(v for k, v in w.items() if k != "z") for w in windows),
            "input_equals_cpu_arm_sample": same_input,
            "seconds": time.perf_counter() - t0}


def run_e2e(ndi, torch, x, shape, douts, args, world):
    """Public API with host buffers: pinned H2D of the stack, the five filters,
    D2H of all five outputs, every step. The H2D of step k + 1 runs on a copy
    stream into a second device buffer while step k's outputs travel back
    (PCIe carries both directions at once), and each output's D2H runs on a
    third stream as soon as its filter is done (the filter of the next step
    that rewrites that output waits for it); the first step's H2D is inside
    the timed region and not overlapped."""
    hx = torch.empty(shape, dtype=torch.uint16, pin_memory=True)
    hx.copy_(x.cpu())
    houts = [torch.empty(shape, dtype=torch.float32, pin_memory=True) for _ in range(4)]
    houts.append(torch.empty(shape, dtype=torch.uint16, pin_memory=True))
    dxs = [torch.empty_like(x), torch.empty_like(x)]
    main = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    back = torch.cuda.Stream()
    loaded = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]
    done = [torch.cuda.Event() for _ in douts]
    sent = [torch.cuda.Event() for _ in douts]

    def load(k):
        # buffer k % 2 is free once the step two before k has read it
        with torch.cuda.stream(copy):
            copy.wait_event(consumed[k % 2])
            dxs[k % 2].copy_(hx, non_blocking=True)
            loaded[k % 2].record(copy)

    def run(steps):
        for ev in consumed + sent:
            ev.record(main)
        copy.wait_stream(main)
        back.wait_stream(main)
        load(0)
        for k in range(steps):
            main.wait_event(loaded[k % 2])
            if k + 1 < steps:
                load(k + 1)
            for i, (op, d) in enumerate(zip(STEP_OPS, douts)):
                main.wait_event(sent[i])  # the previous step's copy of d is out
                op(ndi, dxs[k % 2], d)
                done[i].record(main)
                with torch.cuda.stream(back):
                    back.wait_event(done[i])
                    houts[i].copy_(d, non_blocking=True)
                    sent[i].record(back)
            consumed[k % 2].record(main)
        main.wait_stream(copy)
        main.wait_stream(back)

    steps = max(1, min(args.steps, 5))
    run(1)
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    run(steps)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / steps
    nvox = x.numel()
    return {"value": nvox * world / (ms * 1e-3) / 1e9, "unit": "Gvox/s",
            "h2d_bytes_per_step": int(hx.numel() * 2),
            "d2h_bytes_per_step": int(sum(h.numel() * h.element_size() for h in houts)),
            "ms_per_step": ms, "steps": steps,
            "schedule": "H2D of the next step and each output's D2H overlapped with the "
                        "filters (two input buffers, three streams)"}


# ---------------------------------------------------------- precision path

PRECISION_OPS = (  # (name, function, arguments, taps per pass)
    ("gaussian sigma=16 (K=129)", "gaussian_filter", {"sigma": 16.0}, 129),
    ("gaussian sigma=32 (K=257)", "gaussian_filter", {"sigma": 32.0}, 257),
    ("uniform size=63", "uniform_filter", {"size": 63}, 63),
)


def tf32x3_flops_per_output(K):
    """Tensor FLOPs the TF32x3 kernel executes per output per pass: 3 MMAs
    (hi*hi, hi*lo, lo*hi) of 128 outputs x 8 coordinates (2 FLOPs each) for
    each of the SB = ceil((128 + K' - 1) / 8) slices of a 128-output block;
    K' is K plus the zero taps that align an odd anchor (K // 2 % 4)."""
    Kp = K + ((-(K // 2)) % 4)
    sb = (128 + Kp - 1 + 7) // 8
    return 3 * 16 * sb


def run_precision(torch, ndi, dev, reps=5, crop=2048, size=8192, tf32_peak=None, floor=1e-3):
    """Plain float32 vs TF32x3 tensor-core filters on the precision workload:
    device time per filter (CUDA events, `reps` repetitions after a warm-up)
    and the error of each result over the FULL image against a float64
    reference. The reference is the same filter computed in float64 on the
    device (float64 taps, float64 fused chain: its own error is ~1e-15); it
    is pinned against scipy.ndimage in float64 on a crop, which it must match
    to 1e-12. Errors are pointwise: |out - ref| / max(|ref|, floor); every
    output of this workload is positive and far above the floor (counted in
    `pixels_below_floor`). The error relative to the largest output is given
    beside it."""
    import scipy.ndimage as sndi

    S = load_synthetic()
    img = S.rectangles_image((size, size), n_rect=64, seed=2)
    X = torch.as_tensor(img).to(dev)
    O = torch.empty_like(X)
    X64 = X.double()
    crop = min(crop, size)
    xc = np.ascontiguousarray(img[:crop, :crop]).astype(np.float64)
    Xc64 = torch.as_tensor(xc).to(dev)
    res = {}
    for name, fn, kw, K in PRECISION_OPS:
        f = getattr(ndi, fn)
        ref = f(X64, mode="nearest", **kw)
        sref = getattr(sndi, fn)(xc, mode="nearest", **kw)
        pin = float(np.abs(f(Xc64, mode="nearest", **kw).cpu().numpy() - sref).max()
                    / np.abs(sref).max())
        aref = ref.abs()
        den = aref.clamp_min(floor)
        row = {"reference_vs_scipy_f64_on_crop": pin}
        for algo, key in ((None, "plain_f32"), ("tensor", "tensor_tf32x3")):
            ms = time_kernel(lambda: f(X, mode="nearest", output=O, algorithm=algo, **kw), reps, torch)
            f(X, mode="nearest", output=O, algorithm=algo, **kw)
            err = (O.double() - ref).abs()
            rel = err / den
            row[key] = {"ms": ms, "gpx_s": X.numel() / (ms * 1e-3) / 1e9,
                        "max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean()),
                        "max_err_over_max_output": float(err.max() / aref.max())}
            del err, rel
        row["pixels_below_floor"] = int((aref < floor).sum())
        row["speedup"] = row["plain_f32"]["ms"] / row["tensor_tf32x3"]["ms"]
        tflops = 2 * tf32x3_flops_per_output(K) * X.numel() / (row["tensor_tf32x3"]["ms"] * 1e-3) / 1e12
        row["tensor_tf32x3"]["executed_tflops"] = tflops
        # two passes of K fused multiply-adds (2 flops each) per pixel
        for key in ("plain_f32", "tensor_tf32x3"):
            row[key]["useful_tflops"] = 2 * 2 * K * X.numel() / (row[key]["ms"] * 1e-3) / 1e12
        if tf32_peak:
            row["tensor_tf32x3"]["frac_of_tf32_peak"] = tflops / tf32_peak
        row["tensor_within_2e-6"] = row["tensor_tf32x3"]["max_rel_err"] <= 2e-6
        row["plain_within_2e-6"] = row["plain_f32"]["max_rel_err"] <= 2e-6
        res[name] = row
        del ref, aref, den
    # the oracle's sigma-16 gaussian on the crop with all host threads: the CPU baseline
    from oracle import restate as R

    R.THREADS = os.cpu_count() or 1
    xc32 = xc.astype(np.float32)
    t0 = time.perf_counter()
    R.gaussian_filter(xc32, 16.0, mode="nearest")
    cpu_s = time.perf_counter() - t0
    return {"workload": f"float32 {size}x{size} uniform noise + 64 rectangles (seed 2), mode nearest",
            "cpu_baseline": {"value": xc32.size / cpu_s / 1e9, "unit": "Gpx/s",
                             "cores": R.THREADS, "kind": "port",
                             "sample": f"gaussian sigma 16 (float32 chain) on the {crop}x{crop} "
                                       f"crop, {cpu_s:.2f} s"},
            "tf32_peak_tflops": tf32_peak,
            "tf32_peak_source": "half the measured bf16 dense peak (kind::tf32 MMAs ran at "
                                "4092 vs 8184 flop/clk/SM for kind::f16 in a microbenchmark)",
            "error_reference": f"the filter in float64 on the device over the full {size}x{size} "
                               f"image, pinned against scipy.ndimage float64 on the {crop}x{crop} "
                               "crop; error = |out - ref| / max(|ref|, floor)",
            "floor": floor, "filters": res}


# ------------------------------------------------- skimage sobel variant

def run_sk_sobel(torch, x):
    """The second variant of the stack's sobel: skimage.filters.sobel(axis=a)
    for a = 0, 1, 2 on the uint16 stack (img_as_float to float32 / 65535,
    then the edge pass and two smoothing passes, float32 out), one call per
    axis as a user makes them. Parity: the first 16 z-slices of each output
    against the oracle on the stack's first 17 slices (the real z border is
    inside the window, the 17th slice only feeds the discarded one)."""
    from cucim_b200.skimage import filters
    from oracle import restate as R

    nvox = x.numel()

    def step():
        return [filters.sobel(x, axis=a) for a in range(3)]

    outs = step()
    del outs
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    reps = 3
    s.record()
    for _ in range(reps):
        outs = step()
        del outs
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    outs = step()
    R.THREADS = os.cpu_count() or 1
    host = x[:17].cpu().numpy()
    ok = all(np.array_equal(outs[a][:16].cpu().numpy(), R.sk_sobel(host, axis=a)[:16])
             for a in range(3))
    del outs
    torch.cuda.empty_cache()
    return {"workload": "skimage.filters.sobel(axis=a), a = 0, 1, 2, on the uint16 "
                        "512 x 1024 x 1024 stack (three calls, float32 / 65535 out)",
            "ms": ms, "gvox_s": nvox / (ms * 1e-3) / 1e9,
            "algorithmic_gbs": 3 * 6 * nvox / (ms * 1e-3) / 1e9,
            "note": "6 B per voxel per axis (uint16 in, float32 out); the library converts "
                    "with img_as_float first (one extra float32 round trip per call)",
            "oracle_bit_exact": bool(ok), "parity_window": "z 0..15 of each axis' output"}


# ----------------------------------------------------------- batched tiles

def run_tiles(torch, dev, reps=3, check=64, n_tiles=4096):
    from cucim_b200 import batch

    tiles, sigmas = load_synthetic().rgb_tiles_device(dev, n_tiles=n_tiles)
    npx = sum(int(t.shape[0]) * int(t.shape[1]) for t in tiles)
    b = batch.TileBatch(tiles, sigmas)
    g = b.graph()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    g.replay()
    s.record()
    for _ in range(reps):
        g.replay()
    e.record()
    torch.cuda.synchronize()
    ms_b = s.elapsed_time(e) / reps
    # per tile: rgb2gray, gaussian, sobel through the public API (one pass;
    # it is bounded by the launches and the host work per call)
    batch.gray_gauss_sobel_per_tile(tiles[:8], sigmas[:8])
    torch.cuda.synchronize()
    s.record()
    ref = batch.gray_gauss_sobel_per_tile(tiles, sigmas)
    e.record()
    torch.cuda.synchronize()
    ms_t = s.elapsed_time(e)
    step = max(1, len(tiles) // check)
    same = all(torch.equal(b.outputs[i], ref[i]) for i in range(0, len(tiles), step))
    # the oracle on a sample of tiles: bit for bit, and its time as the CPU baseline
    from oracle import restate as R

    R.THREADS = os.cpu_count() or 1
    sample = list(range(0, len(tiles), max(1, len(tiles) // 16)))[:16]
    host = [tiles[i].cpu().numpy() for i in sample]
    t0 = time.perf_counter()
    exp = [R.sk_sobel(R.sk_gaussian(R.rgb2gray(h), sigmas[i])) for h, i in zip(host, sample)]
    cpu_s = time.perf_counter() - t0
    spx = sum(h.shape[0] * h.shape[1] for h in host)
    oracle_ok = all(np.array_equal(b.outputs[i].cpu().numpy(), e) for i, e in zip(sample, exp))
    # end to end from host memory: the same tiles held on the host through
    # RegionStream (pinned staging, copies overlapped with the launches),
    # results back in host memory
    host_tiles = [t.cpu().numpy() for t in tiles]
    rs = batch.RegionStream(host_tiles, sigmas)
    rs.run()
    t0 = time.perf_counter()
    res = rs.run()
    e2e_s = time.perf_counter() - t0
    e2e_same = all(np.array_equal(res[i], b.outputs[i].cpu().numpy())
                   for i in range(0, len(tiles), step))
    del res, host_tiles, rs
    # compute roofline: the useful float32 FMAs of the path per output pixel
    # (K taps of each Gaussian pass, 3 + 3 taps of each sobel direction);
    # the halo the kernel recomputes around every 64 x 64 block is not useful work
    fma = 0
    for t, sg in zip(tiles, sigmas):
        K = 2 * int(4.0 * sg + 0.5) + 1
        fma += int(t.shape[0]) * int(t.shape[1]) * (2 * K + 12)
    fp32_nominal = 148 * 128 * 2 * 1.965e9 / 1e12
    useful_tflops = 2 * fma / (ms_b * 1e-3) / 1e12
    return {"workload": f"{len(tiles)} uint8 RGB tiles, sides 64..1024 (seed 3), "
                        "rgb2gray -> gaussian(sigma 0.5..8, nearest) -> sobel magnitude, float32 out",
            "pixels": npx, "batched_ms": ms_b, "batched_gpx_s": npx / (ms_b * 1e-3) / 1e9,
            "per_tile_ms": ms_t, "per_tile_gpx_s": npx / (ms_t * 1e-3) / 1e9,
            "speedup": ms_t / ms_b, "launches_batched": 1, "launches_per_tile": "about 7 per tile",
            "e2e_from_host": {"s": e2e_s, "gpx_s": npx / e2e_s / 1e9,
                              "h2d_bytes": 3 * npx, "d2h_bytes": 4 * npx,
                              "bit_identical": bool(e2e_same),
                              "path": "cucim_b200.batch.RegionStream: host tiles gathered into "
                                      "pinned chunks, copies and launches overlapped, results "
                                      "copied back into host arrays"},
            "roofline": {"bound": "fp32", "achieved": useful_tflops, "peak": fp32_nominal,
                         "unit": "TFLOP/s", "frac": useful_tflops / fp32_nominal,
                         "note": "useful float32 FMAs (2K + 12 per output pixel) over the nominal "
                                 "148 SM x 128 FMA/clk x 1.965 GHz; HBM traffic is 7 B per pixel "
                                 f"({7 * npx / (ms_b * 1e-3) / 1e9:.0f} GB/s)"},
            "bit_identical": bool(same), "tiles_compared": len(range(0, len(tiles), step)),
            "oracle_bit_exact": bool(oracle_ok), "oracle_tiles_compared": len(sample),
            "cpu_baseline": {"value": spx / cpu_s / 1e9, "unit": "Gpx/s", "cores": R.THREADS,
                             "kind": "port",
                             "sample": f"{len(sample)} tiles ({spx} px), rgb2gray -> gaussian -> "
                                       f"sobel in the oracle, {cpu_s:.2f} s"}}


# ---------------------------------------------------------- plain 2-D case

def run_plain2d(torch, dev, n_img=16, reps=5, hbm_gbs=None):
    """skimage.filters.gaussian(sigma=4, truncate=4, mode='reflect') on
    float32 2048 x 2048 uniform images (seed 0): two fused passes of 33 taps.
    One image is 16 MiB and would stay in L2, so each timed repetition
    filters 16 distinct images (512 MiB in and out)."""
    from cucim_b200.skimage import filters

    S = load_synthetic()
    base = torch.as_tensor(S.uniform_image((2048, 2048), seed=0)).to(dev)
    imgs = [base + float(i) for i in range(n_img)]
    outs = [torch.empty_like(base) for _ in range(n_img)]

    def one():
        for im, o in zip(imgs, outs):
            o.copy_(filters.gaussian(im, sigma=4.0, mode="reflect", truncate=4.0))

    from cucim_b200 import ndimage as ndi

    def one_direct():
        for im, o in zip(imgs, outs):
            ndi.gaussian_filter(im, 4.0, mode="reflect", truncate=4.0, output=o)

    # the same 16 images as one (16, 2048, 2048) stack filtered over axes
    # (1, 2): one launch, no per-call host work -- the kernel's own rate
    stack = torch.stack(imgs)
    stack_out = torch.empty_like(stack)

    def one_stack():
        ndi.gaussian_filter(stack, 4.0, mode="reflect", truncate=4.0, axes=(1, 2), output=stack_out)

    from cucim_b200 import tune

    with tune.tuning(tune.ON):  # record the schedules of both signatures
        one_stack()
        ndi.gaussian_filter(imgs[0], 4.0, mode="reflect", truncate=4.0, output=outs[0])
    ms = time_kernel(one_direct, reps, torch) / n_img
    ms_api = time_kernel(one, reps, torch) / n_img
    ms_kernel = time_kernel(one_stack, reps, torch) / n_img
    # the 2048 x 2048 image against the oracle, bit for bit, and the oracle's
    # time on it with all host threads as the CPU baseline
    from oracle import restate as R

    R.THREADS = os.cpu_count() or 1
    img = S.uniform_image((2048, 2048), seed=0)
    got = filters.gaussian(base, sigma=4.0, mode="reflect", truncate=4.0).cpu().numpy()
    t0 = time.perf_counter()
    exp = R.sk_gaussian(img, 4.0, mode="reflect", truncate=4.0)
    cpu_s = time.perf_counter() - t0
    gbs = 8 * base.numel() / (ms_kernel * 1e-3) / 1e9
    res = {"workload": "float32 2048x2048 uniform (seed 0), gaussian sigma 4 (K=33), mode reflect; "
                       f"{n_img} distinct images per repetition (inputs above L2)",
           "ms_per_image_kernel": ms_kernel, "gpx_s": base.numel() / (ms_kernel * 1e-3) / 1e9,
           "gb_s": gbs, "kernel_note": f"one launch over the {n_img} images as a stack, axes (1, 2)",
           "ms_per_image_per_call": ms, "ms_per_image_skimage_api": ms_api,
           "per_call_note": "one ndimage.gaussian_filter call per image (includes the host work "
                            "of each call) and one skimage.filters.gaussian call per image",
           "oracle_bit_exact": bool(np.array_equal(got, exp)),
           "cpu_baseline": {"value": img.size / cpu_s / 1e9, "unit": "Gpx/s", "cores": R.THREADS,
                            "kind": "port", "sample": f"the 2048x2048 image, {cpu_s:.3f} s"}}
    if hbm_gbs:
        res["frac_of_hbm"] = gbs / hbm_gbs
    # 33 taps on each of two axes: 2 * 2 * 33 useful flops per pixel, which
    # at the nominal FP32 rate (148 SMs x 128 FMA lanes x 2 x 1965 MHz) take
    # longer than the 8 bytes per pixel at the measured copy bandwidth
    tflops = 2 * 2 * 33 * base.numel() / (ms_kernel * 1e-3) / 1e12
    fp32_nominal = 148 * 128 * 2 * 1.965e9 / 1e12
    res["fp32_tflops"] = tflops
    res["fp32_nominal_tflops"] = fp32_nominal
    res["frac_of_fp32_nominal"] = tflops / fp32_nominal
    return res


# --------------------------------------------------------------- frangi

def frangi_agreement(got, exp):
    """How far the GPU frangi output is from the oracle's: the share of
    voxels that differ, the largest difference in float32 ulps (of the
    oracle's value) and relative to the largest output, and the largest
    pointwise relative difference among outputs above 1e-3 of the largest."""
    g = got.astype(np.float64)
    e = exp.astype(np.float64)
    diff = np.abs(g - e)
    scale = float(np.abs(e).max()) or 1.0
    ulp = np.spacing(np.abs(exp).astype(np.float32)).astype(np.float64)
    big = np.abs(e) >= 1e-3 * scale
    return {"voxels": int(e.size), "voxels_differing": int((diff > 0).sum()),
            "max_ulps": float((diff / ulp).max()),
            "max_diff_over_max_output": float(diff.max() / scale),
            "max_rel_diff_outputs_above_1e-3_of_max": float((diff[big] / np.abs(e[big])).max())
            if big.any() else 0.0,
            "nan_mismatch": int((np.isnan(g) != np.isnan(e)).sum())}


def run_frangi(torch, dev, reps=3, check=True):
    """Multi-scale frangi (sigmas 1..5, alpha = beta = 0.5, automatic gamma,
    black_ridges=False) on the seed-4 segments volume: plain float32 passes
    against algorithm="tensor" (which keeps the plain kernels on these
    256-sample lines, where they measured faster) and against the tensor
    cores forced onto every pass, with the largest difference to the plain
    result relative to the largest output; the plain result against the
    oracle's frangi on the same volume, whose time with all host threads is
    the CPU baseline."""
    from cucim_b200 import ndimage as ndi
    from cucim_b200.skimage import filters

    vol_h = load_synthetic().segments_volume((256, 256, 256), seed=4)
    vol = torch.as_tensor(vol_h).to(dev)
    kw = dict(sigmas=range(1, 6), alpha=0.5, beta=0.5, gamma=None, black_ridges=False)
    from cucim_b200 import tune

    with tune.tuning(tune.ON):  # record the schedules of the Hessian passes
        filters.frangi(vol, **kw)
    res = {}
    outs = {}
    for algo, key, forced in ((None, "plain_f32", False), ("tensor", "tensor_tf32x3", False),
                              ("tensor", "tensor_tf32x3_all_passes", True)):
        def f():
            if forced:
                with ndi.tensor_cores_everywhere():
                    return filters.frangi(vol, algorithm=algo, **kw)
            return filters.frangi(vol, algorithm=algo, **kw)
        ms = time_kernel(f, reps, torch)
        outs[key] = f()
        res[key] = {"ms": ms, "gvox_s": vol.numel() / (ms * 1e-3) / 1e9}
    p = outs["plain_f32"].double()
    scale = float(p.abs().max())
    for key in ("tensor_tf32x3", "tensor_tf32x3_all_passes"):
        t = outs[key].double()
        res[key]["speedup"] = res["plain_f32"]["ms"] / res[key]["ms"]
        res[key]["vs_plain_max_rel"] = float((t - p).abs().max()) / scale
        res[key]["vs_plain_mean_rel"] = float((t - p).abs().mean()) / scale
    out = {"workload": "float32 256^3 segments volume (seed 4), frangi sigmas 1..5, "
                       "27 Gaussian-derivative passes per sigma (taps 143, 23, 35, 47, 57)",
           **res}
    if check:
        from oracle import restate as R

        R.THREADS = os.cpu_count() or 1
        t0 = time.perf_counter()
        exp = R.frangi(vol_h, **kw)
        cpu_s = time.perf_counter() - t0
        out["oracle"] = frangi_agreement(outs["plain_f32"].cpu().numpy(), exp)
        out["cpu_baseline"] = {"value": vol_h.size / cpu_s / 1e9, "unit": "Gvox/s",
                               "cores": R.THREADS, "kind": "port",
                               "sample": f"the whole 256^3 volume, {cpu_s:.1f} s"}
    return out


# ------------------------------------------------------------- CPU leg

def cpu_baseline(x_host, slab_z=8, threads=None):
    """The oracle (exact restatement of cuCIM's arithmetic, C + OpenMP) on a
    slab of the stack: the first `slab_z` z-slices with the full y, x extent
    (the CPU arm's sample)."""
    from oracle import restate as R

    threads = threads or os.cpu_count() or 1
    R.THREADS = threads
    xs = np.ascontiguousarray(x_host[:slab_z])
    t = time.perf_counter()
    R.gaussian_filter(xs, (1, 2, 2), mode="mirror", output=np.float32)
    for a in range(3):
        R.sobel(xs, a, output=np.float32)
    R.uniform_filter(xs, 5, output=np.uint16)
    dt = time.perf_counter() - t
    return {"value": xs.size / dt / 1e9, "unit": "Gvox/s", "cores": threads, "kind": "port",
            "sample": f"z-slab {xs.shape} of the stack, all five filters, {dt:.2f} s"}


def run_reference(args, world):
    """CPU arm: the oracle on the host cores, same workload, metric and
    config; each step filters the first 8 z-slices of the stack (regenerated
    on the CPU by the same generator: bit-identical to those slices of the
    GPU arm's stack). Imports nothing from the cucim_b200 package."""
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else SHAPE
    from oracle import restate as R

    threads = os.cpu_count() or 1
    R.THREADS = threads
    S = load_synthetic()
    sample_z = min(8, shape[0])
    xs = S.stack_window(0, sample_z, shape, R.gaussian_filter)

    def step():
        for op in ORACLE_STEP:
            op(R, xs)

    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t) / args.steps
    v = xs.size / dt / 1e9
    sample = (f"each step filters the first {sample_z} z-slices {list(xs.shape)} of the stack "
              f"(all five filters), {threads} host threads")
    return {
        "metric": METRIC, "value": v, "unit": "Gvox/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": stack_config(shape, world), "sample": sample,
        "cpu_baseline": {"value": v, "unit": "Gvox/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "Gvox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def per_config_records(res, roof, cpu, peaks):
    """One record per workload: its throughput, roofline, CPU baseline (the
    oracle with all host threads) and parity, side by side."""
    out = {"stack_512x1024x1024_u16": {
        "value": res["value"], "unit": "Gvox/s", "roofline": roof, "cpu_baseline": cpu,
        "parity": (res["parity"] or {}).get("bit_exact")}}
    p2 = res["plain2d"]
    if p2:
        out["gaussian_2048x2048_f32_sigma4"] = {
            "value": p2["gpx_s"], "unit": "Gpx/s",
            "roofline": {"bound": "hbm", "achieved": p2["gb_s"], "peak": peaks.get("hbm_gbs"),
                         "unit": "GB/s", "frac": p2.get("frac_of_hbm")},
            "cpu_baseline": p2.get("cpu_baseline"), "parity": p2.get("oracle_bit_exact")}
    pr = res["precision"]
    if pr:
        for name, row in pr["filters"].items():
            t = row["tensor_tf32x3"]
            out[f"precision_8192x8192_f32 {name}"] = {
                "value": t["gpx_s"], "unit": "Gpx/s", "plain_f32_gpx_s": row["plain_f32"]["gpx_s"],
                "speedup_vs_plain_f32": row["speedup"],
                "max_rel_err": t["max_rel_err"], "plain_max_rel_err": row["plain_f32"]["max_rel_err"],
                "roofline": {"bound": "tensor", "achieved": t["executed_tflops"],
                             "peak": pr["tf32_peak_tflops"], "unit": "TFLOP/s",
                             "frac": t.get("frac_of_tf32_peak")},
                "cpu_baseline": pr.get("cpu_baseline")}
    tl = res["tiles"]
    if tl:
        out["batched_tiles_4096_rgb_u8"] = {
            "value": tl["batched_gpx_s"], "unit": "Gpx/s", "speedup_vs_per_tile": tl["speedup"],
            "roofline": tl.get("roofline"),
            "cpu_baseline": tl.get("cpu_baseline"), "parity": tl.get("oracle_bit_exact")}
    sk = res.get("sk_sobel")
    if sk:
        out["stack_512x1024x1024_u16 skimage sobel(axis=0,1,2)"] = {
            "value": sk["gvox_s"], "unit": "Gvox/s",
            "roofline": {"bound": "hbm", "achieved": sk["algorithmic_gbs"],
                         "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": sk["algorithmic_gbs"] / peaks["hbm_gbs"]
                         if peaks.get("hbm_gbs") else None},
            "parity": sk["oracle_bit_exact"]}
    fr = res["frangi"]
    if fr:
        out["frangi_256cube_sigmas1to5"] = {
            "value": fr["plain_f32"]["gvox_s"], "unit": "Gvox/s",
            "cpu_baseline": fr.get("cpu_baseline"), "parity": fr.get("oracle")}
    return out


def _peaks():
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return json.load(open(pk)) if os.path.exists(pk) else {}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, world)))
        return
    import torch
    import torch.distributed as dist

    if args.skip_main:
        from cucim_b200 import ndimage as ndi

        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        if rank == 0:
            out = {}
            if not args.no_precision:
                out["precision_path"] = run_precision(
                    torch, ndi, dev, size=args.precision_size,
                    tf32_peak=_peaks().get("bf16_tflops", 1590.0) / 2)
            if not args.no_tiles:
                out["batched_tiles"] = run_tiles(torch, dev, n_tiles=args.tiles)
            if not args.no_frangi:
                out["frangi"] = run_frangi(torch, dev)
            if not args.no_plain2d:
                out["plain_2d_gaussian"] = run_plain2d(torch, dev, hbm_gbs=_peaks().get("hbm_gbs"))
            print(json.dumps(out))
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = run_ours(args, rank, world, local_rank)
    if rank == 0:
        peaks = _peaks()
        hbm = peaks.get("hbm_gbs", 6650.0)
        # dominant kernel: largest share of the step
        name, kr = max(res["kernels"].items(),
                       key=lambda kv: kv[1]["ms"] * kv[1]["launches_per_step"])
        roof = {"bound": "hbm", "kernel": name, "achieved": kr["gbs"], "peak": hbm,
                "unit": "GB/s", "frac": kr["gbs"] / hbm, "traffic": None,
                "peak_source": "measured" if peaks else "fallback"}
        if name in TRAFFIC and args.shape is None:
            # DRAM bytes of the same kernel captured by ncu on a smaller stack,
            # scaled to the 512-slice launch (traffic grows with the slices)
            tb, slices, prof = TRAFFIC[name]
            roof["traffic"] = tb * SHAPE[0] / slices
            roof["traffic_source"] = (f"ncu dram__bytes_read + dram__bytes_write of the same kernel on "
                                      f"{slices} x 1024 x 1024, x 512/{slices} (profiles/{prof})")
        cpu = None
        if not args.no_cpu:
            cpu = cpu_baseline(res["x"].numpy())
        line = {
            "metric": METRIC, "value": res["value"], "unit": "Gvox/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": stack_config(tuple(res["x"].shape), world),
            "roofline": roof, "kernels": res["kernels"], "cpu_baseline": cpu,
            "e2e": res["e2e"], "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "clocks": res["clocks"], "parity": res["parity"],
            "autotune": {"note": "schedules chosen by the autotuner (first warm-up step; "
                                 "all bit-identical), flags = CIMX_L_* bits",
                         "entries": res["autotune"]},
            "per_config": per_config_records(res, roof, cpu, peaks),
            "precision_path": res["precision"],
            "batched_tiles": res["tiles"], "frangi": res["frangi"],
            "plain_2d_gaussian": res["plain2d"],
            "skimage_sobel_axes": res["sk_sobel"],
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
