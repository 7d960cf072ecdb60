"""The autotuner on the GPU: tuning a call signature records one table
entry, and the result of the tuned schedule is bit-identical to the oracle
and to every forced schedule (volume kernel or not, stream or generic
leading passes, row stream or slab, z chunks, slabs per CTA, one launch
per pass). A later
call of the same signature uses the entry without timing again. With
algorithm="tensor" the tuner may also pick the plain passes; either result
stays within the tensor path's tolerance."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cuda):
    from cucim_b200 import _lib, tune
    from cucim_b200 import ndimage as ndi

    return ndi, tune, _lib


def _schedules(lib):
    z, sp = lib.L_ZCHUNK_SHIFT, lib.L_SLAB_SPAN_SHIFT
    return [lib.L_NO_FUSION, lib.L_NO_VOLUME, lib.L_NO_ROWSTREAM, lib.L_NO_STREAM,
            lib.L_NO_VOLUME | lib.L_NO_ROWSTREAM, lib.L_NO_VOLUME | lib.L_NO_STREAM,
            1 << z, 2 << z, 3 << z, 1 << sp, 2 << sp, 3 << sp,
            lib.L_NO_VOLUME | lib.L_NO_ROWSTREAM | (3 << sp)]


def _u16(shape, seed):
    return np.random.default_rng(seed).integers(0, 65536, shape).astype(np.uint16)


def _f32(shape, seed):
    return np.random.default_rng(seed).random(shape, dtype=np.float32)


WORKLOADS = [
    ("gaussian u16->f32 (1,2,2)", lambda: _u16((24, 96, 128), 1),
     lambda f, x: f.gaussian_filter(x, (1, 2, 2), mode="mirror", output=np.float32)),
    ("sobel u16->f32", lambda: _u16((24, 96, 128), 2),
     lambda f, x: f.sobel(x, 1, output=np.float32)),
    ("uniform u16->u16 5", lambda: _u16((24, 96, 128), 3),
     lambda f, x: f.uniform_filter(x, 5, output=np.uint16)),
    ("gaussian f32 2-D sigma 4", lambda: _f32((300, 260), 4),
     lambda f, x: f.gaussian_filter(x, 4.0, mode="reflect")),
    ("gaussian f32 3-D sigma 3", lambda: _f32((20, 40, 64), 5),
     lambda f, x: f.gaussian_filter(x, 3.0)),
    ("prewitt u8->u8 3-D", lambda: _u16((12, 33, 40), 6).astype(np.uint8),
     lambda f, x: f.prewitt(x, 0)),
]


@pytest.mark.parametrize("name,make,call", WORKLOADS, ids=[w[0] for w in WORKLOADS])
def test_tuned_schedule_is_bit_identical(mods, name, make, call):
    ndi, tune, lib = mods
    x = make()
    xd = torch.as_tensor(x).cuda()
    exp = call(R, x)
    tune.clear()
    with tune.tuning(tune.ON):
        got = call(ndi, xd).cpu().numpy()
    n = len(tune.entries())
    assert n >= 1, "tuning recorded nothing"
    np.testing.assert_array_equal(got, exp)
    for flags in _schedules(lib):
        with ndi.schedule(flags):
            np.testing.assert_array_equal(call(ndi, xd).cpu().numpy(), exp,
                                          err_msg=f"schedule {flags:#x}")
    with tune.tuning(tune.USE):
        again = call(ndi, xd).cpu().numpy()
    assert len(tune.entries()) == n, "a recorded signature was tuned again"
    np.testing.assert_array_equal(again, exp)
    tune.clear()


def test_tuned_tensor_choice_stays_within_tolerance(mods):
    import scipy.ndimage as sndi

    ndi, tune, lib = mods
    x = _f32((64, 4096), 7)
    ref = sndi.gaussian_filter(x.astype(np.float64), 16.0, mode="nearest")
    tune.clear()
    with tune.tuning(tune.ON):
        got = ndi.gaussian_filter(torch.as_tensor(x).cuda(), 16.0, mode="nearest",
                                  algorithm="tensor").cpu().numpy()
    ents = tune.entries()
    assert len(ents) == 1 and ents[0]["candidates"]
    assert np.abs(got - ref).max() / np.abs(ref).max() <= 2e-6
    tune.clear()


def test_tuning_cache_file(mods, tmp_path):
    ndi, tune, lib = mods
    x = torch.as_tensor(_f32((40, 50), 8)).cuda()
    tune.clear()
    with tune.tuning(tune.ON):
        ndi.uniform_filter(x, 7)
    p = tmp_path / "tune.json"
    tune.save(p)
    saved = tune.entries()
    tune.clear()
    tune.load(p)
    assert tune.entries() == saved
    tune.clear()
