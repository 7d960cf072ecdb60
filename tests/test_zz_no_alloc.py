"""cimx_separable_noalloc: the separable filter for callers that cannot
allocate device memory (code inside another component's stream capture,
plug-ins whose host owns every allocation, pipelines that forbid allocation
after start-up). Its ping-pong intermediate lives in a static device array
instead of coming from an allocator.

Checked through the C ABI against cimx_separable, the entry point that
allocates, on two calls in a row with different inputs (the static array
keeps the first call's contents when the second starts). Separable filters in
this suite are compared bit for bit, so the tolerance is exact equality.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _passes(ndi, in_dtype, out_dtype, ndim, sigma, mode):
    specs = ndi._gaussian_specs(ndim, in_dtype, sigma, 0, mode, 4.0, None, None)
    return ndi._build_passes(in_dtype, out_dtype, ndim, specs, 0.0, None)


def _run(entry, x, out, pl, arrays, lib):
    a_in, a_out = arrays.to_cimx(x), arrays.to_cimx(out)
    args = [ctypes.byref(a_in), ctypes.byref(a_out), pl.array(), len(pl)]
    if entry is lib.lib.cimx_separable:
        args.append(0)
    args.append(arrays.stream_of(x))
    return entry(*args)


def test_noalloc_matches_allocating_entry_twice(cuda):
    from cucim_b200 import _arrays, _lib
    from cucim_b200 import ndimage as ndi

    shape = (16, 96, 128)
    pl = _passes(ndi, np.uint16, np.float32, 3, (1.0, 2.0, 2.0), "mirror")
    rng = np.random.default_rng(7)
    for call in range(2):
        x = torch.as_tensor(rng.integers(0, 65536, shape).astype(np.uint16)).to(cuda)
        ref = torch.empty(shape, dtype=torch.float32, device=cuda)
        got = torch.full(shape, float("nan"), dtype=torch.float32, device=cuda)
        rc = _run(_lib.lib.cimx_separable, x, ref, pl, _arrays, _lib)
        assert rc == 0, _lib.last_error()
        rc = _run(_lib.lib.cimx_separable_noalloc, x, got, pl, _arrays, _lib)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got.cpu().numpy(), ref.cpu().numpy(),
                                      err_msg=f"call {call}")


def test_noalloc_rejects_oversized_requests(cuda):
    from cucim_b200 import _lib
    from cucim_b200 import ndimage as ndi

    # an intermediate larger than the 64 MiB static array (fake pointers: the
    # request is rejected before any device access)
    shape = (64, 512, 520)
    pl = _passes(ndi, np.float32, np.float32, 3, 1.0, "reflect")

    def desc(ptr):
        a = _lib.CimxArray()
        a.data, a.dtype, a.ndim = ptr, ord("f"), 3
        acc = 4
        for d in (2, 1, 0):
            a.shape[d] = shape[d]
            a.strides[d] = acc
            acc *= shape[d]
        return a

    a_in, a_out = desc(0x10000000), desc(0x90000000)
    rc = _lib.lib.cimx_separable_noalloc(ctypes.byref(a_in), ctypes.byref(a_out), pl.array(),
                                         len(pl), None)
    assert rc == _lib.E_INVALID
    assert "static scratch" in _lib.last_error()
