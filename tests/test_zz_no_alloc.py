"""cimx_separable_noalloc: the separable filter for callers that cannot
allocate device memory (code inside another component's stream capture,
plug-ins whose host owns every allocation, pipelines that forbid allocation
after start-up). Its ping-pong intermediate lives in a static device array
instead of coming from an allocator.

Checked through the C ABI, on two calls in a row with different inputs (the
static array keeps the first call's contents when the second starts), for
one pass (no intermediate), two passes (the first pass writes the static
array) and three passes (the first pass writes the output), against the
oracle and against cimx_separable, the entry point that allocates. Separable
filters in this suite are compared bit for bit, so the tolerance is exact
equality. While the entry point runs, an allocator that counts its calls and
refuses every request is installed: a call that reached for scratch memory
would fail or show in the count.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

_ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)
_FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                         ctypes.c_void_p)


class _RefusingAllocator:
    """Installs an allocator hook that counts its calls and returns NULL."""

    def __init__(self, lib):
        self.lib = lib
        self.calls = 0

        def alloc(nbytes, stream, user):
            self.calls += 1
            return None

        def free(ptr, nbytes, stream, user):
            self.calls += 1

        self._a, self._f = _ALLOC(alloc), _FREE(free)

    def __enter__(self):
        self.lib.lib.cimx_set_allocator(ctypes.cast(self._a, ctypes.c_void_p),
                                        ctypes.cast(self._f, ctypes.c_void_p), None)
        return self

    def __exit__(self, *exc):
        self.lib.lib.cimx_set_allocator(None, None, None)  # back to the default


def _passes(ndi, in_dtype, out_dtype, ndim, sigma, mode, axes=None):
    specs = ndi._gaussian_specs(ndim, in_dtype, sigma, 0, mode, 4.0, None, axes)
    return ndi._build_passes(in_dtype, out_dtype, ndim, specs, 0.0, None)


def _call(entry, x, out, pl, lib_flags=None):
    from cucim_b200 import _arrays

    a_in, a_out = _arrays.to_cimx(x), _arrays.to_cimx(out)
    args = [ctypes.byref(a_in), ctypes.byref(a_out), pl.array(), len(pl)]
    if lib_flags is not None:
        args.append(lib_flags)
    args.append(_arrays.stream_of(x))
    return entry(*args)


# (shape, in dtype, out dtype, sigma, mode, axes, expected pass count)
CASES = [
    ((16, 96, 128), np.uint16, np.float32, (1.0, 2.0, 2.0), "mirror", None, 3),
    ((200, 300), np.float32, np.float32, 3.0, "reflect", None, 2),
    ((37, 41), np.uint8, np.uint8, 1.5, "constant", None, 2),
    ((64, 130), np.float32, np.float32, 2.0, "nearest", (1,), 1),
    ((9, 20, 33), np.uint16, np.uint16, 1.0, "wrap", (0,), 1),
]


def _input(shape, dtype, rng):
    if np.dtype(dtype).kind == "f":
        return rng.random(shape, dtype=np.float32).astype(dtype)
    return rng.integers(0, np.iinfo(dtype).max + 1, shape).astype(dtype)


@pytest.mark.parametrize("shape,tin,tout,sigma,mode,axes,npasses", CASES)
def test_noalloc_matches_oracle_and_allocating_entry_twice(cuda, shape, tin, tout, sigma, mode,
                                                           axes, npasses):
    from cucim_b200 import _lib
    from cucim_b200 import ndimage as ndi

    pl = _passes(ndi, tin, tout, len(shape), sigma, mode, axes)
    assert len(pl) == npasses
    rng = np.random.default_rng(7)
    for call in range(2):
        x = _input(shape, tin, rng)
        xd = torch.as_tensor(x).to(cuda)
        ref = torch.empty(shape, dtype=getattr(torch, np.dtype(tout).name), device=cuda)
        got = torch.full_like(ref, 0)
        got.view(torch.uint8).fill_(0xA5)  # garbage the call must overwrite
        rc = _call(_lib.lib.cimx_separable, xd, ref, pl, lib_flags=_lib.L_NO_FUSION)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        with _RefusingAllocator(_lib) as hook:
            rc = _call(_lib.lib.cimx_separable_noalloc, xd, got, pl)
            assert rc == 0, _lib.last_error()
            torch.cuda.synchronize()
        assert hook.calls == 0, "the no-allocation entry point called the allocator"
        exp = R.gaussian_filter(x, sigma, mode=mode, output=tout, axes=axes)
        np.testing.assert_array_equal(got.cpu().numpy(), exp, err_msg=f"oracle, call {call}")
        np.testing.assert_array_equal(got.cpu().numpy(), ref.cpu().numpy(),
                                      err_msg=f"allocating entry, call {call}")


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

    # too many taps for the launch parameters
    long_pass = _lib.CimxPass()
    taps = np.ones(1025)
    long_pass.axis, long_pass.ntaps, long_pass.mode = 2, 1025, 0
    long_pass.taps = taps.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    arr = (_lib.CimxPass * 1)(long_pass)
    rc = _lib.lib.cimx_separable_noalloc(ctypes.byref(a_in), ctypes.byref(a_out), arr, 1, None)
    assert rc == _lib.E_INVALID
    assert "launch parameters" in _lib.last_error()
