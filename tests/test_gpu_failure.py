"""Failure detection on the GPU without a GPU fault.

- Bounded device-side waits: cimx_wait_selftest makes the wait helper of the
  TMA-fed kernels (poll-count bound) and of the tensor-core pass
  (%globaltimer bound) wait on an mbarrier that nothing arrives on. The wait
  must run out, record CIMX_E_TIMEOUT in the status word that
  cimx_device_status() reads, and return, leaving the context usable: a
  filter afterwards still matches the oracle.
- A refused scratch allocation: with an allocator hook that returns NULL, a
  filter that needs the ping-pong buffer raises MemoryError (CIMX_E_NOMEM)
  and leaves its output untouched; with the default allocator restored the
  same call succeeds.
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


def _filter_still_works(cuda):
    from cucim_b200 import ndimage as ndi

    x = np.random.default_rng(5).integers(0, 65536, (6, 40, 64)).astype(np.uint16)
    got = ndi.gaussian_filter(torch.as_tensor(x).to(cuda), (1, 2, 2), mode="mirror",
                              output=np.float32)
    np.testing.assert_array_equal(
        got.cpu().numpy(), R.gaussian_filter(x, (1, 2, 2), mode="mirror", output=np.float32))


@pytest.mark.parametrize("which,limit", [(0, 1 << 12), (1, 200_000)])
def test_bounded_wait_runs_out_and_reports_timeout(cuda, which, limit):
    from cucim_b200 import _lib

    torch.cuda.synchronize()
    assert _lib.lib.cimx_device_status(1) in (0, _lib.E_TIMEOUT)  # clear
    assert _lib.lib.cimx_device_status(0) == 0
    rc = _lib.lib.cimx_wait_selftest(which, limit, None)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()  # the kernel ended: the wait was bounded
    assert _lib.lib.cimx_device_status(1) == _lib.E_TIMEOUT
    assert _lib.lib.cimx_device_status(0) == 0
    _filter_still_works(cuda)
    assert _lib.lib.cimx_device_status(0) == 0


def test_refused_allocation_raises_memory_error(cuda):
    from cucim_b200 import _lib
    from cucim_b200 import ndimage as ndi

    x = torch.as_tensor(np.random.default_rng(6).random((48, 80), dtype=np.float32)).to(cuda)
    out = torch.full_like(x, 7.0)
    calls = []
    alloc = _ALLOC(lambda n, s, u: calls.append(n) or None)
    free = _FREE(lambda p, n, s, u: None)
    _lib.lib.cimx_set_allocator(ctypes.cast(alloc, ctypes.c_void_p),
                                ctypes.cast(free, ctypes.c_void_p), None)
    try:
        with ndi.pass_by_pass(), pytest.raises(MemoryError):
            ndi.gaussian_filter(x, 2.0, output=out)
    finally:
        _lib.lib.cimx_set_allocator(None, None, None)
    assert calls, "the allocator hook was not consulted"
    torch.cuda.synchronize()
    assert bool((out == 7.0).all()), "a refused call wrote its output"
    with ndi.pass_by_pass():
        ndi.gaussian_filter(x, 2.0, output=out)
    np.testing.assert_array_equal(out.cpu().numpy(),
                                  R.gaussian_filter(x.cpu().numpy(), 2.0))
