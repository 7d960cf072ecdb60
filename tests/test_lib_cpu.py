"""libcimx.so without a GPU: it loads, exports every entry point that
include/cimx.h declares, rejects bad arguments before touching the device,
and the Python host logic agrees with the oracle's restatement."""

import ctypes
import os
import re

import numpy as np
import pytest

from cucim_b200 import _lib, _util
from cucim_b200 import ndimage as ndi
from oracle import restate as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "cimx.h")).read()
    return re.findall(r"CIMX_API\s+[\w\s\*]+?\b(cimx_\w+)\s*\(", text)


def test_every_declared_symbol_is_exported():
    names = _declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(_lib.lib, n), n
        assert n in _lib.EXPORTED, f"{n} has no ctypes signature"


def test_abi_version():
    assert _lib.lib.cimx_abi_version() == 101


def _arr(shape, dtype, ptr=0x1000, strides=None):
    a = _lib.CimxArray()
    a.data = ptr
    a.dtype = ord(np.dtype(dtype).char)
    a.ndim = len(shape)
    es = np.dtype(dtype).itemsize
    if strides is None:
        strides, acc = [], es
        for n in reversed(shape):
            strides.insert(0, acc)
            acc *= n
    for d, (n, s) in enumerate(zip(shape, strides)):
        a.shape[d] = n
        a.strides[d] = s
    return a


def _corr(a_in, a_out, K=3, axis=0, origin=0, mode=0):
    t, p = _lib.taps_pointer(np.ones(K))
    return _lib.lib.cimx_correlate1d(ctypes.byref(a_in), ctypes.byref(a_out), p, K, axis,
                                     origin, mode, 0.0, 0, None)


def test_validation_happens_before_device_work():
    good_in = _arr((4, 5), np.float32, 0x1000)
    good_out = _arr((4, 5), np.float32, 0x9000)
    assert _corr(good_in, _arr((4, 6), np.float32, 0x9000)) == _lib.E_INVALID
    assert "shape" in _lib.last_error()
    assert _corr(good_in, _arr((4, 5), np.bool_, 0x9000)) == _lib.E_DTYPE
    # complex input needs a complex output (refused before any device work)
    assert _corr(_arr((4, 5), np.complex64, 0x1000), good_out) == _lib.E_DTYPE
    assert "complex" in _lib.last_error()
    # complex64 overlaps by its 8-byte elements
    assert _corr(_arr((4, 5), np.complex64, 0x1000),
                 _arr((4, 5), np.complex64, 0x1000 + 8 * 19)) == _lib.E_INVALID
    assert _corr(_arr((4, 5), np.float32, 0x1000, strides=(4, 16)), good_out) == _lib.E_LAYOUT
    assert _corr(good_in, good_out, K=3, origin=2) == _lib.E_INVALID
    assert "origin" in _lib.last_error()
    assert _corr(good_in, good_out, mode=9) == _lib.E_INVALID
    assert _corr(good_in, good_out, axis=2) == _lib.E_INVALID
    assert _corr(good_in, _arr((4, 5), np.float32, 0x1004)) == _lib.E_INVALID  # overlap
    assert _corr(good_in, good_out, K=0) == _lib.E_INVALID


def test_check_maps_errors_like_cucim():
    with pytest.raises(MemoryError):
        _lib.check(_lib.E_NOMEM, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.E_CUDA, "x")


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("K", [3, 33, 200, 257])
@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32, np.float64])
@pytest.mark.parametrize("mode,cval", [("reflect", 0.0), ("constant", -1.0),
                                       ("constant", np.nan), ("constant", 2.0)])
def test_algorithm_choice_matches_oracle(ndim, K, dtype, mode, cval):
    for axis in range(ndim):
        anchor = K // 2
        assert _util.choose_algorithm(ndim, axis, K, anchor, mode, cval, dtype) == \
            R.choose_path(ndim, axis, K, anchor, mode, cval, dtype)


@pytest.mark.parametrize("sigma", [0.5, 1.0, 0.7071067811865476, 3.3, 16.0, 32.0])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_gaussian_taps_match_oracle(sigma, order):
    r = int(4.0 * sigma + 0.5)
    a = ndi._gaussian_kernel1d(sigma, order, r, np.float32)
    b = R.gaussian_kernel1d(sigma, order, r, np.float32)
    assert a.dtype == b.dtype
    np.testing.assert_array_equal(a, b)


def test_pass_flags():
    f = _util.pass_flags(np.uint16, 3, 0, 9, 0, "mirror", 0.0, np.float64, False, None)
    assert f & _lib.F_SKIP_ZERO_TAPS and not f & _lib.F_W64
    f = _util.pass_flags(np.float64, 2, 0, 9, 0, "mirror", 0.0, np.float64, True, None)
    assert f & _lib.F_CVAL_AS_INPUT and f & _lib.F_W64 and f & _lib.F_CONVOLVE
    f = _util.pass_flags(np.int32, 2, 1, 5, 0, "reflect", 0.0, np.float32, False, None)
    assert f & _lib.F_W64  # promote(int32, float32) = float64


def test_modes_and_axes_checks():
    with pytest.raises(RuntimeError):
        _util.check_mode("grid-reflect")
    with pytest.raises(RuntimeError):
        _util.check_mode("bogus")
    with pytest.raises(ValueError):
        _util.check_axes((0, 0), 2)
    assert _util.check_axes(-1, 3) == (-1,)  # scalars are not normalised (UTIL:114-115)
    assert _util.check_axes([-1], 3) == (2,)


_ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)
_FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                         ctypes.c_void_p)


def test_refused_scratch_allocation_is_e_nomem_and_memory_error():
    """An allocator hook that returns NULL: a multi-pass call that needs the
    ping-pong buffer fails with CIMX_E_NOMEM before any device work (the
    pointers here are fake), and the Python layer turns it into MemoryError."""
    calls = []
    alloc = _ALLOC(lambda n, s, u: calls.append(n) or None)
    free = _FREE(lambda p, n, s, u: None)
    _lib.lib.cimx_set_allocator(ctypes.cast(alloc, ctypes.c_void_p),
                                ctypes.cast(free, ctypes.c_void_p), None)
    try:
        a_in = _arr((6, 7), np.float32, 0x1000)
        a_out = _arr((6, 7), np.float32, 0x9000)
        t, p = _lib.taps_pointer(np.ones(3))
        passes = (_lib.CimxPass * 2)()
        for i in range(2):
            passes[i].axis, passes[i].ntaps, passes[i].mode, passes[i].taps = i, 3, 0, p
        rc = _lib.lib.cimx_separable(ctypes.byref(a_in), ctypes.byref(a_out), passes, 2,
                                     _lib.L_NO_FUSION, None)
        assert rc == _lib.E_NOMEM
        assert calls == [6 * 7 * 4]
        with pytest.raises(MemoryError):
            _lib.check(rc, "separable")
    finally:
        _lib.lib.cimx_set_allocator(None, None, None)


def test_wait_selftest_rejects_bad_arguments():
    assert _lib.lib.cimx_wait_selftest(2, 10, None) == _lib.E_INVALID
    assert _lib.lib.cimx_wait_selftest(0, 0, None) == _lib.E_INVALID
    assert _lib.lib.cimx_wait_selftest(0, 1 << 25, None) == _lib.E_INVALID
    assert _lib.lib.cimx_wait_selftest(1, 10 ** 9, None) == _lib.E_INVALID


@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_c_gaussian_taps_match_numpy(order):
    """cimx_gaussian_taps (float64 taps generated in the library, for hosts
    without numpy) against the numpy taps the Python layer uses: bit for bit
    once rounded to float32, and within 5 ulp in float64 (orders 0-2; order 3
    within 11 ulp of the largest tap): numpy's own exp() differs from the C
    library's in the last bit on AVX-512 hosts."""
    for s in list(np.linspace(0.3, 40, 61)) + [16.0, 32.0, 2 ** -0.5, 3 * 2 ** -0.5]:
        for trunc in (4.0, 8.0, 100.0):
            r = int(trunc * s + 0.5)
            if r <= 0 or r > 2000:
                continue
            ref = ndi._gaussian_taps(float(s), order, r, np.float64)
            got = np.empty(2 * r + 1)
            rc = _lib.lib.cimx_gaussian_taps(float(s), order, r,
                                             got.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            assert rc == 0
            np.testing.assert_array_equal(got.astype(np.float32), ref.astype(np.float32))
            if order < 2:
                ulps = np.abs(got - ref) / np.spacing(np.abs(ref))
                assert ulps.max() <= 5, (s, r, ulps.max())
            else:
                assert (np.abs(got - ref) / np.spacing(np.abs(ref).max())).max() <= 11


def test_c_entries_reject_bad_arguments():
    a = _arr((6, 7), np.float32, 0x1000)
    b = _arr((6, 7), np.float32, 0x9000)
    sig = (ctypes.c_double * 2)(1.0, 1.0)
    modes = (ctypes.c_int * 2)(0, 0)
    axes = (ctypes.c_int * 2)(0, 0)
    rc = _lib.lib.cimx_gaussian_nd(ctypes.byref(a), ctypes.byref(b), sig, None, None, modes,
                                   axes, 2, 4.0, 0.0, 0, 0, None)
    assert rc == _lib.E_INVALID and "unique" in _lib.last_error()
    rc = _lib.lib.cimx_gaussian_nd(ctypes.byref(a), ctypes.byref(b), sig, None, None, modes,
                                   None, 1, 4.0, 0.0, 0, 0, None)
    assert rc == _lib.E_INVALID
    bad_modes = (ctypes.c_int * 2)(0, 9)
    rc = _lib.lib.cimx_sobel_nd(ctypes.byref(a), ctypes.byref(b), 0, bad_modes, 0.0, 0, 0, 0,
                                None)
    assert rc == _lib.E_INVALID and "mode" in _lib.last_error()
    rc = _lib.lib.cimx_frangi(ctypes.byref(_arr((6,), np.float32, 0x1000)),
                              ctypes.byref(_arr((6,), np.float32, 0x9000)), sig, 1, 0.5, 0.5,
                              float("nan"), 1, 0, 0.0, 0, None)
    assert rc == _lib.E_INVALID and "2-dimensional or 3-dimensional" in _lib.last_error()
    u8 = _arr((6, 7), np.uint8, 0x9000)
    rc = _lib.lib.cimx_gaussian_nd(ctypes.byref(a), ctypes.byref(u8), sig, None, None,
                                   (ctypes.c_int * 2)(4, 4), None, 2, 4.0, float("nan"), 0, 0,
                                   None)
    assert rc == _lib.E_INVALID and "Non-finite cval" in _lib.last_error()
    rc = _lib.lib.cimx_uniform_nd(ctypes.byref(a), ctypes.byref(b), (ctypes.c_int * 2)(3, 3),
                                  modes, (ctypes.c_int * 2)(2, 0), None, 2, 0.0, 0, 0, None)
    assert rc == _lib.E_INVALID and "origin" in _lib.last_error()


def test_complex_pass_list():
    """Complex taps travel as (re, im) pairs with ntaps = their count, the
    complex-taps flag set and W = complex<float> / complex<double> by cuCIM's
    rule (UTIL:35-37)."""
    from cucim_b200 import ndimage

    w = np.array([0.2 + 0.1j, -0.5 + 0.3j, 0.0, 0.1 - 0.05j])
    pl = ndimage._build_passes(np.dtype(np.complex64), np.dtype(np.complex64), 1,
                               [(0, w, "reflect", 1, False)], 0.0, None)
    p = pl.items[0]
    assert p.ntaps == 4 and p.origin == 1
    assert p.flags & _lib.F_COMPLEX_TAPS and not p.flags & _lib.F_W64
    assert [p.taps[i] for i in range(8)] == [0.2, 0.1, -0.5, 0.3, 0.0, 0.0, 0.1, -0.05]
    pl = ndimage._build_passes(np.dtype(np.int32), np.dtype(np.complex128), 2,
                               [(1, np.ones(3), "reflect", 0, False)], 0.0, None)
    p = pl.items[0]
    assert p.ntaps == 3 and not p.flags & _lib.F_COMPLEX_TAPS
    pl = ndimage._build_passes(np.dtype(np.complex128), np.dtype(np.complex128), 2,
                               [(1, np.ones(3), "reflect", 0, False)], 0.0, None)
    assert pl.items[0].flags & _lib.F_W64
