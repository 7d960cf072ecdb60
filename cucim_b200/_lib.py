"""ctypes binding of libcimx.so (the C ABI declared in include/cimx.h).

The shared library is built in-tree by ``cucim_b200/build.py``. There is no
fallback: if the library is missing, importing this module raises.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcimx.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libcimx.so not found at {LIB_PATH}; build it with "
        "`python cucim_b200/build.py` (nvcc, sm_100a)"
    )

lib = ctypes.CDLL(LIB_PATH)

MAX_NDIM = 8

MODE_CODES = {
    "reflect": 0,
    "grid-mirror": 0,
    "mirror": 1,
    "nearest": 2,
    "grid-wrap": 3,
    "wrap": 3,
    "constant": 4,
}

F_W64 = 1 << 0
F_CONVOLVE = 1 << 1
F_CVAL_AS_INPUT = 1 << 2
F_SKIP_ZERO_TAPS = 1 << 3
F_COMPLEX_TAPS = 1 << 4
L_NO_FUSION = 1 << 0
L_TENSOR_BF16X3 = 1 << 1
L_TENSOR_TF32X3 = 1 << 2
L_TENSOR_ALL_LINES = 1 << 3
L_NO_VOLUME = 1 << 4
L_NO_STREAM = 1 << 5
L_NO_ROWSTREAM = 1 << 6
L_NO_TUNE = 1 << 7
L_ZCHUNK_SHIFT = 8
L_SLAB_SPAN_SHIFT = 10

E_INVALID, E_DTYPE, E_CUDA, E_NOMEM, E_LAYOUT, E_TIMEOUT = -1, -2, -3, -4, -5, -6


class CimxArray(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("shape", ctypes.c_int64 * MAX_NDIM),
        ("strides", ctypes.c_int64 * MAX_NDIM),
    ]


class CimxBatchTile(ctypes.Structure):
    _fields_ = [
        ("rgb", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("ntaps", ctypes.c_int32),
        ("taps_offset", ctypes.c_int32),
        ("first_block", ctypes.c_int64),
        ("rgb_pitch", ctypes.c_int64),
        ("out_pitch", ctypes.c_int64),
    ]


class CimxPass(ctypes.Structure):
    _fields_ = [
        ("axis", ctypes.c_int32),
        ("ntaps", ctypes.c_int32),
        ("origin", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("cval", ctypes.c_double),
        ("flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("taps", ctypes.POINTER(ctypes.c_double)),
    ]


_P = ctypes.POINTER
_A = _P(CimxArray)
_sigs = {
    "cimx_abi_version": ([], ctypes.c_int),
    "cimx_last_error_string": ([], ctypes.c_char_p),
    "cimx_set_allocator": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "cimx_device_status": ([ctypes.c_int], ctypes.c_int),
    "cimx_wait_selftest": ([ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p], ctypes.c_int),
    "cimx_tune_mode": ([ctypes.c_int], ctypes.c_int),
    "cimx_tune_load": ([ctypes.c_char_p], ctypes.c_int),
    "cimx_tune_save": ([ctypes.c_char_p], ctypes.c_int),
    "cimx_tune_clear": ([], ctypes.c_int),
    "cimx_tune_dump": ([ctypes.c_char_p, ctypes.c_longlong], ctypes.c_longlong),
    "cimx_correlate1d": (
        [_A, _A, _P(ctypes.c_double), ctypes.c_int, ctypes.c_int, ctypes.c_int,
         ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_separable": (
        [_A, _A, _P(CimxPass), ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_separable_noalloc": (
        [_A, _A, _P(CimxPass), ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_gradient_magnitude": (
        [_A, _A, _P(CimxPass), ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_laplace": (
        [_A, _A, _P(CimxPass), ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_combine": ([_A, _A, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "cimx_square_accumulate": ([_A, _A, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "cimx_sqrt": ([_A, ctypes.c_void_p], ctypes.c_int),
    "cimx_unsharp": (
        [_A, _A, _A, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
         ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_any_negative": ([_A, _P(ctypes.c_int), ctypes.c_void_p], ctypes.c_int),
    "cimx_min_max_1d": (
        [_A, _A, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
         ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_eigvals_sym": (
        [_A, ctypes.c_int, _A, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_rgb2gray": ([_A, _A, ctypes.c_void_p], ctypes.c_int),
    "cimx_convert": ([_A, _A, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "cimx_gradient_fd": ([_A, _A, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "cimx_batch_gray_gauss_sobel": (
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
         _P(ctypes.c_float), _P(ctypes.c_float), ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_gaussian_taps": (
        [ctypes.c_double, ctypes.c_int, ctypes.c_int, _P(ctypes.c_double)], ctypes.c_int,
    ),
    "cimx_gaussian_nd": (
        [_A, _A, _P(ctypes.c_double), _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_int),
         _P(ctypes.c_int), ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
         ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_uniform_nd": (
        [_A, _A, _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_int),
         ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_sobel_nd": (
        [_A, _A, ctypes.c_int, _P(ctypes.c_int), ctypes.c_double, ctypes.c_int, ctypes.c_int,
         ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_gaussian_gradient_magnitude_nd": (
        [_A, _A, _P(ctypes.c_double), _P(ctypes.c_int), ctypes.c_double, ctypes.c_double,
         ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_hessian": (
        [_A, _A, ctypes.c_int, _P(ctypes.c_double), ctypes.c_int, ctypes.c_double, ctypes.c_int,
         ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_frangi": (
        [_A, _A, _P(ctypes.c_double), ctypes.c_int, ctypes.c_double, ctypes.c_double,
         ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
         ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_meijering_accumulate": (
        [_A, ctypes.c_int, _A, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_sato_accumulate": (
        [_A, ctypes.c_int, _A, ctypes.c_double, ctypes.c_int, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_nonpositive_to_one": ([_A, ctypes.c_void_p], ctypes.c_int),
    "cimx_mask_erode_multiply": ([_A, _A, ctypes.c_void_p], ctypes.c_int),
    "cimx_multiply": ([_A, _A, _A, ctypes.c_void_p], ctypes.c_int),
    "cimx_corner_response": (
        [ctypes.c_int, _A, ctypes.c_int, _A, _A, ctypes.c_double, ctypes.c_void_p], ctypes.c_int,
    ),
    "cimx_ridge_filter": (
        [_A, _A, ctypes.c_int, _P(ctypes.c_double), ctypes.c_int, ctypes.c_double,
         ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
         ctypes.c_int, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_frangi_hessian_accumulate": (
        [_A, ctypes.c_int, _A, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p],
        ctypes.c_int,
    ),
    "cimx_frangi_accumulate": (
        [_A, ctypes.c_int, _A, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p],
        ctypes.c_int,
    ),
}
for _name, (_args, _res) in _sigs.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res

EXPORTED = tuple(_sigs)

COMBINE_ADD = 0
COMBINE_SUBTRACT = 1

CORNER_KITCHEN_ROSENFELD, CORNER_HARRIS_K, CORNER_HARRIS_EPS, CORNER_SHI_TOMASI, \
    CORNER_FOERSTNER = range(5)


def last_error():
    msg = lib.cimx_last_error_string()
    return msg.decode() if msg else ""


def check(rc, what):
    """Raise the exception cuCIM raises for the condition behind `rc`."""
    if rc == 0:
        return
    msg = last_error() or what
    if rc == E_NOMEM:
        raise MemoryError(msg)
    if rc == E_DTYPE:
        raise TypeError(msg)
    if rc == E_INVALID and "origin" in msg:
        raise ValueError(msg)
    raise RuntimeError(f"{what}: {msg}")


def taps_pointer(taps):
    """A float64 C-contiguous copy of `taps` and a pointer into it; complex
    taps become (re, im) pairs (CIMX_F_COMPLEX_TAPS)."""
    taps = np.asarray(taps)
    if taps.dtype.kind == "c":
        t = np.ascontiguousarray(taps, dtype=np.complex128).view(np.float64)
    else:
        t = np.ascontiguousarray(taps, dtype=np.float64)
    return t, t.ctypes.data_as(_P(ctypes.c_double))
