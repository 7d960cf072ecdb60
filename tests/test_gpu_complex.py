"""GPU parity of the complex passes (complex64 / complex128 arrays, complex
taps) against the oracle, bit for bit: cuCIM's complex<float> /
complex<double> kernels (_vendored/_ndimage_filters.py:224-244,
_vendored/_ndimage_util.py:35-37, _vendored/_ndimage_filters_core.py:195-203).
The oracle itself is checked against scipy in test_oracle_cpu.py."""

import numpy as np
import pytest
import torch

from oracle import restate as R

pytestmark = pytest.mark.gpu

MODES = ["reflect", "mirror", "nearest", "wrap", "constant"]


@pytest.fixture(scope="module")
def ndi(cuda):
    from cucim_b200 import ndimage

    return ndimage


def _crand(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return v.astype(dtype)


def _same(got, exp):
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else np.asarray(got)
    assert got.dtype == exp.dtype, (got.dtype, exp.dtype)
    # equal parts (NaNs in the same places)
    for a, b in ((got.real, exp.real), (got.imag, exp.imag)):
        assert np.array_equal(a, b, equal_nan=True), np.nanmax(np.abs(a - b))


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("shape,axis", [((257,), 0), ((33, 70), 0), ((33, 70), 1),
                                        ((7, 9, 40), 2), ((7, 9, 40), 0)])
@pytest.mark.parametrize("mode", MODES)
def test_complex_input_real_taps(ndi, dtype, shape, axis, mode):
    x = _crand(shape, dtype, 1)
    w = np.array([0.1, 0.25, 0.3, 0.25, 0.1])
    got = ndi.correlate1d(torch.as_tensor(x).cuda(), w, axis=axis, mode=mode, cval=-0.75)
    _same(got, R.correlate1d(x, w, axis=axis, mode=mode, cval=-0.75))


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128, np.float32, np.float64,
                                   np.uint8, np.int16])
@pytest.mark.parametrize("convolve", [False, True])
@pytest.mark.parametrize("mode", ["reflect", "constant", "wrap"])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_complex_taps(ndi, dtype, convolve, mode, ndim):
    shape = {1: (300,), 2: (40, 52), 3: (6, 10, 37)}[ndim]
    dt = np.dtype(dtype)
    if dt.kind == "c":
        x = _crand(shape, dt, 2)
    elif dt.kind in "iu":
        x = np.random.default_rng(2).integers(0, 100, shape).astype(dt)
    else:
        x = np.random.default_rng(2).standard_normal(shape).astype(dt)
    w = np.array([0.2 + 0.1j, -0.5 + 0.3j, 0.0, 0.1 - 0.05j])
    f = ndi.convolve1d if convolve else ndi.correlate1d
    g = R.convolve1d if convolve else R.correlate1d
    got = f(torch.as_tensor(x).cuda(), w, axis=-1, mode=mode, cval=1.5, origin=1)
    _same(got, g(x, w, axis=-1, mode=mode, cval=1.5, origin=1))


@pytest.mark.parametrize("algorithm", ["shared_memory", "elementwise"])
@pytest.mark.parametrize("mode", MODES)
def test_complex_algorithms(ndi, algorithm, mode):
    """Both kernels of cuCIM: the fill-value rounding and the skipped zero
    taps differ between them."""
    x = _crand((48, 66), np.complex64, 3)
    w = np.array([0.0, 0.3, 0.0, 0.4, 0.3])  # zero taps
    got = ndi.correlate1d(torch.as_tensor(x).cuda(), w, axis=0, mode=mode, cval=0.1,
                          algorithm=algorithm)
    _same(got, R.correlate1d(x, w, axis=0, mode=mode, cval=0.1, algorithm=algorithm))


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_complex_filters(ndi, dtype):
    x = _crand((24, 31, 29), dtype, 4)
    xd = torch.as_tensor(x).cuda()
    _same(ndi.gaussian_filter(xd, (1.0, 2.0, 1.5), mode="mirror"),
          R.gaussian_filter(x, (1.0, 2.0, 1.5), mode="mirror"))
    _same(ndi.gaussian_filter1d(xd, 2.0, axis=1, order=1),
          R.gaussian_filter1d(x, 2.0, axis=1, order=1))
    _same(ndi.uniform_filter(xd, 5, mode="nearest"), R.uniform_filter(x, 5, mode="nearest"))
    x2 = np.ascontiguousarray(x[0])
    _same(ndi.gaussian_filter(torch.as_tensor(x2).cuda(), 3.0),
          R.gaussian_filter(x2, 3.0))


def test_complex_non_finite(ndi):
    """inf in one part contaminates the other through the complex product
    (inf * 0 = nan), as in the complex kernels."""
    x = _crand((5, 40), np.complex64, 5)
    x[2, 7] = complex(np.inf, 1.0)
    x[3, 9] = complex(0.5, np.nan)
    w = np.array([0.25, 0.5, 0.25])
    for algorithm in ("shared_memory", "elementwise"):
        got = ndi.correlate1d(torch.as_tensor(x).cuda(), w, axis=1, algorithm=algorithm)
        _same(got, R.correlate1d(x, w, axis=1, algorithm=algorithm))


def test_complex_output_rules(ndi):
    """_get_output (UTIL:49-71) with a complex result."""
    x = np.random.default_rng(6).standard_normal((10, 12)).astype(np.float32)
    w = np.array([0.5j, 0.5])
    xd = torch.as_tensor(x).cuda()
    assert ndi.correlate1d(xd, w).dtype == torch.complex64
    assert ndi.correlate1d(xd.double(), w).dtype == torch.complex128
    out = torch.empty((10, 12), dtype=torch.complex128, device="cuda")
    r = ndi.correlate1d(xd, w, output=out)
    assert r.data_ptr() == out.data_ptr()
    _same(out, R.correlate1d(x, w, output=np.empty((10, 12), np.complex128)))
    with pytest.raises(RuntimeError, match="complex"):
        ndi.correlate1d(xd, w, output=torch.empty_like(xd))
    with pytest.raises(RuntimeError, match="complex"):
        ndi.correlate1d(xd, w, output="float32")
    with pytest.warns(UserWarning, match="complex"):
        r = ndi.correlate1d(xd, w, output=np.float64)
    assert r.dtype == torch.complex128


def test_complex_in_place_and_empty(ndi):
    x = _crand((16, 20), np.complex64, 7)
    xd = torch.as_tensor(x).cuda()
    w = np.array([1.0, 2.0, 1.0]) / 4
    exp = R.correlate1d(x, w, axis=0)
    ndi.correlate1d(xd, w, axis=0, output=xd)  # output overlaps the input
    _same(xd, exp)
    e = torch.empty((0, 5), dtype=torch.complex128, device="cuda")
    assert ndi.correlate1d(e, w).shape == (0, 5)


def test_complex_c_abi(cuda):
    """cimx_correlate1d / cimx_separable take complex arrays through the C ABI
    alone, and the entries that do not filter complex data reject it."""
    import ctypes

    from cucim_b200 import _arrays, _lib

    x = _crand((12, 34), np.complex128, 8)
    xd = torch.as_tensor(x).cuda()
    out = torch.empty_like(xd)
    w = np.array([0.3 + 0.2j, 0.4, 0.3 - 0.2j])
    taps = np.ascontiguousarray(w, np.complex128).view(np.float64)
    a_in, a_out = _arrays.to_cimx(xd), _arrays.to_cimx(out)
    flags = _lib.F_W64 | _lib.F_SKIP_ZERO_TAPS | _lib.F_COMPLEX_TAPS
    rc = _lib.lib.cimx_correlate1d(
        ctypes.byref(a_in), ctypes.byref(a_out),
        taps.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 3, 1, 0,
        _lib.MODE_CODES["reflect"], 0.0, flags, None)
    assert rc == 0, _lib.lib.cimx_last_error_string()
    torch.cuda.synchronize()
    # the C taps are used as given: correlate1d of the conjugate weights
    _same(out, R.correlate1d(x, w.conj(), axis=1, algorithm="elementwise"))
    # a real output is refused
    real = torch.empty((12, 34), dtype=torch.float64, device="cuda")
    a_r = _arrays.to_cimx(real)
    rc = _lib.lib.cimx_correlate1d(
        ctypes.byref(a_in), ctypes.byref(a_r),
        taps.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 3, 1, 0,
        _lib.MODE_CODES["reflect"], 0.0, flags, None)
    assert rc == _lib.E_DTYPE
