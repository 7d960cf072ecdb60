"""The schedule autotuner of libcimx (cimx_tune_* in include/cimx.h).

Every filter call that goes through a pass list (gaussian, uniform, sobel,
prewitt, the Hessian's Gaussian derivatives, ...) can run on several kernel
schedules with bit-identical results; the tuner picks the fastest per call
signature (dtypes, shape, taps, modes) and device model, and with
algorithm="tensor" also between the tensor-core and the plain float32
passes. cuCIM picks its kernel by a fixed rule instead
(_vendored/_ndimage_filters.py:284-297).

    from cucim_b200 import tune
    with tune.tuning():            # time unseen signatures on first use
        ndimage.gaussian_filter(x, 2.0)
    tune.save("tune.json")         # or set CIMX_TUNE_CACHE=tune.json
    tune.entries()                 # the recorded choices

Modes: OFF (built-in rules), USE (recorded choices where present; the
default), ON (also time unseen signatures: that synchronises the stream).
"""

import contextlib
import ctypes
import json

from . import _lib

OFF, USE, ON = 0, 1, 2


def mode(new=None):
    """The current mode; with `new`, set it and return the previous one."""
    rc = _lib.lib.cimx_tune_mode(-1 if new is None else int(new))
    if rc < 0:
        _lib.check(rc, "tune mode")
    return rc


@contextlib.contextmanager
def tuning(new_mode=ON):
    prev = mode(new_mode)
    try:
        yield
    finally:
        mode(prev)


def load(path):
    _lib.check(_lib.lib.cimx_tune_load(str(path).encode()), "tune load")


def save(path):
    _lib.check(_lib.lib.cimx_tune_save(str(path).encode()), "tune save")


def clear():
    _lib.check(_lib.lib.cimx_tune_clear(), "tune clear")


def dump():
    """The whole table as parsed JSON ({"format": ..., "entries": [...]})."""
    n = _lib.lib.cimx_tune_dump(None, 0)
    buf = ctypes.create_string_buffer(int(n))
    _lib.lib.cimx_tune_dump(buf, n)
    return json.loads(buf.value.decode())


def entries():
    return dump()["entries"]
