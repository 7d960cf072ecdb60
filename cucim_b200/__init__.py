"""cucim_b200 — cuCIM's separable n-D filtering path rebuilt for NVIDIA B200.

`cucim_b200.ndimage` mirrors cucim.skimage._vendored.ndimage and
`cucim_b200.skimage` mirrors the cucim.skimage functions on the path; both
call the sm_100a kernels of libcimx.so through its C ABI (include/cimx.h).
"""

from . import _lib  # noqa: F401  (raises if libcimx.so is missing)
from . import ndimage, skimage, tune  # noqa: F401

__version__ = "0.1.0"
