"""Device-array plumbing: accept torch CUDA tensors, CuPy arrays or any object
exposing ``__cuda_array_interface__`` / DLPack, hand C-contiguous device
buffers to libcimx, and return results of the caller's array type.

PyTorch only provides device memory and the current stream here; every
computation runs in libcimx's kernels.
"""

import numpy as np
import torch

from . import _lib

_NP_TO_TORCH = {
    np.dtype(np.uint8): torch.uint8,
    np.dtype(np.int8): torch.int8,
    np.dtype(np.uint16): torch.uint16,
    np.dtype(np.int16): torch.int16,
    np.dtype(np.uint32): torch.uint32,
    np.dtype(np.int32): torch.int32,
    np.dtype(np.uint64): torch.uint64,
    np.dtype(np.int64): torch.int64,
    np.dtype(np.float16): torch.float16,
    np.dtype(np.float32): torch.float32,
    np.dtype(np.float64): torch.float64,
    np.dtype(np.complex64): torch.complex64,
    np.dtype(np.complex128): torch.complex128,
    np.dtype(np.bool_): torch.bool,
}
_TORCH_TO_NP = {v: k for k, v in _NP_TO_TORCH.items()}


def np_dtype(t):
    """numpy dtype of a torch tensor (or a dtype-like)."""
    if isinstance(t, torch.Tensor):
        return _TORCH_TO_NP[t.dtype]
    if isinstance(t, torch.dtype):
        return _TORCH_TO_NP[t]
    return np.dtype(t)


def torch_dtype(dt):
    return _NP_TO_TORCH[np.dtype(dt)]


def _is_cupy(x):
    return type(x).__module__.split(".")[0] == "cupy"


def as_tensor(x):
    """View `x` as a CUDA torch tensor (zero-copy)."""
    if isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise TypeError("expected a CUDA array (got a CPU torch tensor)")
        return x
    if hasattr(x, "__cuda_array_interface__"):
        return torch.as_tensor(x, device="cuda")
    if hasattr(x, "__dlpack__"):
        t = torch.from_dlpack(x)
        if not t.is_cuda:
            raise TypeError("expected a CUDA array")
        return t
    raise TypeError(f"unsupported array type {type(x)!r}: expected a CUDA array")


def wrap_like(like, t):
    """Return tensor `t` as the array type of `like`."""
    if isinstance(like, torch.Tensor) or t is None:
        return t
    if _is_cupy(like):
        import cupy  # noqa: PLC0415

        return cupy.asarray(t)
    return t


def empty(shape, dtype, device):
    return torch.empty(tuple(shape), dtype=torch_dtype(dtype), device=device)


# CimxArray structs by (pointer, dtype, shape, strides): building a ctypes
# struct costs more than the lookup, and filters are called on the same
# buffers over and over. The structs are only read by the library.
_CIMX_CACHE = {}


def to_cimx(t):
    """CimxArray describing a C-contiguous CUDA tensor."""
    key = (t.data_ptr(), t.dtype, t.shape, t.stride())
    a = _CIMX_CACHE.get(key)
    if a is not None:
        return a
    if t.dim() > _lib.MAX_NDIM:
        raise NotImplementedError(f"ndim > {_lib.MAX_NDIM} is not supported")
    a = _lib.CimxArray()
    a.data = t.data_ptr() if t.numel() > 0 else 0
    a.dtype = ord(np_dtype(t).char)
    a.ndim = t.dim()
    es = t.element_size()
    for d in range(t.dim()):
        a.shape[d] = t.shape[d]
        a.strides[d] = t.stride(d) * es
    if len(_CIMX_CACHE) >= 4096:
        _CIMX_CACHE.clear()
    _CIMX_CACHE[key] = a
    return a


_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_of(t):
    """The current torch stream of `t`'s device, as a raw cudaStream_t."""
    if _RAW_STREAM is not None:
        return _RAW_STREAM(t.get_device())
    return torch.cuda.current_stream(t.device).cuda_stream


def shares_memory(a, b):
    """Whether the memory bounds of two tensors overlap (MAY_SHARE_BOUNDS)."""
    if a.numel() == 0 or b.numel() == 0:
        return False
    if a.device != b.device:
        return False
    if a.is_contiguous() and b.is_contiguous():
        a0, b0 = a.data_ptr(), b.data_ptr()
        return a0 < b0 + b.numel() * b.element_size() and b0 < a0 + a.numel() * a.element_size()

    def bounds(t):
        lo = hi = t.data_ptr()
        es = t.element_size()
        for n, s in zip(t.shape, t.stride()):
            if s >= 0:
                hi += (n - 1) * s * es
            else:
                lo += (n - 1) * s * es
        return lo, hi + es

    a0, a1 = bounds(a)
    b0, b1 = bounds(b)
    return a0 < b1 and b0 < a1


class OutputSlot:
    """The caller's output (if any) and the contiguous buffer the kernels
    write; `result()` copies back when the two differ and returns the
    caller's object (or a new array of the input's array type)."""

    def __init__(self, final, work, user=None, like=None):
        self.final = final
        self.work = work
        self.user = user
        self.like = like

    @property
    def dtype(self):
        return np_dtype(self.work)

    def result(self):
        if self.work is not self.final:
            self.final.copy_(self.work)
        if self.user is not None:
            return self.user
        return wrap_like(self.like, self.final)


def is_dtype_like(output):
    return isinstance(output, (type, np.dtype, str, torch.dtype))


def output_slot(output, input_obj, input_t, shape=None, dtype=None):
    """_get_output (_vendored/_ndimage_util.py:49-71) on torch tensors.

    `dtype` is the default output dtype (the input's when None).
    """
    shape = input_t.shape if shape is None else tuple(shape)
    if output is None:
        tdt = input_t.dtype if dtype is None else torch_dtype(dtype)
        t = torch.empty(shape, dtype=tdt, device=input_t.device)
        return OutputSlot(t, t, like=input_obj)
    if isinstance(output, torch.dtype):
        t = torch.empty(shape, dtype=output, device=input_t.device)
        return OutputSlot(t, t, like=input_obj)
    if is_dtype_like(output):
        t = empty(shape, np.dtype(output), input_t.device)
        return OutputSlot(t, t, like=input_obj)
    out_t = as_tensor(output)
    if out_t.shape != shape:
        raise RuntimeError("output shape not correct")
    if out_t.is_contiguous() and not shares_memory(out_t, input_t):
        return OutputSlot(out_t, out_t, user=output)
    work = torch.empty(shape, dtype=out_t.dtype, device=out_t.device)
    return OutputSlot(out_t, work, user=output)
