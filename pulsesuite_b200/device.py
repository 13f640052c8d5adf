"""Device-memory plumbing: torch tensors as the caller-owned buffers of the C ABI."""

import ctypes

import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.PsbError("pulsesuite_b200 needs a CUDA device (no CPU fallback)")
    _lib.load()


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


def to_device(a, device="cuda"):
    """Copy a numpy array (any dtype, structured included) to a device tensor
    holding the same bytes."""
    a = np.ascontiguousarray(a)
    if a.dtype.fields is not None or a.dtype.kind not in "fiuc":
        raw = torch.from_numpy(a.view(np.uint8).reshape(-1).copy())
        return raw.to(device)
    return torch.from_numpy(a.copy()).to(device)


def to_host_struct(t, dtype):
    """Device bytes -> numpy structured array of `dtype`."""
    raw = t.detach().to("cpu").numpy()
    return raw.view(dtype).copy()
