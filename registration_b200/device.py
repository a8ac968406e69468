"""Device plumbing: CUDA tensors, streams and the cached workspace.

torch provides device memory and streams; all arithmetic happens in the CUDA
library.  Host numpy arrays are copied to the device as float64 and results are
copied back as fresh float64 numpy arrays (what the f2py wrapper returned).
"""
import ctypes

import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.LddmmError("registration_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    _lib.load()


def is_device(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def to_dev(a, device=None):
    """float64, contiguous CUDA tensor view/copy of a numpy array or tensor."""
    if isinstance(a, torch.Tensor):
        t = a
        if not t.is_cuda:
            t = t.to("cuda" if device is None else device)
        if t.dtype != torch.float64:
            t = t.to(torch.float64)
        return t.contiguous()
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return torch.from_numpy(arr).to("cuda" if device is None else device)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def stream_handle():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class _WorkspaceCache:
    """One growing uint8 buffer per (device, stream); calls on one stream are
    ordered, so consecutive calls can reuse it."""

    def __init__(self):
        self.bufs = {}

    def get(self, nbytes):
        key = (torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
        buf = self.bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            cap = max(int(nbytes), 1 << 20)
            if buf is not None:
                cap = max(cap, int(buf.numel() * 1.25))
            buf = torch.empty(cap, dtype=torch.uint8, device="cuda")
            self.bufs[key] = buf
        return buf

    def clear(self):
        self.bufs.clear()


workspace = _WorkspaceCache()


def output_like(host_input, t):
    """Returns a numpy array when the caller passed numpy, else the tensor."""
    if isinstance(host_input, torch.Tensor) and host_input.is_cuda:
        return t
    return t.cpu().numpy()
