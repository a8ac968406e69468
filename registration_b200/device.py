"""Device plumbing: CUDA tensors, streams and the cached workspace.

torch provides device memory and streams; all arithmetic happens in the CUDA
library.  Host numpy arrays are copied to the device as float64 and results are
copied back as fresh float64 numpy arrays (what the f2py wrapper returned).
"""
import contextlib
import ctypes
import threading

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
    ordered, so consecutive calls can reuse it.

    scope(owner) routes the calls made inside it to buffers of their own,
    one per call position, held by `owner`: a captured CUDA graph keeps
    pointing at the buffers it was captured with, so they must be neither
    shared with eager calls nor regrown afterwards."""

    def __init__(self):
        self.bufs = {}
        self._tls = threading.local()

    def get(self, nbytes):
        sc = getattr(self._tls, "scope", None)
        if sc is not None:
            owner, pos = sc
            sc[1] = pos + 1
            bufs = owner.__dict__.setdefault("_private_workspaces", [])
            if pos < len(bufs):
                if bufs[pos].numel() < nbytes:
                    raise RuntimeError("a scoped workspace cannot grow once captured")
                return bufs[pos]
            buf = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")
            bufs.append(buf)
            return buf
        key = (torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
        buf = self.bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            cap = max(int(nbytes), 1 << 20)
            if buf is not None:
                cap = max(cap, int(buf.numel() * 1.25))
            buf = torch.empty(cap, dtype=torch.uint8, device="cuda")
            self.bufs[key] = buf
        return buf

    @contextlib.contextmanager
    def scope(self, owner):
        prev = getattr(self._tls, "scope", None)
        self._tls.scope = [owner, 0]
        try:
            yield
        finally:
            self._tls.scope = prev

    def clear(self):
        self.bufs.clear()


workspace = _WorkspaceCache()


def output_like(host_input, t):
    """Returns a numpy array when the caller passed numpy, else the tensor."""
    if isinstance(host_input, torch.Tensor) and host_input.is_cuda:
        return t
    return t.cpu().numpy()
