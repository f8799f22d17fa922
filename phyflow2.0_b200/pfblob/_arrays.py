"""Argument handling shared by the pHyFlow-compatible entry points.

Inputs may be numpy arrays (copied to the device through pinned memory, the
result copied back and returned as numpy, like the reference extension
functions) or CUDA torch tensors (used in place, results returned as CUDA
tensors, no host round trip).  torch is used only for device buffers and
streams.
"""
import ctypes

import numpy as np
import torch


class Marshal:
    """Collects device views of the arguments of one call."""

    def __init__(self, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.host = False

    def dev(self, a, name="array"):
        if isinstance(a, torch.Tensor):
            if not a.is_cuda:
                self.host = True
                return a.to(torch.float64).contiguous().pin_memory().to(self.device, non_blocking=True)
            if a.device != self.device:
                self.device = a.device
            t = a
            if t.dtype != torch.float64:
                t = t.to(torch.float64)
            return t.contiguous()
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        self.host = True
        return torch.from_numpy(arr).pin_memory().to(self.device, non_blocking=True)

    def empty(self, n):
        return torch.empty(int(n), dtype=torch.float64, device=self.device)

    def out(self, t):
        return self.outs(t)[0]

    def outs(self, *ts):
        """Results in the caller's form.  Host results are copied straight into
        pinned buffers (no staging, no first-touch page faults of fresh
        pageable memory) with one synchronisation for all of them; the numpy
        arrays returned keep those buffers alive."""
        if not self.host:
            return ts
        hs = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in ts]
        for h, t in zip(hs, ts):
            h.copy_(t, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return tuple(h.numpy() for h in hs)

    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def index(self):
        return self.device.index


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)
