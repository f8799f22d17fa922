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
        self.placed = False  # an argument already lives on (or was copied to) self.device

    def dev(self, a, name="array"):
        if isinstance(a, torch.Tensor):
            if not a.is_cuda:
                self.host = True
                self.placed = True
                return a.to(torch.float64).contiguous().pin_memory().to(self.device, non_blocking=True)
            if a.device != self.device:
                # one call runs on one device: a kernel given another device's
                # pointer would fault, so mixed devices are refused here
                if self.placed:
                    raise ValueError(f"pfblob: {name} is on {a.device}, the other arguments on "
                                     f"{self.device}")
                self.device = a.device
            self.placed = True
            t = a
            if t.dtype != torch.float64:
                t = t.to(torch.float64)
            return t.contiguous()
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        self.host = True
        self.placed = True
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


def require(n, device, dtype=torch.float64, **tensors):
    """Checks the arguments of a device-tensor entry point: each a contiguous
    CUDA tensor of `dtype` with `n` elements on `device`.  The kernels index
    them by n on one device, so anything else would read or write memory the
    tensor does not own; it is refused here instead."""
    for name, t in tensors.items():
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise TypeError(f"pfblob: {name} must be a CUDA tensor")
        if t.device != device:
            raise ValueError(f"pfblob: {name} is on {t.device}, the other arguments on {device}")
        if t.dtype != dtype:
            raise TypeError(f"pfblob: {name} must be {dtype}, not {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"pfblob: {name} must be contiguous")
        if t.numel() != n:
            raise ValueError(f"pfblob: {name} has {t.numel()} elements, expected {n}")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)
