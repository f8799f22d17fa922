"""A resident blob set's step -- induced velocity at the blobs, then the M4'
remesh of the same blobs -- captured once as a CUDA graph and replayed with one
graph launch per step (pf_step_graph_* of include/pfblob.h).

The step is pf_blob_step: FMM on a tree box the caller knows (or the direct
sum), then the remesh with the lattice window found on the device; nothing
waits for the host.  The blob arrays may change in value between launches (a
stepping loop writes the next positions into them), not in address or size.
There is no reference counterpart: pHyFlow issues every kernel of a step
separately (src/python/blobs/__blobsClass.py:546-626, 828-897).
"""
import ctypes

import torch

from . import _lib
from .induced import FMM_METHOD
from ._arrays import ptr, require


class StepGraph:
    """Velocity + remesh step of the blobs (x, y, g) (CUDA float64 tensors),
    captured at construction.  ``box = (xmin, xmax, ymin, ymax)`` holds every
    blob (the FMM tree box); ``max_base_cells`` bounds the remesh window (the
    status word gets 8 when a step's window exceeds it).  After ``launch()``
    the velocity is in ``vx``, ``vy``; ``result()`` waits and returns the new
    blobs (x, y, g) and the status word."""

    def __init__(self, x, y, g, ksigmasqr, xopt, cutoff, tol, box, h, xb0, yb0, c=0.0,
                 method=FMM_METHOD, leaf_level=0, max_base_cells=None, capacity=None):
        n = x.numel()
        dev = x.device
        require(n, dev, x=x, y=y, g=g)
        self.device = dev
        self.n = n
        mb = int(max_base_cells) if max_base_cells is not None else max(4 * n, 4096)
        if capacity is None:
            capacity = mb + mb // 2 + 65536
        f64 = dict(dtype=torch.float64, device=dev)
        self.x, self.y, self.g = x, y, g
        self.vx = torch.empty(n, **f64)
        self.vy = torch.empty(n, **f64)
        self.out = torch.empty((3, capacity), **f64)
        self.n_out = torch.zeros(1, dtype=torch.int64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.moments = torch.zeros(8, **f64)
        d = _lib.Step()
        d.n, d.x, d.y, d.g = n, ptr(x), ptr(y), ptr(g)
        d.ksigmasqr, d.xopt, d.cutoff, d.tol = float(ksigmasqr), float(xopt), float(cutoff), \
            float(tol)
        d.method, d.leaf_level = int(method), int(leaf_level)
        for i, v in enumerate(box):
            d.box[i] = float(v)
        d.vx, d.vy = ptr(self.vx), ptr(self.vy)
        d.h, d.xb0, d.yb0, d.c = float(h), float(xb0), float(yb0), float(c)
        d.max_base_cells, d.capacity = mb, int(capacity)
        d.x_out, d.y_out, d.g_out = ptr(self.out[0]), ptr(self.out[1]), ptr(self.out[2])
        d.n_out_dev, d.status_dev = ptr(self.n_out), ptr(self.status)
        d.moments_dev = ptr(self.moments)
        self._desc = d
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib.pf_step_graph_create(_lib.context(dev.index), ctypes.byref(d),
                                                 ctypes.byref(self._h)))

    @property
    def kernels(self):
        """Kernel nodes of the captured step."""
        k = ctypes.c_int64()
        _lib.check(_lib.lib.pf_step_graph_kernels(self._h, ctypes.byref(k)))
        return k.value

    def launch(self, stream=None):
        """Enqueue the whole step on ``stream`` (default: the current stream)."""
        if not self._h:
            raise ValueError("pfblob: StepGraph used after close()")
        st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream
                             if stream is None else stream)
        _lib.check(_lib.lib.pf_step_graph_launch(self._h, st))

    def result(self):
        """Wait for the last launch; (x, y, g) of the new blobs and the status
        word (0 = done)."""
        k = int(self.n_out.item())
        return self.out[0, :k], self.out[1, :k], self.out[2, :k], int(self.status.item())

    def close(self):
        if self._h:
            _lib.check(_lib.lib.pf_step_graph_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
