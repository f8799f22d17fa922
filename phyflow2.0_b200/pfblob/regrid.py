"""M4' remesh with pHyFlow's ``Regrid`` call surface
(``src/python/blobs/base/regrid/_regridding.py:36-222``)."""
import ctypes

import numpy as np
import torch

from . import _lib
from ._arrays import Marshal, ptr

M4PRIME_INTERPKERNEL = 0


def remesh_device(x, y, g, h, xb0, yb0, c=0.0, capacity=None, with_indices=False, stream=None):
    """Device-tensor entry.  Returns (x, y, g[, ix, iy]) CUDA tensors of the
    new blobs in (ix, iy) order.  ``capacity`` bounds the output (default
    16 n, the window count); a retry with the exact size follows a capacity
    error."""
    n = x.numel()
    dev = x.device
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    ctx = _lib.context(dev.index)
    if capacity is None:
        capacity = 16 * n
    while True:
        xo = torch.empty(capacity, dtype=torch.float64, device=dev)
        yo = torch.empty(capacity, dtype=torch.float64, device=dev)
        go = torch.empty(capacity, dtype=torch.float64, device=dev)
        ixo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
        iyo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
        nout = ctypes.c_int64(0)
        s = _lib.lib.pf_remesh(ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0), float(yb0),
                               float(c), capacity, ptr(xo), ptr(yo), ptr(go), ptr(ixo), ptr(iyo),
                               ctypes.byref(nout), st)
        if s == 6 and nout.value > capacity:  # PF_ERR_CAPACITY
            capacity = nout.value
            continue
        _lib.check(s)
        k = nout.value
        out = (xo[:k], yo[:k], go[:k])
        if with_indices:
            out = out + (ixo[:k], iyo[:k])
        return out


def Regrid(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, interpKernel=0, c=0.0):
    """Redistribute blobs onto the lattice of spacing h = sigma*overlap.

    Same arguments and results as pHyFlow's ``Regrid``: new (x, y, g) of every
    lattice node touched by a blob's 4x4 M4' window, explicit zeros kept,
    ordered by (ix, iy); ``c`` is the Wee diffusion coefficient.
    """
    if interpKernel != M4PRIME_INTERPKERNEL:
        raise NotImplementedError("pfblob: only the M4' kernel (interpKernel=0) exists")
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if x.numel() < 1:  # the reference returns its inputs unchanged (:143-146)
        return xBlob, yBlob, wBlob
    h = sigma * overlap
    xb0 = float(np.asarray(xBounds)[0]) if not isinstance(xBounds, torch.Tensor) else float(xBounds[0])
    yb0 = float(np.asarray(yBounds)[0]) if not isinstance(yBounds, torch.Tensor) else float(yBounds[0])
    xn, yn, gn = remesh_device(x, y, g, h, xb0, yb0, c)
    return m.out(xn), m.out(yn), m.out(gn)
