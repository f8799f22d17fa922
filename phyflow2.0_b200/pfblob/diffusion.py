"""Diffusion by modified redistribution, with pHyFlow's call surface
(``src/python/blobs/base/evolution/_evolution.py``):

* ``diffusion_wee``   (:138-235) - M4' remesh with the Wee coefficient
  c = sqrt(nu dt)/h;
* ``diffusion_tutty`` (:238-445) - Tutty's redistribution weights with
  hNu = sqrt(dt nu).

Both remesh onto the lattice of spacing sigma*overlap anchored at xBounds[0],
yBounds[0] (the ``h`` argument only scales the Wee coefficient, as in the
reference), on the GPU through ``pf_remesh`` / ``pf_remesh_tutty``.
"""
import math

import numpy as np
import torch

from ._arrays import Marshal
from .regrid import M4PRIME_INTERPKERNEL, remesh_device


def _first(b):
    return float(b[0]) if isinstance(b, torch.Tensor) else float(np.asarray(b)[0])


def _run(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, **kw):
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if x.numel() < 1:  # the reference returns its inputs unchanged
        return xBlob, yBlob, wBlob
    xn, yn, gn = remesh_device(x, y, g, sigma * overlap, _first(xBounds), _first(yBounds), **kw)
    return m.outs(xn, yn, gn)


def diffusion_wee(dt, nu, h, xBlob, yBlob, wBlob, sigma, xBounds, yBounds, overlap=0.5, k=2,
                  kernel=1, interpKernel=0, diffusion_method=1):
    """Wee diffusion: remesh with c = sqrt(nu dt)/h (``_evolution.py:227-232``)."""
    if interpKernel != M4PRIME_INTERPKERNEL:
        raise NotImplementedError("pfblob: only the M4' kernel (interpKernel=0) exists")
    c = float(np.sqrt(nu * dt) / h)
    return _run(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, c=c)


def diffusion_tutty(dt, nu, h, xBlob, yBlob, wBlob, sigma, xBounds, yBounds, overlap=0.5, k=2,
                    kernel=1, interpKernel=0, diffusion_method=1):
    """Tutty diffusion: redistribution weights with hNu = sqrt(dt nu)
    (``_evolution.py:366-404``)."""
    hnu = float(np.sqrt(dt * nu))
    return _run(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, tutty_hnu=hnu)
