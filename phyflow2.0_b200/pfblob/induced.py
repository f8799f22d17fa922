"""Blob induced velocity with pHyFlow's call surface.

``velocity`` keeps the signature, argument meaning and option constants of
``pHyFlow.blobs.base.induced.velocity`` (``src/python/blobs/base/induced/
_induced.py:34-166``): ``fullOption = 100*method + 10*hardware + kernel``
selects direct or FMM summation of the Gaussian kernel (``kernel=1``) or the
direct sum of the cutoff kernel (``kernel=0``); the FMM of the cutoff kernel
raises the reference's own exception (:159-163).

Differences, by design of this library:
* every combination runs on the B200 (``hardware`` is accepted for
  compatibility, and selects only which of the reference's messages an
  unavailable combination raises; there is no CPU path);
* ``blocksize`` is accepted and ignored: no padding is needed.
"""
import ctypes
import math

import torch

from . import _lib
from ._arrays import Marshal, ptr, require

GAUSS_KERNEL = 1
CUTOFF_KERNEL = 0
CPU_HARDWARE = 0
GPU_HARDWARE = 1
FMM_METHOD = 0
DIRECT_METHOD = 1

# Oseen smoother constant of the reference FMM binding (_induced.py:239, :321)
FMM_ALPHA = 1.2564312086261696770


def default_cutoff(ksigmasqr, tol=1e-6):
    """FMM near-field radius when the caller gives none.  The reference uses
    5 xopt (``_induced.py:239-241``), where the Gaussian core's correction to
    the point-vortex kernel, exp(-r^2/ksigmasqr), is 2e-14.  With a tolerance
    the radius is lowered to where that correction is tol/100
    (r^2 = ksigmasqr ln(100/tol)), never raised: beyond it the far field's
    point-vortex expansions are exact to well below tol."""
    cut = 5.0 * math.sqrt(FMM_ALPHA * ksigmasqr)
    if tol and tol > 0.0:
        cut = min(cut, math.sqrt(ksigmasqr * math.log(100.0 / tol)))
    return cut


def fmm_parameters(sigma, k=2.0, cutoff=None, tol=1e-6):
    """(ksigmasqr, xopt, cutoff) as ``_velocity_fmm_*_gauss`` derives them,
    the cutoff from ``default_cutoff`` unless given."""
    ksigmasqr = k * sigma * sigma
    xopt = math.sqrt(FMM_ALPHA * ksigmasqr)
    if cutoff is None:
        cutoff = default_cutoff(ksigmasqr, tol)
    return ksigmasqr, xopt, cutoff


def velocity_device(x, y, g, ksigmasqr, xt, yt, vx, vy, method=DIRECT_METHOD, xopt=None,
                    cutoff=None, tol=1e-6, ndirect=35, stream=None, device=None, box=None):
    """Device-tensor entry: all arguments CUDA float64 tensors; writes vx, vy.
    ``box = (xmin, xmax, ymin, ymax)`` containing all sources and targets lets
    the FMM skip its bounding-box read-back (pf_velocity_fmm_box)."""
    require(x.numel(), x.device, x=x, y=y, g=g)
    require(xt.numel(), x.device, xt=xt, yt=yt, vx=vx, vy=vy)
    if device is not None and device != x.device.index:
        raise ValueError(f"pfblob: device {device} given for tensors on {x.device}")
    dev = x.device.index
    st = ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream if stream is None
                         else stream)
    ctx = _lib.context(dev)
    if method == DIRECT_METHOD or tol == 0.0:
        _lib.check(_lib.lib.pf_velocity_direct(ctx, x.numel(), ptr(x), ptr(y), ptr(g), xt.numel(),
                                               ptr(xt), ptr(yt), float(ksigmasqr), ptr(vx),
                                               ptr(vy), st))
    else:
        if xopt is None:
            xopt = math.sqrt(FMM_ALPHA * ksigmasqr)
        if cutoff is None:
            cutoff = default_cutoff(ksigmasqr, tol)
        if box is None:
            _lib.check(_lib.lib.pf_velocity_fmm(ctx, x.numel(), ptr(x), ptr(y), ptr(g),
                                                xt.numel(), ptr(xt), ptr(yt), float(ksigmasqr),
                                                float(xopt), float(cutoff), float(tol),
                                                int(ndirect), ptr(vx), ptr(vy), st))
        else:
            b = (ctypes.c_double * 4)(*[float(v) for v in box])
            _lib.check(_lib.lib.pf_velocity_fmm_box(ctx, x.numel(), ptr(x), ptr(y), ptr(g),
                                                    xt.numel(), ptr(xt), ptr(yt),
                                                    float(ksigmasqr), float(xopt), float(cutoff),
                                                    float(tol), int(ndirect), b, ptr(vx),
                                                    ptr(vy), st))


def velocity(xBlob, yBlob, wBlob, sigma, k=2, kernel=1, xEval=None, yEval=None, hardware=0,
             blocksize=128, method=0, Ndirect=35, tol=1.0e-6, cutoff=None):
    """Induced velocity of vortex blobs at (xEval, yEval): Gaussian kernel
    (direct or FMM) or cutoff kernel (direct).

    Same arguments and return value as pHyFlow's ``velocity``; returns
    ``(vx, vy)`` as numpy arrays for numpy input, CUDA tensors for CUDA input.
    """
    if kernel not in (GAUSS_KERNEL, CUTOFF_KERNEL):
        raise ValueError(f"pfblob: unknown kernel {kernel}")
    if method not in (FMM_METHOD, DIRECT_METHOD):
        raise ValueError(f"pfblob: unknown method {method}")
    if kernel == CUTOFF_KERNEL and method == FMM_METHOD:
        # the reference's messages for these combinations (_induced.py:159-163)
        where = "GPU" if hardware == GPU_HARDWARE else "CPU"
        raise Exception(f'FMM calculation of cutoff kernel on the {where} not yet available')
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if not (x.numel() == y.numel() == g.numel()):
        raise ValueError("pfblob: xBlob, yBlob, wBlob must have the same length")
    if xEval is None:
        xt, yt = x, y
    else:
        xt, yt = m.dev(xEval), m.dev(yEval)
        if xt.numel() != yt.numel():
            raise ValueError("pfblob: xEval and yEval must have the same length")
    vx, vy = m.empty(xt.numel()), m.empty(xt.numel())
    if kernel == CUTOFF_KERNEL:
        velocity_cutoff_device(x, y, g, float(sigma) * float(sigma), xt, yt, vx, vy,
                               device=m.index)
        return m.outs(vx, vy)
    ksigmasqr, xopt, cut = fmm_parameters(float(sigma), float(k), cutoff, float(tol))
    velocity_device(x, y, g, ksigmasqr, xt, yt, vx, vy, method=method, xopt=xopt, cutoff=cut,
                    tol=float(tol), ndirect=int(Ndirect), device=m.index)
    return m.outs(vx, vy)


def velocity_cutoff_device(x, y, g, sigmasqr, xt, yt, vx, vy, stream=None, device=None):
    """Device-tensor entry of the cutoff kernel's direct sum
    (pf_velocity_direct_cutoff): v = 1/(2 pi) sum g (-dy, dx)/(r^2 + sigmasqr)."""
    require(x.numel(), x.device, x=x, y=y, g=g)
    require(xt.numel(), x.device, xt=xt, yt=yt, vx=vx, vy=vy)
    if device is not None and device != x.device.index:
        raise ValueError(f"pfblob: device {device} given for tensors on {x.device}")
    st = ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream if stream is None
                         else stream)
    _lib.check(_lib.lib.pf_velocity_direct_cutoff(_lib.context(x.device.index), x.numel(), ptr(x),
                                                  ptr(y), ptr(g), xt.numel(), ptr(xt), ptr(yt),
                                                  float(sigmasqr), ptr(vx), ptr(vy), st))


def vorticity(xBlob, yBlob, wBlob, sigma, k=2, kernel=1, xEval=None, yEval=None, hardware=0,
              blocksize=128, method=1):
    """Induced vorticity of vortex blobs at (xEval, yEval) (the blobs if
    None), by direct summation on the GPU: Gaussian kernel (``kernel=1``) or,
    as the reference computes it, the cutoff kernel (``kernel=0``).

    Same arguments and return value as pHyFlow's ``vorticity``
    (``src/python/blobs/base/induced/_induced.py:702-789``); like the
    reference, the FMM method is not available for the vorticity."""
    if kernel not in (GAUSS_KERNEL, CUTOFF_KERNEL):
        raise ValueError(f"pfblob: unknown kernel {kernel}")
    if method != DIRECT_METHOD:
        raise Exception('FMM method not implemented yet')
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if xEval is None:
        xt, yt = x, y
    else:
        xt, yt = m.dev(xEval), m.dev(yEval)
    require(x.numel(), m.device, xBlob=x, yBlob=y, wBlob=g)
    require(xt.numel(), m.device, xEval=xt, yEval=yt)
    w = m.empty(xt.numel())
    ctx = _lib.context(m.index)
    if kernel == CUTOFF_KERNEL:
        _lib.check(_lib.lib.pf_vorticity_direct_cutoff(ctx, x.numel(), ptr(x), ptr(y), ptr(g),
                                                       xt.numel(), ptr(xt), ptr(yt),
                                                       float(sigma) * float(sigma), ptr(w),
                                                       m.stream))
    else:
        _lib.check(_lib.lib.pf_vorticity_direct(ctx, x.numel(), ptr(x), ptr(y), ptr(g),
                                                xt.numel(), ptr(xt), ptr(yt),
                                                float(k) * sigma * sigma, ptr(w), m.stream))
    return m.outs(w)[0]
