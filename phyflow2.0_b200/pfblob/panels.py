"""Vortex and source panels with pHyFlow's ``panelSolver`` surface
(``src/python/panels/base/panelSolver.py``): ``inducedVelocity`` (:148-262)
and ``influenceMatrix`` (:31-144) for constant-strength vortex
(``panelKernel=1``) and constant-strength source (``panelKernel=0``) panels,
plus the LU factor / solve pair the ``Panels`` class uses for the panel
strengths (``__panelsClass.py:782, :960-962``), all on the GPU."""
import ctypes
import warnings

import numpy as np
import torch

from . import _lib
from ._arrays import Marshal, ptr, require

CPU_HARDWARE = 0
GPU_HARDWARE = 1
FMM_METHOD = 0
DIRECT_METHOD = 1
PANEL_KERNEL_CSV = 1  # constant-strength vortex
PANEL_KERNEL_CSS = 0  # constant-strength source


def panel_velocity_device(gamma, xs, ys, xe, ye, cosa, sina, xv, yv, vx, vy, accumulate=False,
                          stream=None, panelKernel=PANEL_KERNEL_CSV):
    """Device-tensor panel velocity (vortex panels, or source panels with
    ``panelKernel=0``), written to or added onto (vx, vy)."""
    dev = xv.device
    require(gamma.numel(), dev, gamma=gamma, xs=xs, ys=ys, xe=xe, ye=ye, cosa=cosa, sina=sina)
    require(xv.numel(), dev, xv=xv, yv=yv, vx=vx, vy=vy)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    fn = _lib.lib.pf_source_panel_velocity if panelKernel == PANEL_KERNEL_CSS \
        else _lib.lib.pf_panel_velocity
    _lib.check(fn(_lib.context(dev.index), gamma.numel(), ptr(gamma), ptr(xs), ptr(ys), ptr(xe),
                  ptr(ye), ptr(cosa), ptr(sina), xv.numel(), ptr(xv), ptr(yv), ptr(vx), ptr(vy),
                  int(bool(accumulate)), st))


def inducedVelocity(strength, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd, cosAlpha, sinAlpha,
                    xEval, yEval, hardware=0, method=1, panelKernel=1):
    """Velocity induced by constant-strength vortex (``panelKernel=1``) or
    source (``panelKernel=0``) panels at (xEval, yEval).

    Same arguments and results as pHyFlow's ``inducedVelocity``; always runs
    on the B200 (the reference's GPU branch is unimplemented, :257-258).
    """
    if panelKernel not in (PANEL_KERNEL_CSV, PANEL_KERNEL_CSS):
        raise ValueError(f"pfblob: unknown panel kernel {panelKernel}")
    if method != DIRECT_METHOD:
        raise NotImplementedError("pfblob: panel velocity is direct summation (method=1)")
    m = Marshal(xEval.device.index if isinstance(xEval, torch.Tensor) and xEval.is_cuda else None)
    arrs = [m.dev(a) for a in (strength, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd, cosAlpha,
                               sinAlpha)]
    xv, yv = m.dev(xEval), m.dev(yEval)
    vx, vy = m.empty(xv.numel()), m.empty(xv.numel())
    panel_velocity_device(*arrs, xv, yv, vx, vy, panelKernel=panelKernel)
    return m.outs(vx, vy)


def influenceMatrix(xCP, yCP, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd, cosAlpha, sinAlpha,
                    hardware=0, method=1, panelKernel=1):
    """Self-induction influence matrix A (M x M) of constant-strength vortex
    (tangential velocity) or source (``panelKernel=0``, normal velocity)
    panels on their collocation points; same arguments and result as
    pHyFlow's ``influenceMatrix``."""
    if panelKernel not in (PANEL_KERNEL_CSV, PANEL_KERNEL_CSS):
        raise ValueError(f"pfblob: unknown panel kernel {panelKernel}")
    if method != DIRECT_METHOD:
        raise NotImplementedError("pfblob: the influence matrix is assembled directly (method=1)")
    m = Marshal(xCP.device.index if isinstance(xCP, torch.Tensor) and xCP.is_cuda else None)
    arrs = [m.dev(a) for a in (xCP, yCP, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd,
                               cosAlpha, sinAlpha)]
    n = arrs[0].numel()
    require(n, m.device, **dict(zip(("xCP", "yCP", "xPanelStart", "yPanelStart", "xPanelEnd",
                                     "yPanelEnd", "cosAlpha", "sinAlpha"), arrs)))
    A = torch.empty((n, n), dtype=torch.float64, device=m.device)
    fn = _lib.lib.pf_source_panel_influence_matrix if panelKernel == PANEL_KERNEL_CSS \
        else _lib.lib.pf_panel_influence_matrix
    _lib.check(fn(_lib.context(m.index), n, *[ptr(a) for a in arrs], ptr(A), m.stream))
    return m.outs(A)[0]


def lu_factor(a, overwrite_a=False):
    """LU factorisation with partial pivoting on the GPU, for ``lu_solve``
    (the factors are this library's row-major form, not LAPACK's layout).
    Returns (lu, piv) in the input's kind (numpy or CUDA tensors); warns, as
    scipy does, when a diagonal of U is exactly zero."""
    if len(a.shape) != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("expected a square matrix")
    n = int(a.shape[0])
    m = Marshal(a.device.index if isinstance(a, torch.Tensor) and a.is_cuda else None)
    A = m.dev(a).reshape(n, n)
    if isinstance(a, torch.Tensor) and a.is_cuda and not overwrite_a and A.data_ptr() == a.data_ptr():
        A = A.clone()
    piv = torch.empty(n, dtype=torch.int32, device=m.device)
    info = torch.zeros(1, dtype=torch.int32, device=m.device)
    _lib.check(_lib.lib.pf_dense_lu_factor(_lib.context(m.index), n, ptr(A), ptr(piv), ptr(info),
                                           m.stream))
    k = int(info.item())
    if k > 0:
        warnings.warn("Diagonal number %d is exactly zero. Singular matrix." % k, RuntimeWarning)
    lu, p = m.outs(A, piv)
    return lu, p


def lu_solve(lu_and_piv, b):
    """Solution x of A x = b from ``lu_factor``'s factors."""
    lu, piv = lu_and_piv
    m = Marshal(b.device.index if isinstance(b, torch.Tensor) and b.is_cuda else None)
    LU = m.dev(lu)
    P = piv.to(m.device, torch.int32) if isinstance(piv, torch.Tensor) else \
        torch.from_numpy(np.ascontiguousarray(piv, dtype=np.int32)).to(m.device)
    x = m.dev(b).clone()
    n = x.numel()
    require(n * n, m.device, lu=LU)
    require(n, m.device, dtype=torch.int32, piv=P)
    _lib.check(_lib.lib.pf_dense_lu_solve(_lib.context(m.index), n, ptr(LU), ptr(P), ptr(x),
                                          m.stream))
    return m.outs(x)[0]
