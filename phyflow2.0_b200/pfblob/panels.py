"""Vortex-panel induced velocity with pHyFlow's ``inducedVelocity`` surface
(``src/python/panels/base/panelSolver.py:148-262``)."""
import ctypes

import torch

from . import _lib
from ._arrays import Marshal, ptr

CPU_HARDWARE = 0
GPU_HARDWARE = 1
FMM_METHOD = 0
DIRECT_METHOD = 1
PANEL_KERNEL_CSV = 1  # constant-strength vortex


def panel_velocity_device(gamma, xs, ys, xe, ye, cosa, sina, xv, yv, vx, vy, accumulate=False,
                          stream=None):
    dev = xv.device
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    _lib.check(_lib.lib.pf_panel_velocity(_lib.context(dev.index), gamma.numel(), ptr(gamma),
                                          ptr(xs), ptr(ys), ptr(xe), ptr(ye), ptr(cosa), ptr(sina),
                                          xv.numel(), ptr(xv), ptr(yv), ptr(vx), ptr(vy),
                                          int(bool(accumulate)), st))


def inducedVelocity(strength, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd, cosAlpha, sinAlpha,
                    xEval, yEval, hardware=0, method=1, panelKernel=1):
    """Velocity induced by constant-strength vortex panels at (xEval, yEval).

    Same arguments and results as pHyFlow's ``inducedVelocity``; always runs
    on the B200 (the reference's GPU branch is unimplemented, :257-258).
    """
    if panelKernel != PANEL_KERNEL_CSV:
        raise NotImplementedError("pfblob: only constant-strength vortex panels (panelKernel=1)")
    if method != DIRECT_METHOD:
        raise NotImplementedError("pfblob: panel velocity is direct summation (method=1)")
    m = Marshal(xEval.device.index if isinstance(xEval, torch.Tensor) and xEval.is_cuda else None)
    arrs = [m.dev(a) for a in (strength, xPanelStart, yPanelStart, xPanelEnd, yPanelEnd, cosAlpha,
                               sinAlpha)]
    xv, yv = m.dev(xEval), m.dev(yEval)
    vx, vy = m.empty(xv.numel()), m.empty(xv.numel())
    panel_velocity_device(*arrs, xv, yv, vx, vy)
    return m.outs(vx, vy)
