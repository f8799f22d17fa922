"""Convection of vortex blobs with pHyFlow's call surface
(``src/python/blobs/base/evolution/_evolution.py``): ``convection`` (:37-135)
with forward Euler (``_convection_fe`` :448-554) or the reference's RK4
(``_convection_rk4`` :557-701).

The reference's RK4 evaluates every stage at the start positions: the stage
increment it adds (``kx_rk4``) is never updated from zero (:679-693), so the
four stage velocities are the same.  Here the velocity is evaluated once and
the four weighted position updates are applied in the reference's order,
which gives the reference's result with a quarter of the work.  Circulations
are unchanged by convection.
"""
import torch

from ._arrays import Marshal, require
from .induced import (CUTOFF_KERNEL, DIRECT_METHOD, FMM_METHOD, GAUSS_KERNEL, GPU_HARDWARE,
                      fmm_parameters, velocity_cutoff_device, velocity_device)

FE_INTEGRATOR = 0
RK4_INTEGRATOR = 1
RK4_WEIGHTS = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)


def convection_device(dt, x, y, g, sigma, k=2.0, vInf=(0.0, 0.0), method=DIRECT_METHOD,
                      integrator=RK4_INTEGRATOR, kernel=GAUSS_KERNEL, hardware=0):
    """Device-tensor convection step: returns new (x, y) tensors; g is
    unchanged.  The blob velocity comes from ``velocity_device`` at the blobs
    (tol 1e-6, Ndirect 35, default cutoff, as ``velocity``'s defaults), or
    for ``kernel=0`` from the cutoff kernel's direct sum (whose FMM raises, as
    the reference's ``velocity`` does)."""
    if integrator not in (FE_INTEGRATOR, RK4_INTEGRATOR):
        raise ValueError("pfblob: integrator must be 0 (forward Euler) or 1 (RK4)")
    if method not in (FMM_METHOD, DIRECT_METHOD):
        raise ValueError(f"pfblob: unknown method {method}")
    if kernel not in (GAUSS_KERNEL, CUTOFF_KERNEL):
        raise ValueError(f"pfblob: unknown kernel {kernel}")
    vx, vy = torch.empty_like(x), torch.empty_like(x)
    if kernel == CUTOFF_KERNEL:
        if method == FMM_METHOD:
            where = "GPU" if hardware == GPU_HARDWARE else "CPU"
            raise Exception(f'FMM calculation of cutoff kernel on the {where} not yet available')
        velocity_cutoff_device(x, y, g, float(sigma) * float(sigma), x, y, vx, vy)
    else:
        ks, xopt, cut = fmm_parameters(float(sigma), float(k))
        velocity_device(x, y, g, ks, x, y, vx, vy, method=method, xopt=xopt, cutoff=cut)
    if integrator == FE_INTEGRATOR:
        # _evolution.py:545-546: x + dt * (v + vInf)
        return x + dt * (vx + vInf[0]), y + dt * (vy + vInf[1])
    kx, ky = vx + vInf[0], vy + vInf[1]
    xn, yn = x.clone(), y.clone()
    for w in RK4_WEIGHTS:  # _evolution.py:692-693: x += w * k * dt
        xn += w * kx * dt
        yn += w * ky * dt
    return xn, yn


def convection(dt, xBlob, yBlob, wBlob, sigma, k=2, kernel=1, vInf=[0.0, 0.0], hardware=0,
               method=1, blocksize=128, integrator=1):
    """New (x, y, g) of the blobs after one convection step of size dt; same
    arguments and results as pHyFlow's ``convection`` (numpy in and out, or
    CUDA tensors in and out).  Every call runs on the GPU (``hardware`` and
    ``blocksize`` are accepted and ignored; ``kernel=0`` is the cutoff
    kernel)."""
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob, "xBlob"), m.dev(yBlob, "yBlob"), m.dev(wBlob, "wBlob")
    require(x.numel(), m.device, xBlob=x, yBlob=y, wBlob=g)
    xn, yn = convection_device(float(dt), x, y, g, sigma, k, (float(vInf[0]), float(vInf[1])),
                               method, integrator, kernel, hardware)
    return m.outs(xn, yn, g.clone())
