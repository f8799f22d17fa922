"""Near-wall shear layer (annulus 1 <= r <= 1.5, exponential vorticity layer)
with 512 vortex panels on the unit circle: FMM blob velocity plus the panel
velocity accumulated on top (LagrangianSolver.evaluateVelocity's sum,
__lagrangianSolverClass.py:257-263), against the FP64 oracle."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err

pytestmark = pytest.mark.gpu


def test_fmm_plus_panels_vs_oracle():
    import pfblob
    from pfblob import workloads as wl
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    b = wl.shear_layer(n=1 << 20)
    ps = wl.cylinder_panels(512)
    x, y, g = T(b.x), T(b.y), T(b.g)
    vx, vy = torch.empty_like(x), torch.empty_like(x)
    ks, xo, cut = pfblob.fmm_parameters(b.sigma)
    pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=pfblob.FMM_METHOD, xopt=xo, cutoff=cut)
    pfblob.panel_velocity_device(*[T(a) for a in (ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa,
                                                  ps.sina)], x, y, vx, vy, accumulate=True)
    idx = np.random.default_rng(3).choice(b.n, 1500, replace=False)
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
    px, py = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina,
                                   b.x[idx], b.y[idx])
    assert normwise_err(vx.cpu().numpy()[idx], vy.cpu().numpy()[idx], rx + px, ry + py) <= 1e-6
    # the blob part alone also meets the gate
    vx2, vy2 = torch.empty_like(x), torch.empty_like(x)
    pfblob.velocity_device(x, y, g, ks, x, y, vx2, vy2, method=pfblob.FMM_METHOD, xopt=xo,
                           cutoff=cut)
    assert normwise_err(vx2.cpu().numpy()[idx], vy2.cpu().numpy()[idx], rx, ry) <= 1e-6


def test_c3_full_size_fmm_plus_panels_and_remesh_conservation():
    """The near-wall shear-layer configuration at its stated size: N = 2^22
    blobs in the annulus plus 512 panels.  FMM blob velocity + panel velocity
    against the FP64 oracle on 2048 seeded targets (gate 1e-6 normwise), then
    the remesh of the layer (window found on the device) with its FP64
    circulation and linear impulse conserved to 1e-12."""
    import pfblob
    from pfblob import workloads as wl
    from pfblob.regrid import remesh_device_async
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    b = wl.shear_layer(n=1 << 22)
    ps = wl.cylinder_panels(512)
    x, y, g = T(b.x), T(b.y), T(b.g)
    vx, vy = torch.empty_like(x), torch.empty_like(x)
    ks, xo, cut = pfblob.fmm_parameters(b.sigma)
    pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=pfblob.FMM_METHOD, xopt=xo, cutoff=cut)
    pfblob.panel_velocity_device(*[T(a) for a in (ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa,
                                                  ps.sina)], x, y, vx, vy, accumulate=True)
    idx = np.sort(np.random.default_rng(5).choice(b.n, 2048, replace=False))
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
    px, py = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina,
                                   b.x[idx], b.y[idx])
    assert normwise_err(vx.cpu().numpy()[idx], vy.cpu().numpy()[idx], rx + px, ry + py) <= 1e-6
    xb, yb = b.bounds()
    h = b.h
    out = remesh_device_async(x, y, g, h, xb[0], yb[0], max_base_cells=int((3.1 / h) ** 2))
    k, st, mom = int(out[3].item()), int(out[4].item()), out[6].cpu().numpy()
    assert st == 0 and k > b.n // 2
    m_in = oracle.moments(b.x, b.y, b.g)
    assert np.allclose(mom[:4], m_in, rtol=1e-12, atol=1e-12 * m_in[3])
    circ, imp = pfblob.conservation_error(mom[:4], mom[4:], float(np.abs(b.x).max()))
    assert circ <= 1e-12 and imp <= 1e-12
