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
