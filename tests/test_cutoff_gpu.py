"""Cutoff (Rosenhead-Krasny) kernel on the GPU: velocity
(pf_velocity_direct_cutoff) and induced vorticity
(pf_vorticity_direct_cutoff) against the reference's own vv2par_C_cpu /
ww2par_C_cpu loops (golden) and the FP64 oracle, through the reference's
dispatchers (``velocity(kernel=0)``, ``vorticity(kernel=0)``, ``convection``).
Gate: normwise relative error <= 1e-6 (velocity as in the other velocity
tests, vorticity max |w - w_ref| / max |w_ref|)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def werr(w, r):
    return float(np.abs(np.asarray(w) - r).max() / np.abs(r).max())


def test_c1_vs_reference_golden(golden):
    import pfblob
    d = golden("cutoff_c1")
    vx, vy = pfblob.velocity(d["x"], d["y"], d["g"], float(d["sigma"]), kernel=0, method=1)
    assert normwise_err(vx, vy, d["vx"], d["vy"]) <= TOL
    w = pfblob.vorticity(d["x"], d["y"], d["g"], float(d["sigma"]), kernel=0)
    assert werr(w, d["w"]) <= TOL


def test_edge_cases_and_separate_targets_vs_reference_golden(golden):
    import pfblob
    d = golden("cutoff_rand")
    vx, vy = pfblob.velocity(d["x"], d["y"], d["g"], float(d["sigma"]), kernel=0, method=1,
                             xEval=d["xt"], yEval=d["yt"], hardware=1)
    assert np.all(np.isfinite(vx)) and np.all(np.isfinite(vy))
    assert normwise_err(vx, vy, d["vx"], d["vy"]) <= TOL
    w = pfblob.vorticity(d["x"], d["y"], d["g"], float(d["sigma"]), kernel=0, xEval=d["xt"],
                         yEval=d["yt"])
    assert werr(w, d["w"]) <= TOL


@pytest.mark.parametrize("n", [1, 300, 5000, 70000])
def test_sizes_vs_oracle(n):
    """The source-segment path (small sets) and the plain path."""
    import pfblob
    rng = np.random.default_rng(100 + n)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    sigma = 0.004
    xt, yt = rng.random(2048), rng.random(2048)
    rx, ry = oracle.velocity_direct_cutoff(x, y, g, sigma * sigma, xt, yt)
    vx, vy = pfblob.velocity(x, y, g, sigma, kernel=0, method=1, xEval=xt, yEval=yt)
    assert normwise_err(vx, vy, rx, ry) <= TOL
    rw = oracle.vorticity_direct_cutoff(x, y, g, sigma * sigma, xt, yt)
    w = pfblob.vorticity(x, y, g, sigma, kernel=0, xEval=xt, yEval=yt)
    assert werr(w, rw) <= TOL


def test_device_tensors_and_convection():
    """CUDA tensors in, CUDA tensors out; a forward-Euler convection step with
    the cutoff kernel moves the blobs by dt (v + vInf) of the oracle velocity."""
    import pfblob
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    n = 4000
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    sigma, dt, vinf = 0.01, 1e-3, (0.2, -0.1)
    T = lambda a: torch.from_numpy(a).to(dev)
    vx, vy = pfblob.velocity(T(x), T(y), T(g), sigma, kernel=0, method=1)
    assert isinstance(vx, torch.Tensor) and vx.is_cuda
    rx, ry = oracle.velocity_direct_cutoff(x, y, g, sigma * sigma)
    assert normwise_err(vx.cpu().numpy(), vy.cpu().numpy(), rx, ry) <= TOL
    xn, yn, gn = pfblob.convection(dt, x, y, g, sigma, kernel=0, vInf=list(vinf), method=1,
                                   integrator=0)
    ex, ey = x + dt * (rx + vinf[0]), y + dt * (ry + vinf[1])
    assert np.abs(xn - ex).max() <= 1e-6 * dt * np.abs(rx).max() + 1e-15
    assert np.abs(yn - ey).max() <= 1e-6 * dt * np.abs(ry).max() + 1e-15
    assert np.array_equal(gn, g)


def test_fmm_with_cutoff_kernel_raises_as_the_reference():
    import pfblob
    x = np.random.default_rng(1).random(100)
    for hw, where in ((0, "CPU"), (1, "GPU")):
        with pytest.raises(Exception, match=f"FMM calculation of cutoff kernel on the {where}"):
            pfblob.velocity(x, x, x, 0.01, kernel=0, method=0, hardware=hw)
