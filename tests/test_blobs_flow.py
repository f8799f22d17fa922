"""The Blobs orchestration on the host (no GPU): construction, evolve and the
property surface run with the device entry points replaced by the oracle on
CPU tensors, and are compared with the same sequence of oracle steps written
out by hand (the reference's order: convection, diffusion, redistribution,
time advance, population control; __blobsClass.py:705-781), and the
convection function against the reference's integrators.  This checks the
orchestration only; the device kernels are checked against the oracle by the
GPU tests."""
import numpy as np
import pytest
import torch

import oracle
from pfblob import blobs as B
from pfblob import evolution as E
from pfblob import workloads as wl

T = torch.from_numpy


def _velocity(x, y, g, ks, xt, yt, vx, vy, **kw):
    rx, ry = oracle.velocity_direct(x.numpy(), y.numpy(), g.numpy(), ks, xt.numpy(), yt.numpy())
    vx.copy_(T(rx))
    vy.copy_(T(ry))


def _remesh(x, y, g, h, xb0, yb0, c=0.0, population_control=None, tutty_hnu=None, **kw):
    xb, yb = [xb0, -xb0], [yb0, -yb0]
    if tutty_hnu is not None:
        xn, yn, gn, _, _ = oracle.diffusion_tutty(x.numpy(), y.numpy(), g.numpy(), tutty_hnu ** 2,
                                                  1.0, h, 1.0, xb, yb)
        return T(xn), T(yn), T(gn)
    xn, yn, gn, _, _ = oracle.regrid(x.numpy(), y.numpy(), g.numpy(), h, 1.0, xb, yb, c)
    if population_control is None:
        return T(xn), T(yn), T(gn)
    xk, yk, gk, thr = oracle.population_control(xn, yn, gn, *population_control)
    return T(xk), T(yk), T(gk), thr


def _popctl(x, y, g, tl, tg, **kw):
    xk, yk, gk, thr = oracle.population_control(x.numpy(), y.numpy(), g.numpy(), tl, tg)
    return T(xk), T(yk), T(gk), thr


@pytest.fixture
def host_blobs(monkeypatch):
    monkeypatch.setattr(B.Blobs, "_device_for", staticmethod(lambda device: torch.device("cpu")))
    monkeypatch.setattr(B, "velocity_device", _velocity)
    monkeypatch.setattr(E, "velocity_device", _velocity)
    monkeypatch.setattr(B, "remesh_device", _remesh)
    monkeypatch.setattr(B, "population_control_device", _popctl)
    return B.Blobs


def _c1():
    c1 = wl.lamb_oseen_lattice(n_side=30, h=0.05)
    rng = np.random.default_rng(5)
    # off the lattice, so that the first redistribution moves every blob
    return c1, c1.x + 0.3 * c1.h * rng.random(c1.n), c1.y - 0.2 * c1.h * rng.random(c1.n)


def _regrid(x, y, g, h, c=0.0):
    b = [-1.5 * h, 1.5 * h]
    return oracle.regrid(x, y, g, h, 1.0, b, b, c)[:3]


def test_construction_is_population_control_then_redistribution(host_blobs):
    c1, x, y = _c1()
    b = host_blobs((x, y, c1.g), vInf=[0.0, 0.0], nu=0.0, deltaTc=0.01, h=c1.h, overlap=0.8)
    xk, yk, gk, _ = oracle.population_control(x, y, c1.g, 1e-8, 1e-8)
    rx, ry, rg = _regrid(xk, yk, gk, c1.h)
    assert np.array_equal(b.x, rx) and np.array_equal(b.y, ry) and np.array_equal(b.g, rg)
    assert b.numBlobs == rx.shape[0] and b.tStep == 0 and b.t == 0.0


def test_euler_step_with_wee_diffusion(host_blobs):
    c1, x, y = _c1()
    nu, dt, vinf = 1e-3, 0.01, (0.1, -0.05)
    ctl = {'stepRedistribution': 1, 'stepPopulationControl': 1,
           'gThresholdLocal': 1e-10, 'gThresholdGlobal': 1e-10}
    b = host_blobs((x, y, c1.g), vInf=list(vinf), nu=nu, deltaTc=dt, h=c1.h, overlap=0.8,
                   timeIntegrationParams={'method': 'euler'}, blobControlParams=ctl,
                   velocityComputationParams={'method': 'direct', 'hardware': 'gpu'})
    x0, y0, g0 = b.x, b.y, b.g
    b.evolve()
    # by hand: Euler, Wee diffusion (tStep 0 is a multiple of stepDiffusion),
    # redistribution, time advance, population control
    sigma = c1.h / 0.8
    vx, vy = oracle.velocity_direct(x0, y0, g0, 2 * sigma * sigma, x0, y0)
    x1 = T(x0) + (T(vx) + vinf[0]) * dt
    y1 = T(y0) + (T(vy) + vinf[1]) * dt
    h = sigma * 0.8
    c = np.sqrt(nu * b.deltaTd) / c1.h
    x2, y2, g2 = _regrid(x1.numpy(), y1.numpy(), g0, h, c)
    x3, y3, g3 = _regrid(x2, y2, g2, h)
    x4, y4, g4, _ = oracle.population_control(x3, y3, g3, 1e-10, 1e-10)
    assert np.array_equal(b.x, x4) and np.array_equal(b.y, y4) and np.array_equal(b.g, g4)
    assert b.tStep == 1 and b.t == dt


def test_rk4_step_applies_the_reference_weights(host_blobs):
    c1, x, y = _c1()
    ctl = {'stepRedistribution': 0, 'stepPopulationControl': 0,
           'gThresholdLocal': 1e-8, 'gThresholdGlobal': 1e-8}
    b = host_blobs((x, y, c1.g), vInf=[0.2, 0.0], nu=0.0, deltaTc=0.02, h=c1.h, overlap=0.8,
                   blobControlParams=ctl)
    assert np.array_equal(b.x, x)  # no construction-time steps
    b.evolve()
    sigma = c1.h / 0.8
    vx, vy = oracle.velocity_direct(x, y, c1.g, 2 * sigma * sigma, x, y)
    kx, ky = T(vx) + 0.2, T(vy) + 0.0
    xr, yr = T(x).clone(), T(y).clone()
    for w in (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0):
        xr += w * kx * 0.02
        yr += w * ky * 0.02
    assert np.array_equal(b.x, xr.numpy()) and np.array_equal(b.y, yr.numpy())
    assert b.tStep == 1


def test_tutty_step_redistributes_then_diffuses(host_blobs):
    c1, x, y = _c1()
    nu, dt = 1e-3, 0.01
    ctl = {'stepRedistribution': 0, 'stepPopulationControl': 0,
           'gThresholdLocal': 1e-8, 'gThresholdGlobal': 1e-8}
    b = host_blobs((x, y, c1.g), vInf=[0.0, 0.0], nu=nu, deltaTc=dt, h=c1.h, overlap=0.8,
                   timeIntegrationParams={'method': 'euler'}, blobControlParams=ctl,
                   diffusionParams={'method': 'regrid_tutty'})
    assert b.deltaTd == dt and b.stepDiffusion == 1
    b.evolve()
    sigma = c1.h / 0.8
    vx, vy = oracle.velocity_direct(x, y, c1.g, 2 * sigma * sigma, x, y)
    x1 = (T(x) + T(vx) * dt).numpy()
    y1 = (T(y) + T(vy) * dt).numpy()
    h = sigma * 0.8
    x2, y2, g2 = _regrid(x1, y1, c1.g, h)
    b0 = [-1.5 * h, 1.5 * h]
    x3, y3, g3, _, _ = oracle.diffusion_tutty(x2, y2, g2, np.sqrt(dt * nu) ** 2, 1.0, h, 1.0,
                                              b0, b0)
    assert np.array_equal(b.x, x3) and np.array_equal(b.y, y3) and np.array_equal(b.g, g3)


def test_property_surface(host_blobs):
    c1, x, y = _c1()
    b = host_blobs((x, y, c1.g), vInf=[0.0, 0.0], nu=0.0, deltaTc=0.01, h=c1.h, overlap=0.8)
    for name in ("h", "sigma", "overlap", "deltaTc", "deltaTd", "nu", "x", "y", "g", "numBlobs",
                 "tStep", "t", "stepDiffusion", "stepRedistribution", "stepPopulationControl",
                 "gThresholdLocal", "gThresholdGlobal", "integrationMethod", "computationMethod",
                 "diffusionParams", "timeIntegrationParams", "blobControlParams",
                 "velocityComputationParams"):
        getattr(b, name)
        with pytest.raises(AttributeError, match="cannot be manually set"):
            setattr(b, name, 1)
        with pytest.raises(AttributeError):
            delattr(b, name)
    assert b.sigma == c1.h / 0.8 and b.computationMethod == 'fmm' and b.integrationMethod == 'rk4'
    b.vInf = np.array([1.0, 2.0])
    assert np.array_equal(b.vInf, [1.0, 2.0])
    with pytest.raises(ValueError):
        b.vInf = np.zeros(3)
    b.hardware = 'cpu'
    assert b.hardware == 'cpu' and b.velocityComputationParams['hardware'] == 'cpu'
    with pytest.raises(ValueError):
        b.hardware = 'tpu'
    assert b.plotVelocity is False
    b.plotVelocity = True
    with pytest.raises(TypeError):
        b.plotVelocity = 1
    assert b.evaluateVorticity(np.zeros(2), np.zeros(2)) is None


def test_convection_matches_the_reference_integrators(monkeypatch):
    """convection_device with the oracle velocity against the reference's two
    integrators written out in numpy: forward Euler (_evolution.py:539-546)
    and the RK4 loop with its stage increment left at zero (:664-693), four
    velocity evaluations included."""
    monkeypatch.setattr(E, "velocity_device", _velocity)
    c1, x, y = _c1()
    g = c1.g
    sigma, dt, vinf = c1.h / 0.8, 0.02, (0.3, -0.1)
    ks = 2 * sigma * sigma
    # forward Euler
    xn, yn = E.convection_device(dt, T(x), T(y), T(g), sigma, vInf=vinf, integrator=0)
    vx, vy = oracle.velocity_direct(x, y, g, ks, x, y)
    assert np.array_equal(xn.numpy(), x + dt * (vx + vinf[0]))
    assert np.array_equal(yn.numpy(), y + dt * (vy + vinf[1]))
    # RK4 as the reference runs it
    xr, yr = x.copy(), y.copy()
    kx_rk4, ky_rk4 = np.zeros(x.shape), np.zeros(y.shape)
    tf = np.array([0.0, 0.5, 0.5, 1.0])
    kw = np.array([1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0])
    for i in range(4):
        xs, ys = x + kx_rk4 * dt * tf[i], y + ky_rk4 * dt * tf[i]
        vx, vy = oracle.velocity_direct(xs, ys, g, ks, xs, ys)
        xr += kw[i] * (vx + vinf[0]) * dt
        yr += kw[i] * (vy + vinf[1]) * dt
    xn, yn = E.convection_device(dt, T(x), T(y), T(g), sigma, vInf=vinf, integrator=1)
    assert np.array_equal(xn.numpy(), xr) and np.array_equal(yn.numpy(), yr)
    with pytest.raises(ValueError):
        E.convection_device(dt, T(x), T(y), T(g), sigma, integrator=2)
