"""Population control on the GPU (pf_population_control and the fused
pf_remesh_population_control) vs the reference PopulationControl (golden
fixtures) and the oracle.

Gates: kept blobs and their order bit-exact, the threshold used equal to the
reference's; the fused remesh + population control equal to remesh followed
by population control."""
import math

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("name", ["popctl_c1", "popctl_decades", "popctl_deep"])
def test_vs_reference_golden(golden, name):
    import pfblob
    d = golden(name)
    tl, tg = float(d["thr_local"]), float(d["thr_global"])
    xo, yo, go = pfblob.PopulationControl(d["x"], d["y"], d["g"], tl, tg)
    assert np.array_equal(xo, d["xo"]) and np.array_equal(yo, d["yo"])
    assert np.array_equal(go, d["go"])
    _, _, _, thr = pfblob.population_control_device(_dev(d["x"]), _dev(d["y"]), _dev(d["g"]), tl, tg)
    assert thr == oracle.population_control(d["x"], d["y"], d["g"], tl, tg)[3]


def test_large_random_vs_oracle():
    import pfblob
    rng = np.random.Generator(np.random.PCG64(5))
    n = 3_000_000
    x = rng.uniform(0, 1, n)
    y = rng.uniform(0, 1, n)
    g = rng.standard_normal(n) * 10.0 ** rng.uniform(-16, -4, n)
    for tl, tg in ((1e-8, 1e-8), (1e-4, 1e-9), (1.0, 1e-40)):
        ex, ey, eg, et = oracle.population_control(x, y, g, tl, tg)
        xo, yo, go, thr = pfblob.population_control_device(_dev(x), _dev(y), _dev(g), tl, tg)
        assert thr == et
        assert np.array_equal(go.cpu().numpy(), eg) and np.array_equal(xo.cpu().numpy(), ex)
        assert np.array_equal(yo.cpu().numpy(), ey)


def test_edge_cases():
    import pfblob
    from pfblob._lib import PfError
    e = torch.zeros(0, dtype=torch.float64, device="cuda")
    xo, yo, go, thr = pfblob.population_control_device(e, e, e, 1e-8, 1e-8)
    assert xo.numel() == 0 and thr == 1e-8
    # everything below the threshold and the loss admissible: all dropped
    g = _dev(np.full(1000, 1e-12))
    xo, _, _, thr = pfblob.population_control_device(g, g, g, 1e-8, 1e-6)
    assert xo.numel() == 0 and thr == 1e-8
    # NaN circulations are never flagged (|NaN| < thr is false): kept
    gn = np.array([1.0, np.nan, 1e-12, -2.0])
    _, _, go, _ = pfblob.population_control_device(_dev(gn), _dev(gn), _dev(gn), 1e-8, 1e-8)
    assert go.numel() == 3 and math.isnan(float(go[1]))
    # a global limit <= 0 never ends the reference's loop: rejected
    with pytest.raises(PfError):
        pfblob.population_control_device(g, g, g, 1e-8, 0.0)
    with pytest.raises(PfError):
        pfblob.population_control_device(g, g, g, float("inf"), 1e-8)


@pytest.mark.parametrize("name", ["regrid_c1", "regrid_rand_c3"])
def test_fused_remesh_equals_remesh_then_control(golden, name):
    import pfblob
    r = golden(name)
    h = float(r["sigma"]) * float(r["overlap"])
    x, y, g = _dev(r["x"]), _dev(r["y"]), _dev(r["g"])
    xb, yb, c = float(r["xb"][0]), float(r["yb"][0]), float(r["c"])
    for tl, tg in ((1e-8, 1e-8), (1e-5, 1e-9)):
        xn, yn, gn = pfblob.remesh_device(x, y, g, h, xb, yb, c)
        ex, ey, eg, et = pfblob.population_control_device(xn, yn, gn, tl, tg)
        fx, fy, fg, ft = pfblob.remesh_device(x, y, g, h, xb, yb, c, population_control=(tl, tg))
        assert ft == et
        assert torch.equal(fx, ex) and torch.equal(fy, ey) and torch.equal(fg, eg)
        # and against the reference's Regrid -> PopulationControl on the host
        ox, oy, og, ot = oracle.population_control(r["xn"], r["yn"], r["gn"], tl, tg)
        assert ot == ft and np.array_equal(fx.cpu().numpy(), ox)


def test_blobs_evolve_fused_step_matches_separate_steps():
    import pfblob
    from pfblob import workloads as wl
    c1 = wl.lamb_oseen_lattice()
    kw = dict(timeIntegrationParams={"method": "euler"},
              velocityComputationParams={"method": "direct", "hardware": "gpu"})
    b = pfblob.Blobs((c1.x, c1.y, c1.g), (0.0, 0.0), 0.0, 0.01, c1.h, c1.overlap, **kw)
    b.evolve()
    # the same step done by hand: velocity, move, remesh, then population control
    r = pfblob.Blobs((c1.x, c1.y, c1.g), (0.0, 0.0), 0.0, 0.01, c1.h, c1.overlap, **kw)
    vx, vy = r.evaluateVelocity()
    x = r.x + vx * 0.01
    y = r.y + vy * 0.01
    h = r.h
    xn, yn, gn = pfblob.Regrid(x, y, r.g, r.sigma, r.overlap, [-1.5 * h, 1.5 * h], [-1.5 * h, 1.5 * h])
    xo, yo, go = pfblob.PopulationControl(xn, yn, gn, 1e-8, 1e-8)
    assert b.numBlobs == go.size
    assert np.array_equal(b.x, xo) and np.array_equal(b.y, yo) and np.array_equal(b.g, go)
