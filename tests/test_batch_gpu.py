"""Batched execution (one CUDA graph launch for many simulations) vs the
single-simulation calls: every result is the same alone and in the mix
(bitwise: same kernels, same trees), and within 1e-6 of the FP64 oracle."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def make_sims(sizes, config=4):
    from pfblob import workloads as wl
    sims = []
    for i, n in enumerate(sizes):
        b = wl.mixed_instance(int(n), config=config, instance=i)
        sims.append({"x": T(b.x), "y": T(b.y), "g": T(b.g), "sigma": b.sigma, "blob": b})
    return sims


def alone(s, method, L):
    import pfblob
    from pfblob import _lib
    b = s["blob"]
    ks, xo, cut = pfblob.fmm_parameters(b.sigma)
    vx, vy = torch.empty_like(s["x"]), torch.empty_like(s["x"])
    if method == 0:
        _lib.fmm_set_tuning(L, 0, 1)
        try:
            pfblob.velocity_device(s["x"], s["y"], s["g"], ks, s["x"], s["y"], vx, vy, method=0,
                                   xopt=xo, cutoff=cut, tol=1e-6)
        finally:
            _lib.fmm_set_tuning(0, 0, 1)
    else:
        pfblob.velocity_device(s["x"], s["y"], s["g"], ks, s["x"], s["y"], vx, vy, method=1)
    xb, yb = b.bounds()
    xn, yn, gn = pfblob.remesh_device(s["x"], s["y"], s["g"], b.h, xb[0], yb[0])
    return vx, vy, xn, yn, gn


def test_batch_equals_alone_and_oracle():
    from pfblob.batch import Batch
    sizes = [700, 2048, 5000, 12000, 30000, 64000, 150000, 3000]
    sims = make_sims(sizes)
    bt = Batch(sims, tol=1e-6, n_streams=4)
    methods = [r["method"] for r in bt.sims]
    assert 0 in methods and 1 in methods, methods  # both paths exercised
    bt.run()
    res = bt.results()
    for s, r in zip(sims, res):
        assert r["status"] == 0
        vx, vy, xn, yn, gn = alone(s, r["method"], r["leaf_level"])
        assert torch.equal(vx, r["vx"]) and torch.equal(vy, r["vy"])
        assert torch.equal(xn, r["x"]) and torch.equal(yn, r["y"]) and torch.equal(gn, r["g"])
    # accuracy of one instance of each method against the FP64 oracle
    for want in (0, 1):
        i = methods.index(want)
        b = sims[i]["blob"]
        idx = np.random.default_rng(i).choice(b.n, min(b.n, 2000), replace=False)
        rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
        assert normwise_err(res[i]["vx"].cpu().numpy()[idx], res[i]["vy"].cpu().numpy()[idx],
                            rx, ry) <= 1e-6
    bt.close()


def test_batch_replay_is_deterministic_and_tracks_inputs():
    from pfblob.batch import Batch
    sims = make_sims([4000, 20000, 90000], config=5)
    bt = Batch(sims, tol=1e-6, n_streams=2)
    bt.run()
    a = [(r["vx"].clone(), r["g"].clone()) for r in bt.results()]
    bt.run()
    b = bt.results()
    for (vx, g), r in zip(a, b):
        assert torch.equal(vx, r["vx"]) and torch.equal(g, r["g"])
    # the graph reads the inputs in place: scaling circulations scales velocities
    for s in sims:
        s["g"].mul_(2.0)
    bt.run()
    c = bt.results()
    for (vx, _), r in zip(a, c):
        assert torch.allclose(r["vx"], 2.0 * vx, rtol=1e-6, atol=1e-12)
    bt.close()


def test_autotuner_prefers_direct_for_small_and_fmm_for_large():
    from pfblob.tune import Tuner
    t = Tuner(0)
    assert t.choose(2000, 2 * 0.005 ** 2, (-1, 1, -1, 1))[0] == 1
    assert t.choose(1 << 20, 2 * 0.002 ** 2, (0, 1, 0, 1))[0] == 0


def test_batch_of_256_simulations_equals_alone_and_oracle():
    """The batched configuration at its stated size: 256 simulations, N
    log-uniform in [2048, 262144] (Lamb-Oseen + uniform mix, sigma in
    [0.002, 0.01]).  Every simulation's velocity and remesh equal its
    single-simulation calls bitwise; eight of them (both methods) are within
    1e-6 of the FP64 oracle."""
    from pfblob import workloads as wl
    from pfblob.batch import Batch
    sizes = wl.log_uniform_sizes(256, 2048, 262144, config=4)
    sims = make_sims(sizes)
    bt = Batch(sims, tol=1e-6, n_streams=8)
    bt.run()
    res = bt.results()
    methods = [r["method"] for r in bt.sims]
    assert 0 in methods and 1 in methods
    for s, r in zip(sims, res):
        assert r["status"] == 0
        vx, vy, xn, yn, gn = alone(s, r["method"], r["leaf_level"])
        assert torch.equal(vx, r["vx"]) and torch.equal(vy, r["vy"])
        assert torch.equal(xn, r["x"]) and torch.equal(yn, r["y"]) and torch.equal(gn, r["g"])
    picks = [i for i, m in enumerate(methods) if m == 0][:4] + \
            [i for i, m in enumerate(methods) if m == 1][:4]
    for i in picks:
        b = sims[i]["blob"]
        idx = np.random.default_rng(i).choice(b.n, min(b.n, 1000), replace=False)
        rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
        assert normwise_err(res[i]["vx"].cpu().numpy()[idx], res[i]["vy"].cpu().numpy()[idx],
                            rx, ry) <= 1e-6, (i, methods[i])
    bt.close()
