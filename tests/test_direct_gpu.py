"""Direct Gaussian-blob velocity on the GPU vs the FP64 oracle.

Tolerance (the accuracy gate of the velocity): max_i |v_i - v_ref_i| / max_i |v_ref_i| <= 1e-6."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def test_c1_lamb_oseen_vs_reference_golden(golden):
    import pfblob
    d = golden("direct_c1")
    vx, vy = pfblob.velocity(d["x"], d["y"], d["g"], float(d["sigma"]), method=1, hardware=1)
    assert normwise_err(vx, vy, d["vx"], d["vy"]) <= TOL


def test_edge_cases_vs_reference_golden(golden):
    import pfblob
    d = golden("direct_rand")
    vx, vy = pfblob.velocity(d["x"], d["y"], d["g"], float(d["sigma"]), method=1, hardware=1)
    assert np.all(np.isfinite(vx)) and np.all(np.isfinite(vy))
    assert normwise_err(vx, vy, d["vx"], d["vy"]) <= TOL


@pytest.mark.parametrize("n,sigma", [(1, 0.01), (255, 0.01), (257, 0.05), (4099, 0.002),
                                     (20000, 0.002)])
def test_random_sizes_vs_oracle(n, sigma):
    import pfblob
    rng = np.random.default_rng(n)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    vx, vy = pfblob.velocity(x, y, g, sigma, method=1, hardware=1)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma)
    if n == 1:
        assert vx[0] == 0.0 and vy[0] == 0.0
    else:
        assert normwise_err(vx, vy, rx, ry) <= TOL


def test_near_coincident_pairs():
    """Blobs at distances far below sigma (the 1 - exp(-x) series branch)."""
    import pfblob
    rng = np.random.default_rng(5)
    n = 3000
    x, y = rng.random(n), rng.random(n)
    x[1::2] = x[0::2] + rng.uniform(-1e-7, 1e-7, n // 2)
    y[1::2] = y[0::2] + rng.uniform(-1e-7, 1e-7, n // 2)
    g = rng.standard_normal(n) / n
    sigma = 0.002
    vx, vy = pfblob.velocity(x, y, g, sigma, method=1)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma)
    assert normwise_err(vx, vy, rx, ry) <= TOL


def test_separate_targets_and_torch_inputs():
    import pfblob
    rng = np.random.default_rng(9)
    n, m = 5000, 777
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    g = rng.standard_normal(n) / n
    xt, yt = rng.uniform(-1.2, 1.2, m), rng.uniform(-1.2, 1.2, m)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * 0.01 ** 2, xt, yt)
    vx, vy = pfblob.velocity(x, y, g, 0.01, xEval=xt, yEval=yt, method=1)
    assert normwise_err(vx, vy, rx, ry) <= TOL
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(a).to(dev)
    tx, ty = pfblob.velocity(T(x), T(y), T(g), 0.01, xEval=T(xt), yEval=T(yt), method=1)
    assert tx.is_cuda and tx.dtype == torch.float64
    assert np.array_equal(tx.cpu().numpy(), vx) and np.array_equal(ty.cpu().numpy(), vy)


def test_empty_inputs():
    import pfblob
    e = np.zeros(0)
    vx, vy = pfblob.velocity(e, e, e, 0.01, xEval=np.array([0.1, 0.2]),
                             yEval=np.array([0.0, 0.3]), method=1)
    assert np.array_equal(vx, [0.0, 0.0]) and np.array_equal(vy, [0.0, 0.0])
    vx, vy = pfblob.velocity(np.array([0.1]), np.array([0.2]), np.array([1.0]), 0.01,
                             xEval=e, yEval=e, method=1)
    assert vx.shape == (0,)


def test_large_uniform_subset_vs_oracle():
    """C2 shape (N = 2^20, sigma = 0.002) checked on 2048 targets."""
    import pfblob
    from pfblob import workloads as wl
    b = wl.uniform_square()
    idx = np.random.default_rng(1).choice(b.n, 2048, replace=False)
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    vx, vy = pfblob.velocity(T(b.x), T(b.y), T(b.g), b.sigma, xEval=T(b.x[idx]),
                             yEval=T(b.y[idx]), method=1)
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
    assert normwise_err(vx.cpu().numpy(), vy.cpu().numpy(), rx, ry) <= TOL


def test_invalid_sigma_raises():
    import pfblob
    with pytest.raises(pfblob._lib.PfError):
        pfblob.velocity(np.ones(4), np.ones(4), np.ones(4), 0.0, method=1)


@pytest.mark.parametrize("n", [1025, 4096, 30000, 200000])
def test_source_split_sizes_deterministic_vs_oracle(n):
    """Sizes where the sources are cut into segments (fewer target tiles than
    CTAs to fill the GPU): within tolerance, and bitwise repeatable."""
    import pfblob
    rng = np.random.default_rng(n + 7)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    sigma = 0.004
    a = pfblob.velocity(x, y, g, sigma, method=1)
    b = pfblob.velocity(x, y, g, sigma, method=1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    sub = rng.choice(n, min(n, 4096), replace=False)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma, x[sub].copy(), y[sub].copy())
    assert normwise_err(a[0][sub], a[1][sub], rx, ry) <= TOL
