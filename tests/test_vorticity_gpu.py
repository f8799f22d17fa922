"""Induced vorticity of Gaussian blobs on the GPU (pf_vorticity_direct) vs the
reference's own ww2parGauss loop (golden) and the FP64 oracle.

Tolerance: max_i |w_i - w_ref_i| / max_i |w_ref_i| <= 1e-6."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-6


def err(w, r):
    return float(np.abs(np.asarray(w) - r).max() / np.abs(r).max())


def test_c1_vs_reference_golden(golden):
    import pfblob
    d = golden("vort_c1")
    w = pfblob.vorticity(d["x"], d["y"], d["g"], float(d["sigma"]))
    assert err(w, d["w"]) <= TOL


def test_edge_cases_and_separate_targets_vs_reference_golden(golden):
    import pfblob
    d = golden("vort_rand")
    w = pfblob.vorticity(d["x"], d["y"], d["g"], float(d["sigma"]), xEval=d["xt"], yEval=d["yt"])
    assert np.all(np.isfinite(w))
    assert err(w, d["w"]) <= TOL


@pytest.mark.parametrize("n", [1, 300, 5000, 70000])
def test_sizes_vs_oracle_and_repeatable(n):
    """Covers the source-segment path (small sets) and the plain path."""
    import pfblob
    rng = np.random.default_rng(n)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    sigma = 0.005
    a = pfblob.vorticity(x, y, g, sigma)
    b = pfblob.vorticity(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(),
                         torch.from_numpy(g).cuda(), sigma)
    assert np.array_equal(a, b.cpu().numpy())
    sub = rng.choice(n, min(n, 2000), replace=False)
    r = oracle.vorticity_direct(x, y, g, 2 * sigma * sigma, x[sub].copy(), y[sub].copy())
    assert err(a[sub], r) <= TOL


def test_empty_and_options():
    import pfblob
    x = np.zeros(0)
    assert pfblob.vorticity(x, x, x, 0.01).shape == (0,)
    w = pfblob.vorticity(x, x, x, 0.01, xEval=np.ones(3), yEval=np.ones(3))
    assert np.array_equal(w, np.zeros(3))
    with pytest.raises(Exception):
        pfblob.vorticity(np.ones(3), np.ones(3), np.ones(3), 0.01, method=0)
