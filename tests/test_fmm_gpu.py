"""FMM blob velocity on the GPU vs the FP64 direct oracle (the reference's own
direct Gauss sum restated; pinned to the reference Cython kernel).

Gate: max_i |v_i - v_ref_i| / max_i |v_ref_i| <= 1e-6 (at the default tol)."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err
from oracle import lists

pytestmark = pytest.mark.gpu
TOL = 1e-6
DEV = torch.device("cuda", 0)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def fmm(x, y, g, sigma, xt=None, yt=None, tol=1e-6, ndirect=35):
    import pfblob
    vx, vy = pfblob.velocity(T(x), T(y), T(g), sigma, method=pfblob.FMM_METHOD, hardware=1,
                             xEval=None if xt is None else T(xt),
                             yEval=None if yt is None else T(yt), tol=tol, Ndirect=ndirect)
    return vx.cpu().numpy(), vy.cpu().numpy()


def test_c1_lamb_oseen_vs_reference_golden(golden):
    d = golden("direct_c1")
    vx, vy = fmm(d["x"], d["y"], d["g"], float(d["sigma"]), ndirect=8)
    assert normwise_err(vx, vy, d["vx"], d["vy"]) <= TOL


def test_random_vs_reference_fmm_golden(golden):
    """Same input the reference CPU FMM was run on (tests/golden/fmm_rand)."""
    f = golden("fmm_rand")
    sig = float(f["sigma"])
    vx, vy = fmm(f["x"], f["y"], f["g"], sig, ndirect=8)
    rx, ry = oracle.velocity_direct(f["x"], f["y"], f["g"], 2 * sig * sig)
    assert normwise_err(vx, vy, rx, ry) <= TOL
    # and within 2e-6 of the reference's own FMM result
    assert normwise_err(vx, vy, f["vx"], f["vy"]) <= 2e-6


@pytest.mark.parametrize("n,sigma,seed", [(20000, 0.002, 1), (50000, 0.01, 2), (65536, 0.002, 3)])
def test_uniform_vs_oracle(n, sigma, seed):
    rng = np.random.default_rng(seed)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    vx, vy = fmm(x, y, g, sigma)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma)
    assert normwise_err(vx, vy, rx, ry) <= TOL


def test_c2_full_size_subset_vs_oracle():
    """C2 (N = 2^20, sigma = 0.002) at all blobs; oracle on 4096 of them."""
    from pfblob import workloads as wl
    b = wl.uniform_square()
    vx, vy = fmm(b.x, b.y, b.g, b.sigma)
    idx = np.random.default_rng(4).choice(b.n, 4096, replace=False)
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[idx], b.y[idx])
    assert normwise_err(vx[idx], vy[idx], rx, ry) <= TOL


def test_shear_layer_annulus_subset():
    """Non-uniform fill (annulus) with separate targets."""
    from pfblob import workloads as wl
    b = wl.shear_layer(n=1 << 18)
    rng = np.random.default_rng(5)
    xt = rng.uniform(-1.6, 1.6, 3000)
    yt = rng.uniform(-1.6, 1.6, 3000)
    vx, vy = fmm(b.x, b.y, b.g, b.sigma, xt, yt)
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, xt, yt)
    assert normwise_err(vx, vy, rx, ry) <= TOL


def test_mixed_instance_and_clusters():
    from pfblob import workloads as wl
    b = wl.mixed_instance(100000, config=4, instance=1)
    x, y, g = b.x.copy(), b.y.copy(), b.g.copy()
    x[:5000] = 0.3 + 1e-4 * np.random.default_rng(6).standard_normal(5000)  # dense cluster
    y[:5000] = -0.2 + 1e-4 * np.random.default_rng(7).standard_normal(5000)
    vx, vy = fmm(x, y, g, b.sigma)
    idx = np.random.default_rng(8).choice(x.shape[0], 3000, replace=False)
    idx[:100] = np.arange(100)
    rx, ry = oracle.velocity_direct(x, y, g, b.ksigmasqr, x[idx], y[idx])
    assert normwise_err(vx[idx], vy[idx], rx, ry) <= TOL


def test_tol_zero_is_direct_and_small_n():
    import pfblob
    rng = np.random.default_rng(9)
    x, y, g = rng.random(500), rng.random(500), rng.standard_normal(500)
    a = fmm(x, y, g, 0.01, tol=0.0)
    b = pfblob.velocity(x, y, g, 0.01, method=1)
    assert np.array_equal(a[0], b[0])
    c = fmm(x, y, g, 0.01)  # too small for a tree: direct path
    assert normwise_err(c[0], c[1], b[0], b[1]) <= TOL


def test_deterministic_repeat():
    from pfblob import workloads as wl
    b = wl.uniform_square(n=200000, config=2, instance=5)
    a = fmm(b.x, b.y, b.g, b.sigma)
    c = fmm(b.x, b.y, b.g, b.sigma)
    assert np.array_equal(a[0], c[0]) and np.array_equal(a[1], c[1])


def test_morton_keys_bit_exact():
    import pfblob._lib as lb
    from pfblob._arrays import ptr
    from pfblob import workloads as wl
    b = wl.uniform_square(n=300000, config=2, instance=6)
    x, y = T(b.x), T(b.y)
    L = 9
    x0, y0, w = 0.0, 0.0, 1.0 / 512
    keys = torch.empty(b.n, dtype=torch.int32, device=DEV)
    lb.check(lb.lib.pf_fmm_tree_keys(lb.context(0), b.n, ptr(x), ptr(y), x0, y0, w, L,
                                     ptr(keys), None))
    got = keys.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, lists.leaf_keys(b.x, b.y, x0, y0, w, L))


def test_nan_input_rejected():
    import pfblob
    x = np.random.default_rng(1).random(5000)
    x[7] = np.nan
    with pytest.raises(pfblob._lib.PfError) as ei:
        fmm(x, x, x, 0.01)
    assert ei.value.status == 5


def test_point_vortex_limit_theta_bound():
    """sigma far below the leaf width: every separation is set by theta alone,
    so the multipole truncation (not the near field) bounds the error."""
    rng = np.random.default_rng(10)
    n = 200000
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    sigma = 1e-5
    vx, vy = fmm(x, y, g, sigma)
    idx = rng.choice(n, 3000, replace=False)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma, x[idx], y[idx])
    assert normwise_err(vx[idx], vy[idx], rx, ry) <= TOL


def test_caller_box_equals_computed_box():
    """pf_velocity_fmm_box with the exact bounding box gives bitwise the
    pf_velocity_fmm result; a larger box is a different tree, same tolerance."""
    import pfblob
    from pfblob import workloads as wl
    b = wl.uniform_square(n=150000, config=2, instance=9)
    x, y, g = T(b.x), T(b.y), T(b.g)
    ks, xo, cut = pfblob.fmm_parameters(b.sigma)
    out = []
    for box in (None, (b.x.min(), b.x.max(), b.y.min(), b.y.max()), (-0.5, 1.5, -0.25, 1.25)):
        vx, vy = torch.empty_like(x), torch.empty_like(x)
        pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=pfblob.FMM_METHOD, xopt=xo,
                               cutoff=cut, box=box)
        out.append((vx.cpu().numpy(), vy.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert normwise_err(out[2][0], out[2][1], out[0][0], out[0][1]) <= TOL


def test_stats_pair_counts():
    """pf_fmm_last_stats (the C struct read through ctypes): sizes as given,
    the far-pair count (sources beyond the Gaussian's reach of their whole
    target group) strictly between 0 and the near-field pair count for a
    uniform set, the pair count between n and n^2, M2L translations > 0."""
    import pfblob
    from pfblob import _lib
    n, sigma = 65536, 0.002
    rng = np.random.default_rng(11)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    fmm(x, y, g, sigma)
    st = _lib.fmm_last_stats(0)
    assert st["used_direct"] == 0
    assert st["n_src"] == n and st["n_tgt"] == n
    assert 0 < st["p2p_pairs_far"] < st["p2p_pairs"]
    assert st["m2l_translations"] > 0
    assert n <= st["p2p_pairs"] <= n * n  # each blob meets at least itself


def test_plan_reused_while_the_box_drifts():
    """A blob set that moves a little every step (its box width drifting by
    about 1e-4) keeps its FMM plan: plans are keyed by the separation key of
    cutoff / width, not by the exact ratio.  Results stay within the gate."""
    import pfblob
    from pfblob import _lib
    from pfblob import workloads as wl
    b = wl.uniform_square(n=65536, sigma=0.004, config=2, instance=21)
    fmm(b.x, b.y, b.g, b.sigma)  # builds (or finds) the plan
    n0 = _lib.fmm_plan_builds()
    rng = np.random.default_rng(1)
    for step in range(8):
        s = 1.0 + 1e-4 * rng.uniform(-1.0, 1.0)
        x, y = 0.5 + (b.x - 0.5) * s, 0.5 + (b.y - 0.5) * s
        vx, vy = fmm(x, y, b.g, b.sigma)
    assert _lib.fmm_plan_builds() - n0 <= 1
    idx = np.arange(0, b.n, 97)
    rx, ry = oracle.velocity_direct(x, y, b.g, 2 * b.sigma ** 2, x[idx], y[idx])
    assert normwise_err(vx[idx], vy[idx], rx, ry) <= TOL


@pytest.mark.parametrize("terms", [16, 20, 24, 28, 32])
@pytest.mark.parametrize("sigma", [0.002, 1e-5])
def test_every_expansion_order_vs_oracle(terms, sigma):
    """Every instantiated expansion order, forced through pf_fmm_set_tuning
    (the tensor-core M2M, M2L and L2L pad their 8 x 4 tiles for 20 and 28
    terms); sigma = 1e-5 is the point-vortex limit, where the far field
    carries most of the velocity."""
    from pfblob import _lib
    rng = np.random.default_rng(7)
    n = 30000
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    _lib.fmm_set_tuning(0, terms, 1)
    try:
        vx, vy = fmm(x, y, g, sigma)
        st = _lib.fmm_last_stats(DEV.index)
    finally:
        _lib.fmm_set_tuning(0, 0, 1)
    assert st["expansion_terms"] == terms
    sub = np.arange(0, n, 15)
    rx, ry = oracle.velocity_direct(x, y, g, 2 * sigma * sigma, x[sub].copy(), y[sub].copy())
    assert normwise_err(vx[sub], vy[sub], rx, ry) <= TOL
