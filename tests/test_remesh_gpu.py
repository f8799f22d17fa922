"""M4' remesh on the GPU vs the reference Regrid (golden) and the oracle.

Gates: lattice indices and new coordinates bit-exact, circulations within
1e-12 relative (normwise), circulation and linear impulse conserved to 1e-12."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
GTOL = 1e-12


def _regrid_gpu(x, y, g, sigma, overlap, xb, yb, c=0.0):
    import pfblob
    return pfblob.Regrid(x, y, g, sigma, overlap, xb, yb, 0, c)


@pytest.mark.parametrize("name", ["regrid_c1", "regrid_rand_c0", "regrid_rand_c3", "regrid_far"])
def test_vs_reference_regrid_golden(golden, name):
    """regrid_far: four blobs thousands of units from the other 2000, so that
    the dense lattice window would hold ~1e11 cells; the remesh then runs on
    the window compressed to the lattice rows and columns the blobs touch."""
    r = golden(name)
    xn, yn, gn = _regrid_gpu(r["x"], r["y"], r["g"], float(r["sigma"]), float(r["overlap"]),
                             r["xb"], r["yb"], float(r["c"]))
    assert xn.shape == r["xn"].shape
    assert np.array_equal(xn, r["xn"]) and np.array_equal(yn, r["yn"])
    assert np.abs(gn - r["gn"]).max() <= GTOL * np.abs(r["gn"]).max()
    # explicit zero-weight cells are kept, as in the reference
    assert np.array_equal(gn == 0.0, r["gn"] == 0.0) or np.abs(gn[r["gn"] == 0]).max() < 1e-300


def test_c2_full_size_indices_bit_exact_and_conservation():
    import pfblob
    from pfblob import workloads as wl
    b = wl.uniform_square()
    xb, yb = b.bounds()
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x, y, g = T(b.x), T(b.y), T(b.g)
    xn, yn, gn, ixn, iyn = pfblob.remesh_device(x, y, g, b.h, xb[0], yb[0], with_indices=True)
    rx, ry, rg, rix, riy = oracle.regrid(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
    assert np.array_equal(ixn.cpu().numpy(), rix) and np.array_equal(iyn.cpu().numpy(), riy)
    assert np.array_equal(xn.cpu().numpy(), rx) and np.array_equal(yn.cpu().numpy(), ry)
    assert np.abs(gn.cpu().numpy() - rg).max() <= GTOL * np.abs(rg).max()
    m0 = pfblob.moments_device(x, y, g).cpu().numpy()
    m1 = pfblob.moments_device(xn, yn, gn).cpu().numpy()
    circ, imp = pfblob.conservation_error(m0, m1, float(np.abs(b.x).max()))
    assert circ <= 1e-12 and imp <= 1e-12


def test_deterministic_repeat():
    import pfblob
    from pfblob import workloads as wl
    b = wl.mixed_instance(50000, config=4, instance=3)
    xb, yb = b.bounds()
    a = _regrid_gpu(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
    c = _regrid_gpu(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
    for u, v in zip(a, c):
        assert np.array_equal(u, v)


def test_coincident_blobs_and_nodes():
    """Many blobs in one cell, blobs exactly on lattice nodes."""
    rng = np.random.default_rng(3)
    h = 0.01
    n = 3000
    x = np.full(n, 0.123)
    y = np.full(n, -0.456)
    x[:1000] = (np.arange(1000) % 37) * h + 0.5 * h - 1.5 * h
    y[:1000] = (np.arange(1000) // 37) * h + 0.5 * h - 1.5 * h
    g = rng.standard_normal(n)
    xb = np.array([-1.5 * h, 1.5 * h])
    xn, yn, gn = _regrid_gpu(x, y, g, h / 0.8, 0.8, xb, xb)
    rx, ry, rg, _, _ = oracle.regrid(x, y, g, h / 0.8, 0.8, xb, xb)
    assert np.array_equal(xn, rx) and np.array_equal(yn, ry)
    assert np.abs(gn - rg).max() <= GTOL * np.abs(rg).max()


@pytest.mark.parametrize("tutty", [False, True])
def test_dense_cells_beyond_one_sort_chunk(tutty):
    """Base cells holding 10 000, 5 000 and 70 blobs (above the per-thread
    sort's 64 and the segment sort's 4096-value chunk) among a spread set:
    lattice nodes bit-exact, circulations within 1e-12, both for the M4'
    and the Tutty weights."""
    import pfblob
    rng = np.random.default_rng(11)
    h = 0.01
    sigma, ov = h / 0.8, 0.8
    parts = []
    for cx, cy, m in ((0.0335, -0.0265, 10000), (0.2035, 0.1535, 5000), (-0.1165, 0.0735, 70)):
        # base cell k holds k h < x <= (k + 1) h: each cluster stays in one cell
        parts.append((cx + 0.3 * h * rng.random(m), cy + 0.3 * h * rng.random(m)))
    parts.append((rng.uniform(-0.3, 0.3, 20000), rng.uniform(-0.3, 0.3, 20000)))
    x = np.concatenate([p[0] for p in parts])
    y = np.concatenate([p[1] for p in parts])
    perm = rng.permutation(x.shape[0])
    x, y = x[perm], y[perm]
    g = rng.standard_normal(x.shape[0])
    b = np.array([-1.5 * h, 1.5 * h])
    if tutty:
        dt, nu = 1e-3, 0.01
        xn, yn, gn = pfblob.diffusion_tutty(dt, nu, 0.0, x, y, g, sigma, b, b, overlap=ov)
        rx, ry, rg, _, _ = oracle.diffusion_tutty(x, y, g, dt, nu, sigma, ov, b, b)
    else:
        xn, yn, gn = _regrid_gpu(x, y, g, sigma, ov, b, b)
        rx, ry, rg, _, _ = oracle.regrid(x, y, g, sigma, ov, b, b)
    assert np.array_equal(xn, rx) and np.array_equal(yn, ry)
    assert np.abs(gn - rg).max() <= GTOL * np.abs(rg).max()
    again = (pfblob.diffusion_tutty(dt, nu, 0.0, x, y, g, sigma, b, b, overlap=ov) if tutty
             else _regrid_gpu(x, y, g, sigma, ov, b, b))
    assert np.array_equal(again[2], gn)  # fixed summation order: bitwise repeatable


def test_single_blob_and_empty():
    import pfblob
    xn, yn, gn = _regrid_gpu(np.array([0.3]), np.array([0.7]), np.array([2.0]), 0.1, 0.8,
                             [-0.12, 0.12], [-0.12, 0.12])
    assert xn.shape == (16,) and abs(gn.sum() - 2.0) < 1e-15
    e = np.zeros(0)
    out = pfblob.Regrid(e, e, e, 0.1, 0.8, [0, 1], [0, 1])
    assert out[0].shape == (0,)


def test_nan_input_is_an_error():
    import pfblob
    x = np.array([0.1, np.nan, 0.3])
    with pytest.raises(pfblob._lib.PfError) as ei:
        pfblob.Regrid(x, x * 0, x * 0 + 1, 0.1, 0.8, [0, 1], [0, 1])
    assert ei.value.status == 5


def test_capacity_error_reports_needed_size():
    import ctypes
    import pfblob
    from pfblob import _lib
    from pfblob._arrays import ptr
    dev = torch.device("cuda", 0)
    x = torch.tensor([0.3, 0.5], dtype=torch.float64, device=dev)
    out = torch.empty(4, dtype=torch.float64, device=dev)
    n = ctypes.c_int64(0)
    s = _lib.lib.pf_remesh(_lib.context(0), 2, ptr(x), ptr(x), ptr(x), 0.08, -0.12, -0.12, 0.0, 4,
                           ptr(out), ptr(out), ptr(out), None, None, ctypes.byref(n), None)
    assert s == 6 and n.value > 4


def test_window_remesh_equals_remesh():
    """The sync-free remesh on the window of the blobs' bounding box gives
    bitwise the pf_remesh result."""
    import pfblob
    from pfblob import workloads as wl
    from pfblob.regrid import lattice_window, remesh_window_device
    b = wl.mixed_instance(100000, config=4, instance=3)
    dev = torch.device("cuda", 0)
    x, y, g = (torch.from_numpy(a).to(dev) for a in (b.x, b.y, b.g))
    h = b.h
    xb, yb = b.bounds()
    xn, yn, gn = pfblob.remesh_device(x, y, g, h, xb[0], yb[0])
    box = (b.x.min(), b.x.max(), b.y.min(), b.y.max())
    win = lattice_window(box, h, xb[0], yb[0])
    wx, wy, wg, nout = remesh_window_device(x, y, g, h, xb[0], yb[0], win)
    k = int(nout.item())
    assert k == xn.numel()
    assert torch.equal(wx[:k], xn) and torch.equal(wy[:k], yn) and torch.equal(wg[:k], gn)


@pytest.mark.parametrize("name", ["tutty_rand", "tutty_rand_nu0", "tutty_c1"])
def test_tutty_vs_reference_golden(golden, name):
    """Tutty diffusive redistribution: lattice nodes and their order bit-exact,
    circulations within 1e-12, circulation and linear impulse conserved."""
    import pfblob
    d = golden(name)
    xn, yn, gn = pfblob.diffusion_tutty(float(d["dt"]), float(d["nu"]), 0.0, d["x"], d["y"],
                                        d["g"], float(d["sigma"]), d["xb"], d["yb"],
                                        overlap=float(d["overlap"]))
    assert np.array_equal(xn, d["xn"]) and np.array_equal(yn, d["yn"])
    assert np.abs(gn - d["gn"]).max() <= GTOL * np.abs(d["gn"]).max()
    m0 = oracle.moments(d["x"], d["y"], d["g"])
    m1 = oracle.moments(xn, yn, gn)
    assert abs(m1[0] - m0[0]) <= 1e-12 * m0[3]
    xs = max(np.abs(d["x"]).max(), np.abs(d["y"]).max())
    assert max(abs(m1[1] - m0[1]), abs(m1[2] - m0[2])) <= 1e-12 * m0[3] * xs


def test_wee_diffusion_matches_remesh_with_c():
    """diffusion_wee is the remesh with c = sqrt(nu dt)/h (oracle Regrid)."""
    import pfblob
    rng = np.random.default_rng(3)
    n = 3000
    x, y = rng.uniform(-0.2, 0.3, n), rng.uniform(-0.2, 0.3, n)
    g = rng.standard_normal(n) / n
    sigma, ov, h, dt, nu = 0.01, 0.8, 0.008, 1e-3, 0.01
    b = np.array([-1.5 * h, 1.5 * h])
    xn, yn, gn = pfblob.diffusion_wee(dt, nu, h, x, y, g, sigma, b, b, overlap=ov)
    c = np.sqrt(nu * dt) / h
    rx, ry, rg, _, _ = oracle.regrid(x, y, g, sigma, ov, b, b, c)
    assert np.array_equal(xn, rx) and np.array_equal(yn, ry)
    assert np.abs(gn - rg).max() <= GTOL * np.abs(rg).max()


def test_async_remesh_equals_remesh_and_reports_its_window():
    """pf_remesh_async (window found on the device, no host synchronisation)
    gives bitwise the pf_remesh result; a bound below the blobs' window does
    nothing, sets status bit 8 and returns the window, and the retry with
    that window's size succeeds."""
    import pfblob
    from pfblob import workloads as wl
    from pfblob.regrid import lattice_window, remesh_device_async
    b = wl.mixed_instance(100000, config=4, instance=5)
    dev = torch.device("cuda", 0)
    x, y, g = (torch.from_numpy(a).to(dev) for a in (b.x, b.y, b.g))
    xb, yb = b.bounds()
    ref = pfblob.remesh_device(x, y, g, b.h, xb[0], yb[0], with_indices=True)
    box = (b.x.min(), b.x.max(), b.y.min(), b.y.max())
    win = lattice_window(box, b.h, xb[0], yb[0])
    out = remesh_device_async(x, y, g, b.h, xb[0], yb[0], max_base_cells=win[2] * win[3],
                              with_indices=True)
    nout, status, window, moments = out[5:]
    k = int(nout.item())
    assert int(status.item()) == 0 and k == ref[0].numel()
    assert tuple(window.cpu().tolist()) == tuple(win)
    for u, v in zip(out[:5], ref):
        assert torch.equal(u[:k], v)
    m = moments.cpu().numpy()
    m_in = oracle.moments(b.x, b.y, b.g)
    assert np.allclose(m[:4], m_in, rtol=0, atol=1e-13 * m_in[3])
    circ, imp = pfblob.conservation_error(m[:4], m[4:], float(np.abs(b.x).max()))
    assert circ <= 1e-12 and imp <= 1e-12
    small = remesh_device_async(x, y, g, b.h, xb[0], yb[0], max_base_cells=100)
    assert int(small[4].item()) == 8 and int(small[3].item()) == 0
    w = small[5].cpu().tolist()
    assert tuple(w) == tuple(win)
    again = remesh_device_async(x, y, g, b.h, xb[0], yb[0], max_base_cells=w[2] * w[3])
    assert int(again[4].item()) == 0 and int(again[3].item()) == k
    assert torch.equal(again[2][:k], ref[2])


def test_remesh_window_larger_than_the_previous_one():
    """pf_remesh sizes its scratch from the context's previous window; a set
    with a much larger window is found on the device and redone on its exact
    window, with the same result as the oracle."""
    import pfblob
    rng = np.random.default_rng(21)
    h = 0.004
    b = np.array([-1.5 * h, 1.5 * h])
    xs, ys = rng.uniform(0, 0.05, 2000), rng.uniform(0, 0.05, 2000)
    _regrid_gpu(xs, ys, rng.standard_normal(2000), h / 0.8, 0.8, b, b)
    x, y = rng.uniform(-2.0, 2.0, 3000), rng.uniform(-1.0, 1.0, 3000)
    g = rng.standard_normal(3000)
    xn, yn, gn = _regrid_gpu(x, y, g, h / 0.8, 0.8, b, b)
    rx, ry, rg, _, _ = oracle.regrid(x, y, g, h / 0.8, 0.8, b, b)
    assert np.array_equal(xn, rx) and np.array_equal(yn, ry)
    assert np.abs(gn - rg).max() <= GTOL * np.abs(rg).max()


@pytest.mark.parametrize("case", ["uniform_fmm", "sparse_direct"])
def test_velocity_and_regrid_equals_the_two_calls(case):
    """The one-upload step (velocity at the blobs, then Regrid of the same
    blobs, velocities read back while the remesh runs) gives bitwise the
    results of pfblob.velocity and pfblob.Regrid called one after the other,
    from numpy, from pinned host tensors and from device tensors, on a dense
    set with the FMM and on a sparse one (3,000 blobs over [-1, 1]^2) with the
    direct sum."""
    import pfblob
    from pfblob import workloads as wl
    if case == "uniform_fmm":
        b, meth = wl.uniform_square(n=60000, sigma=0.004, config=2, instance=13), pfblob.FMM_METHOD
    else:
        b, meth = wl.mixed_instance(3000, config=4, instance=5, sigma=0.002), pfblob.DIRECT_METHOD
    xb, yb = b.bounds()
    vx, vy = pfblob.velocity(b.x, b.y, b.g, b.sigma, method=meth, hardware=1)
    xn, yn, gn = pfblob.Regrid(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
    for inp in ((b.x, b.y, b.g), tuple(torch.from_numpy(a).pin_memory() for a in (b.x, b.y, b.g))):
        out = pfblob.velocity_and_regrid(*inp, b.sigma, b.overlap, xb, yb, method=meth)
        for u, v in zip(out, (vx, vy, xn, yn, gn)):
            assert isinstance(u, np.ndarray) and np.array_equal(u, v)
    dev = torch.device("cuda", 0)
    out = pfblob.velocity_and_regrid(*(torch.from_numpy(a).to(dev) for a in (b.x, b.y, b.g)),
                                     b.sigma, b.overlap, xb, yb, method=meth)
    for u, v in zip(out, (vx, vy, xn, yn, gn)):
        assert np.array_equal(u.cpu().numpy(), v)
