"""Pin the CPU oracle against outputs of the reference's own code (fixtures in
tests/golden/, made by tests/golden/make_golden.py from the compiled reference
Cython kernels, the reference Regrid and the reference C++ FMM)."""
import numpy as np
import pytest

import oracle
from conftest import normwise_err


def test_direct_c1_bit_exact(golden):
    d = golden("direct_c1")
    vx, vy = oracle.velocity_direct(d["x"], d["y"], d["g"], float(d["ksigmasqr"]))
    assert np.array_equal(vx, d["vx"]) and np.array_equal(vy, d["vy"])


def test_direct_edge_cases_bit_exact(golden):
    d = golden("direct_rand")
    vx, vy = oracle.velocity_direct(d["x"], d["y"], d["g"], float(d["ksigmasqr"]))
    assert np.array_equal(vx, d["vx"]) and np.array_equal(vy, d["vy"])


def test_direct_separate_targets_match_self_targets(golden):
    d = golden("direct_rand")
    vx, vy = oracle.velocity_direct(d["x"], d["y"], d["g"], float(d["ksigmasqr"]),
                                    d["x"][:100].copy(), d["y"][:100].copy())
    assert np.array_equal(vx, d["vx"][:100])


def test_panel_bit_exact(golden):
    p = golden("panel_cyl")
    vx, vy = oracle.panel_velocity(p["gamma"], p["xs"], p["ys"], p["xe"], p["ye"], p["cosa"],
                                   p["sina"], p["xv"], p["yv"])
    assert np.array_equal(vx, p["vx"]) and np.array_equal(vy, p["vy"])


def test_regrid_matches_reference_regrid(golden):
    for name in ("regrid_c1", "regrid_rand_c0", "regrid_rand_c3", "regrid_far"):
        r = golden(name)
        xn, yn, gn, ix, iy = oracle.regrid(r["x"], r["y"], r["g"], float(r["sigma"]),
                                           float(r["overlap"]), r["xb"], r["yb"], float(r["c"]))
        assert np.array_equal(xn, r["xn"]) and np.array_equal(yn, r["yn"]), name
        assert np.array_equal(gn, r["gn"]), name


def test_regrid_conserves_moments(golden):
    r = golden("regrid_c1")
    m0 = oracle.moments(r["x"], r["y"], r["g"])
    m1 = oracle.moments(r["xn"], r["yn"], r["gn"])
    assert abs(m1[0] - m0[0]) / m0[3] < 1e-13
    xs = np.abs(r["x"]).max()
    assert max(abs(m1[1] - m0[1]), abs(m1[2] - m0[2])) / (m0[3] * xs) < 1e-13


def test_m4prime_branches():
    x = np.array([0.0, 0.5, -0.5, 1.0, -1.0, 1.5, 2.0, -2.5])
    w = oracle.m4prime(x, 0.0)
    assert w[0] == 1.0
    assert w[3] == 0.0 and w[4] == 0.0  # |x| == 1 falls through to 0
    assert w[6] == 0.0 and w[7] == 0.0
    assert np.isclose(w[1], 1 - 2.5 * 0.25 + 1.5 * 0.125)
    assert np.isclose(w[5], 0.5 * 0.25 * (-0.5))
    # partition of unity on a shifted window (c = 0)
    for s in (0.1, 0.37, 0.73):
        u = np.array([1.0, 0.0, -1.0, -2.0]) + s
        assert abs(oracle.m4prime(u, 0.0).sum() - 1.0) < 1e-15


def test_m4prime_matches_reference_loop(golden):
    """The oracle's M4' equals, bit for bit, the reference's own m4kernel_1d
    loop (_interpolation_kernels_1d.cpp:74-89, compiled from its source lines)
    on the branch boundaries, just inside and outside them, and a dense sweep,
    for four Wee coefficients."""
    r = golden("m4_ref")
    for k, c in enumerate(r["c"]):
        assert np.array_equal(oracle.m4prime(r["x"], float(c)), r["w"][k]), float(c)


def test_m4prime_matches_compiled_reference_when_present():
    """Same check against the compiled loop itself on fresh random points
    (where oracle/_ref holds it)."""
    from oracle import ref
    if not ref.m4_available():
        pytest.skip("oracle/_ref/libref_m4.so not built here")
    x = np.random.default_rng(9).uniform(-2.5, 2.5, 100000)
    for c in (0.0, 0.25, 1.3):
        assert np.array_equal(oracle.m4prime(x, c), ref.m4kernel_1d(x, c))


def test_reference_fmm_within_tolerance_of_direct_oracle(golden):
    f = golden("fmm_rand")
    sig = float(f["sigma"])
    vx, vy = oracle.velocity_direct(f["x"], f["y"], f["g"], 2.0 * sig * sig)
    assert normwise_err(f["vx"], f["vy"], vx, vy) < 1e-6


def test_population_control_matches_reference(golden):
    for name, k in (("popctl_c1", 3), ("popctl_decades", 6), ("popctl_deep", 32)):
        d = golden(name)
        tl, tg = float(d["thr_local"]), float(d["thr_global"])
        xo, yo, go, thr = oracle.population_control(d["x"], d["y"], d["g"], tl, tg)
        assert np.array_equal(xo, d["xo"]) and np.array_equal(yo, d["yo"]), name
        assert np.array_equal(go, d["go"]), name
        # the threshold went down k decades (each division rounded)
        t = tl
        for _ in range(k):
            t /= 10.0
        assert thr == t, name


def test_tutty_matches_reference(golden):
    for name in ("tutty_rand", "tutty_rand_nu0", "tutty_c1"):
        d = golden(name)
        xn, yn, gn, _, _ = oracle.diffusion_tutty(d["x"], d["y"], d["g"], float(d["dt"]),
                                                  float(d["nu"]), float(d["sigma"]),
                                                  float(d["overlap"]), d["xb"], d["yb"])
        assert np.array_equal(xn, d["xn"]) and np.array_equal(yn, d["yn"]), name
        assert np.array_equal(gn, d["gn"]), name


def test_vorticity_matches_reference_loop(golden):
    d = golden("vort_c1")
    w = oracle.vorticity_direct(d["x"], d["y"], d["g"], float(d["ksigmasqr"]))
    assert np.array_equal(w, d["w"])
    d = golden("vort_rand")
    w = oracle.vorticity_direct(d["x"], d["y"], d["g"], float(d["ksigmasqr"]), d["xt"], d["yt"])
    assert np.array_equal(w, d["w"])


def test_cutoff_kernels_match_reference_loops(golden):
    """The cutoff-kernel restatements are bit-exact against the reference's
    own vv2par_C_cpu / ww2par_C_cpu loops (golden, at the blobs and at
    separate points with a duplicated, a zero and a far blob)."""
    d = golden("cutoff_c1")
    s2 = float(d["sigmasqr"])
    vx, vy = oracle.velocity_direct_cutoff(d["x"], d["y"], d["g"], s2)
    assert np.array_equal(vx, d["vx"]) and np.array_equal(vy, d["vy"])
    assert np.array_equal(oracle.vorticity_direct_cutoff(d["x"], d["y"], d["g"], s2), d["w"])
    d = golden("cutoff_rand")
    s2 = float(d["sigmasqr"])
    vx, vy = oracle.velocity_direct_cutoff(d["x"], d["y"], d["g"], s2, d["xt"], d["yt"])
    assert np.array_equal(vx, d["vx"]) and np.array_equal(vy, d["vy"])
    w = oracle.vorticity_direct_cutoff(d["x"], d["y"], d["g"], s2, d["xt"], d["yt"])
    assert np.array_equal(w, d["w"])


def test_source_panel_matches_reference_cython(golden):
    """The constant-source panel restatement is bit-exact against the
    reference's Cython kernel (_sourcePanel_Cython_cpu.inducedVelocity)."""
    d = golden("source_panel")
    vx, vy = oracle.source_panel_velocity(d["sigma"], d["xs"], d["ys"], d["xe"], d["ye"],
                                          d["cosa"], d["sina"], d["xv"], d["yv"])
    assert np.array_equal(vx, d["vx"]) and np.array_equal(vy, d["vy"])
