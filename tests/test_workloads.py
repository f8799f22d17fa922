"""The seeded synthetic blob configurations on the host (no GPU): sizes,
ranges and the physical facts each one is built to have."""
import numpy as np

from pfblob import workloads as wl


def test_c1_lamb_oseen_lattice():
    b = wl.lamb_oseen_lattice()
    assert b.n == 10000
    assert b.x.min() == -1.0 + 0.01 and b.x.max() == 1.0 - 0.01
    assert abs(b.sigma - 0.02 / 0.8) < 1e-15 and abs(b.h - 0.02) < 1e-15
    # the Gaussian core (rc = 0.2) lies well inside [-1,1]^2: total circulation Gamma0
    assert abs(b.g.sum() - 1.0) < 1e-9
    assert (b.g > 0).all()


def test_c2_uniform_square_is_seeded():
    a = wl.uniform_square(n=1 << 16)
    b = wl.uniform_square(n=1 << 16)
    c = wl.uniform_square(n=1 << 16, instance=1)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.g, b.g)
    assert not np.array_equal(a.x, c.x)
    assert 0.0 <= a.x.min() and a.x.max() < 1.0 and 0.0 <= a.y.min() and a.y.max() < 1.0
    assert abs(a.g.std() * a.n - 1.0) < 0.05
    assert a.ksigmasqr == 2 * 0.002 ** 2


def test_c2_full_size():
    b = wl.uniform_square()
    assert b.n == 1 << 20
    xb, yb = b.bounds()
    assert np.array_equal(xb, [-1.5 * b.h, 1.5 * b.h]) and np.array_equal(xb, yb)


def test_c3_shear_layer_annulus():
    n = 1 << 18
    b = wl.shear_layer(n=n)
    assert b.n == n
    r = np.hypot(b.x, b.y)
    assert r.min() >= 1.0 and r.max() <= 1.5
    h = np.sqrt(np.pi * (1.5 ** 2 - 1.0) / n)
    assert abs(b.sigma * b.overlap - h) < 1e-15
    # vorticity -(2/delta) exp(-(r-1)/delta): all negative, strongest at the wall
    assert (b.g < 0).all()
    assert b.g[np.argmin(r)] < b.g[np.argmax(r)]
    # no two blobs on one lattice point
    assert np.unique(np.stack([b.x, b.y]), axis=1).shape[1] == n


def test_c3_cylinder_panels_close_on_the_circle():
    p = wl.cylinder_panels()
    assert p.m == 512
    assert np.allclose(p.xe[:-1], p.xs[1:]) and np.allclose(p.ye[:-1], p.ys[1:])
    assert np.allclose([p.xe[-1], p.ye[-1]], [p.xs[0], p.ys[0]])
    assert np.allclose(p.cosa ** 2 + p.sina ** 2, 1.0)
    mid = np.hypot(0.5 * (p.xs + p.xe), 0.5 * (p.ys + p.ye))
    assert np.allclose(mid, 1.0, atol=1e-12)


def test_c4_sizes_and_instances():
    sizes = wl.log_uniform_sizes(256, 2048, 262144, config=4)
    assert sizes.shape == (256,) and sizes.min() >= 2048 and sizes.max() <= 262144
    expected_mean = (262144 - 2048) / np.log(262144 / 2048)  # log-uniform mean, ~53.6k
    assert abs(sizes.mean() / expected_mean - 1.0) < 0.25
    for i in range(8):
        b = wl.mixed_instance(1000, config=4, instance=i)
        assert 0.002 <= b.sigma <= 0.01
        assert np.abs(b.x).max() <= 1.0 and np.abs(b.y).max() <= 1.0
