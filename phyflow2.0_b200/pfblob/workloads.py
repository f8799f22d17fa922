"""Seeded synthetic blob configurations.

The reference ships no datasets; these generators stand in for the blob
distributions its examples build (Lamb-Oseen lattice of
``src/examples/blobs/ex03_evaluate_velocity_test/ex03_evaluate_velocity_test.py``,
the cylinder panel recipe of
``src/examples/panels/ex02_evaluateVelocity_test/ex02_evaluateVelocity_test.py:27-40``)
at the sizes of the five benchmark configurations:

* ``lamb_oseen_lattice``  - C1: Lamb-Oseen vortex (Gamma0=1, core 0.2) on the
  100x100 cell-centred lattice of [-1,1]^2, h=0.02, sigma=h/0.8.
* ``uniform_square``      - C2: N blobs U[0,1)^2, g ~ N(0,1)/N, sigma=0.002.
* ``shear_layer``         - C3: near-wall layer in 1<=r<=1.5 with
  omega = -(2/delta) exp(-(r-1)/delta), delta=0.02, jittered lattice,
  exactly N blobs, plus straight vortex panels on the unit circle.
* ``mixed_instance``      - C4/C5 instances: uniform positions in [-1,1]^2
  carrying a Lamb-Oseen circulation plus N(0,1)/N noise, sigma ~ U[0.002,0.01].

Seeds: numpy PCG64, seed = 20261203 + 1000*config + instance.
"""
from dataclasses import dataclass

import numpy as np

SEED0 = 20261203


def rng_for(config, instance=0):
    return np.random.Generator(np.random.PCG64(SEED0 + 1000 * config + instance))


@dataclass
class BlobSet:
    x: np.ndarray
    y: np.ndarray
    g: np.ndarray
    sigma: float
    overlap: float = 0.8
    k: float = 2.0

    @property
    def n(self):
        return self.x.shape[0]

    @property
    def h(self):
        return self.sigma * self.overlap

    @property
    def ksigmasqr(self):
        return self.k * self.sigma * self.sigma

    def bounds(self):
        """Remesh lattice bounds used by ``Blobs.redistribute``
        (``src/python/blobs/__blobsClass.py:891-892``): [-1.5h, 1.5h]."""
        h = self.h
        return np.array([-1.5 * h, 1.5 * h]), np.array([-1.5 * h, 1.5 * h])


def lamb_oseen_omega(x, y, gamma0=1.0, rc=0.2):
    r2 = x * x + y * y
    return gamma0 / (np.pi * rc * rc) * np.exp(-r2 / (rc * rc))


def lamb_oseen_lattice(h=0.02, n_side=100, gamma0=1.0, rc=0.2, overlap=0.8):
    """C1: cell-centred lattice x_i = -1 + (i + 1/2) h, i = 0..n_side-1."""
    c = -1.0 + (np.arange(n_side) + 0.5) * h
    X, Y = np.meshgrid(c, c, indexing="ij")
    x = X.ravel().copy()
    y = Y.ravel().copy()
    g = lamb_oseen_omega(x, y, gamma0, rc) * h * h
    return BlobSet(x, y, g, sigma=h / overlap, overlap=overlap)


def uniform_square(n=1 << 20, sigma=0.002, overlap=0.8, config=2, instance=0):
    """C2: x, y ~ U[0,1)^2, g ~ N(0,1)/N."""
    rng = rng_for(config, instance)
    x = rng.random(n)
    y = rng.random(n)
    g = rng.standard_normal(n) / n
    return BlobSet(x, y, g, sigma=sigma, overlap=overlap)


def shear_layer(n=1 << 22, delta=0.02, r0=1.0, r1=1.5, overlap=0.8, config=3, instance=0):
    """C3 blobs: annulus r0<=r<=r1, exactly n blobs on a jittered lattice.

    The lattice spacing is h = sqrt(area/n); lattice points inside the annulus
    are jittered by U(-h/4, h/4) and then n of them are drawn without
    replacement (a slightly finer lattice guarantees at least n candidates).
    """
    rng = rng_for(config, instance)
    area = np.pi * (r1 * r1 - r0 * r0)
    h = np.sqrt(area / n)
    hl = h * 0.995
    m = int(np.ceil(r1 / hl)) + 1
    c = (np.arange(-m, m + 1)) * hl
    X, Y = np.meshgrid(c, c, indexing="ij")
    X = X.ravel()
    Y = Y.ravel()
    X = X + rng.uniform(-h / 4, h / 4, X.shape[0])
    Y = Y + rng.uniform(-h / 4, h / 4, Y.shape[0])
    R = np.sqrt(X * X + Y * Y)
    keep = np.nonzero((R >= r0) & (R <= r1))[0]
    if keep.shape[0] < n:
        raise RuntimeError("shear_layer: lattice too coarse")
    sel = np.sort(rng.choice(keep, size=n, replace=False))
    x = X[sel].copy()
    y = Y[sel].copy()
    r = R[sel]
    omega = -(2.0 / delta) * np.exp(-(r - r0) / delta)
    g = omega * h * h
    return BlobSet(x, y, g, sigma=h / overlap, overlap=overlap)


@dataclass
class PanelSet:
    gamma: np.ndarray
    xs: np.ndarray
    ys: np.ndarray
    xe: np.ndarray
    ye: np.ndarray
    cosa: np.ndarray
    sina: np.ndarray

    @property
    def m(self):
        return self.gamma.shape[0]


def cylinder_panels(n_panel=512, radius=1.0, config=3, instance=0, strengths=None):
    """Straight panels on a circle; geometry as in the reference panel example
    (end points at polar angles linspace(pi, -pi, n+1) - dtheta/2 on a radius
    enlarged by 1/cos(dtheta/2)); cos/sin alpha from the panel direction as
    ``Panels.__updateCoordinates`` computes them
    (``src/python/panels/__panelsClass.py:1037-1041``)."""
    theta = np.linspace(np.pi, -np.pi, n_panel + 1)
    dtheta = theta[1] - theta[0]
    r = (radius + np.spacing(100)) / np.cos(dtheta / 2.0)
    xp = r * np.cos(theta - dtheta / 2)
    yp = r * np.sin(theta - dtheta / 2)
    xs, ys, xe, ye = xp[:-1].copy(), yp[:-1].copy(), xp[1:].copy(), yp[1:].copy()
    lx, ly = xe - xs, ye - ys
    L = np.sqrt(lx * lx + ly * ly)
    if strengths is None:
        strengths = rng_for(config, 500 + instance).standard_normal(n_panel)
    return PanelSet(np.asarray(strengths, dtype=np.float64), xs, ys, xe, ye, lx / L, ly / L)


def log_uniform_sizes(count, lo, hi, config, instance=0):
    rng = rng_for(config, 900 + instance)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def mixed_instance(n, config=4, instance=0, sigma=None):
    """C4/C5 instance: positions U[-1,1]^2; g = Lamb-Oseen omega * (4/n) plus
    N(0,1)/n noise; sigma ~ U[0.002, 0.01] unless given."""
    rng = rng_for(config, instance)
    x = rng.uniform(-1.0, 1.0, n)
    y = rng.uniform(-1.0, 1.0, n)
    g = lamb_oseen_omega(x, y) * (4.0 / n) + rng.standard_normal(n) / n
    if sigma is None:
        sigma = float(rng.uniform(0.002, 0.01))
    return BlobSet(x, y, g, sigma=sigma, overlap=0.8)
