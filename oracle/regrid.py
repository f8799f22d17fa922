"""M4' remesh (``Regrid``) restated with numpy + scipy.sparse (test infrastructure).

Follows ``src/python/blobs/base/regrid/_regridding.py:107-222`` step by step:

1. ``h = sigma*overlap`` (:118).
2. window-left indices ``xL = int64(ceil((x - xB0 - 2h + 0.5h)/h)) - 1`` (:157-158).
3. 16 window cells per blob, x offset fastest (:170-172).
4. weight ``M4'(xK + 0.5 + xB0/h - x/h) * M4'(yK + 0.5 + yB0/h - y/h) * g``
   (:183-184, kernel from ``_interpolation_kernels_1d.cpp:75-89``).
5. duplicate cells summed by building a CSR matrix and reading it back as COO
   (:200-202); this keeps cells whose sum is exactly zero and orders the
   output by (ix, iy).
6. cell coordinates back: ``x = ix*h + 0.5h + xB0`` (:217-218).

The kernel-size half is the integer 2 (the reference is Python 2, where
``kernelSize/2`` is integer division).

``population_control`` restates PopulationControl (same module, :316-330);
``diffusion_tutty`` restates the Tutty redistribution of
``src/python/blobs/base/evolution/_evolution.py:334-443``.
"""
import numpy as np
import scipy.sparse

from .core import m4prime, remesh_left_index

KERNEL_SIZE = 4


def window(x, y, g, h, xb0, yb0, c=0.0):
    """Per-blob window indices and weights: (ix (16,N), iy (16,N), w (16,N))."""
    n = x.shape[0]
    xl = remesh_left_index(x, xb0, h)
    yl = remesh_left_index(y, yb0, h)
    k = KERNEL_SIZE
    ix = np.tile(xl, (k * k, 1)) + np.tile(np.arange(k), k).reshape(k * k, 1)
    iy = np.tile(yl, (k * k, 1)) + np.repeat(np.arange(k), k).reshape(k * k, 1)
    ux = ix + 0.5 + xb0 / h - x / h
    uy = iy + 0.5 + yb0 / h - y / h
    w = m4prime(ux, c) * m4prime(uy, c)
    w *= np.tile(g, (k * k, 1))
    assert ix.shape == (k * k, n)
    return ix, iy, w


def regrid(x, y, g, sigma, overlap, xbounds, ybounds, c=0.0):
    """Remesh blobs onto the lattice of spacing ``h = sigma*overlap``.

    Returns (x_new, y_new, g_new, ix, iy): the new blobs in (ix, iy) order and
    their integer lattice indices.
    """
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    if x.size < 1:
        e = np.zeros(0, dtype=np.int64)
        return x, y, g, e, e
    h = sigma * overlap
    xb0, yb0 = float(xbounds[0]), float(ybounds[0])
    ix, iy, w = window(x, y, g, h, xb0, yb0, c)
    half = KERNEL_SIZE // 2
    ixmin = ix.min()
    iymin = iy.min()
    mat = scipy.sparse.csr_matrix((w.flatten(), (ix.flatten() - ixmin + half,
                                                 iy.flatten() - iymin + half))).tocoo()
    gn, ii, jj = mat.data, mat.row.astype(np.int64), mat.col.astype(np.int64)
    ixn = ii + ixmin - half
    iyn = jj + iymin - half
    xn = ixn * h + 0.5 * h + xb0
    yn = iyn * h + 0.5 * h + yb0
    return xn, yn, gn, ixn, iyn


def population_control(x, y, g, thr_local, thr_global):
    """Drop blobs with |g| < thr, thr divided by 10 while the dropped
    circulation sum(|g|) is not below thr_global (``_regridding.py:316-330``).
    Returns (x, y, g, thr) of the kept blobs in input order."""
    a = np.abs(np.asarray(g, dtype=np.float64))
    thr = float(thr_local)
    if not (np.isfinite(thr) and np.isfinite(thr_global) and thr_global > 0.0):
        raise ValueError("thresholds must be finite and thr_global > 0")
    while True:
        flagged = a < thr
        if a[flagged].sum() < thr_global:
            break
        thr /= 10.0
    keep = ~flagged
    return x[keep], y[keep], g[keep], thr


def diffusion_tutty(x, y, g, dt, nu, sigma, overlap, xbounds, ybounds):
    """Tutty diffusive redistribution (``_evolution.py:334-443``): same window
    and duplicate summation as ``regrid``, weights from the reference node
    i = xL + 1.  Returns (x_new, y_new, g_new, ix, iy)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    if x.size < 1:
        e = np.zeros(0, dtype=np.int64)
        return x, y, g, e, e
    h = sigma * overlap
    xb0, yb0 = float(xbounds[0]), float(ybounds[0])
    k = KERNEL_SIZE
    xl = remesh_left_index(x, xb0, h)
    yl = remesh_left_index(y, yb0, h)
    ix = np.tile(xl, (k * k, 1)) + np.tile(np.arange(k), k).reshape(k * k, 1)
    iy = np.tile(yl, (k * k, 1)) + np.repeat(np.arange(k), k).reshape(k * k, 1)
    hnu = np.sqrt(dt * nu)
    q = 1.0 - 2.0 * (hnu / h) ** 2.0

    def weights(v, il, b0):
        vi = (il + 1) * h + 0.5 * h + b0
        d = (v - vi) / h
        d1 = d - 1.0
        f = q - d * d
        gg = q - d1 * d1
        return ((1.0 - d) * (0.5 * (1.0 - f - d)),
                (1.0 - d) * f + d * (0.5 * (1.0 - gg - d1)),
                (1.0 - d) * (0.5 * (1.0 - f + d)) + d * gg,
                d * (0.5 * (1.0 - gg + d1)))

    fx = weights(x, xl, xb0)
    gy = weights(y, yl, yb0)
    fw = np.tile(np.vstack(fx), (k, 1)).flatten()
    gw = np.vstack([np.tile(w, (k, 1)) for w in gy]).flatten()
    w = fw * gw
    w *= np.tile(g, (k * k, 1)).flatten()
    half = k // 2
    ixmin, iymin = ix.min(), iy.min()
    mat = scipy.sparse.csr_matrix((w, (ix.flatten() - ixmin + half,
                                       iy.flatten() - iymin + half))).tocoo()
    gn, ii, jj = mat.data, mat.row.astype(np.int64), mat.col.astype(np.int64)
    ixn = ii + ixmin - half
    iyn = jj + iymin - half
    return ixn * h + 0.5 * h + xb0, iyn * h + 0.5 * h + yb0, gn, ixn, iyn
