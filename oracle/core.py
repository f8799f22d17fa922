"""ctypes bindings to ``liboracle.so`` (our C restatement; test infrastructure).

Each wrapper names the reference function it restates; the C file cites the
reference lines.  All arrays are float64, C-contiguous.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int64)


def _build():
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)


def oracle_lib():
    """Load (building on first use if needed) the C oracle library."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path) or (
                os.path.getmtime(path) < os.path.getmtime(os.path.join(_HERE, "pf_oracle.c"))):
            _build()
        lib = ctypes.CDLL(path)
        i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
        lib.or_velocity_direct_gauss.argtypes = [i64, _dp, _dp, _dp, i64, _dp, _dp, dbl, _dp, _dp, cint]
        lib.or_vorticity_direct_gauss.argtypes = [i64, _dp, _dp, _dp, i64, _dp, _dp, dbl, _dp,
                                                  cint]
        lib.or_velocity_direct_cutoff.argtypes = [i64, _dp, _dp, _dp, i64, _dp, _dp, dbl, _dp,
                                                  _dp, cint]
        lib.or_vorticity_direct_cutoff.argtypes = [i64, _dp, _dp, _dp, i64, _dp, _dp, dbl, _dp,
                                                   cint]
        lib.or_panel_velocity.argtypes = [i64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, i64, _dp, _dp, _dp, _dp, cint]
        lib.or_source_panel_velocity.argtypes = lib.or_panel_velocity.argtypes
        lib.or_m4prime.argtypes = [i64, _dp, dbl, _dp]
        lib.or_remesh_left_index.argtypes = [i64, _dp, dbl, dbl, _ip]
        lib.or_moments.argtypes = [i64, _dp, _dp, _dp, _dp]
        for f in (lib.or_velocity_direct_gauss, lib.or_vorticity_direct_gauss,
                  lib.or_velocity_direct_cutoff, lib.or_vorticity_direct_cutoff,
                  lib.or_panel_velocity, lib.or_source_panel_velocity, lib.or_m4prime,
                  lib.or_remesh_left_index, lib.or_moments):
            f.restype = None
        _LIB = lib
    return _LIB


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_dp)


def velocity_direct(xs, ys, gs, ksigmasqr, xt=None, yt=None, nthreads=0):
    """FP64 direct Gauss velocity; restates ``vv2parGauss_C_cpu`` (targets
    default to the blobs, as ``_velocity_direct_cpu_gauss`` does)."""
    xs, ys, gs = _f64(xs), _f64(ys), _f64(gs)
    xt = xs if xt is None else _f64(xt)
    yt = ys if yt is None else _f64(yt)
    vx = np.empty(xt.shape[0])
    vy = np.empty(xt.shape[0])
    oracle_lib().or_velocity_direct_gauss(xs.shape[0], _p(xs), _p(ys), _p(gs), xt.shape[0],
                                          _p(xt), _p(yt), float(ksigmasqr), _p(vx), _p(vy),
                                          int(nthreads))
    return vx, vy


def vorticity_direct(xs, ys, gs, ksigmasqr, xt=None, yt=None, nthreads=0):
    """FP64 induced vorticity of Gaussian blobs; restates ``ww2parGauss_C_cpu``
    (targets default to the blobs, as ``_vorticity_direct_cpu_gauss``)."""
    xs, ys, gs = _f64(xs), _f64(ys), _f64(gs)
    xt = xs if xt is None else _f64(xt)
    yt = ys if yt is None else _f64(yt)
    w = np.empty(xt.shape[0])
    oracle_lib().or_vorticity_direct_gauss(xs.shape[0], _p(xs), _p(ys), _p(gs), xt.shape[0],
                                           _p(xt), _p(yt), float(ksigmasqr), _p(w), int(nthreads))
    return w


def velocity_direct_cutoff(xs, ys, gs, sigmasqr, xt=None, yt=None, nthreads=0):
    """FP64 cutoff-kernel velocity; restates ``vv2par_C_cpu`` (sigmasqr =
    sigma^2, as ``_velocity_direct_cpu_cutoff`` passes it)."""
    xs, ys, gs = _f64(xs), _f64(ys), _f64(gs)
    xt = xs if xt is None else _f64(xt)
    yt = ys if yt is None else _f64(yt)
    vx = np.empty(xt.shape[0])
    vy = np.empty(xt.shape[0])
    oracle_lib().or_velocity_direct_cutoff(xs.shape[0], _p(xs), _p(ys), _p(gs), xt.shape[0],
                                           _p(xt), _p(yt), float(sigmasqr), _p(vx), _p(vy),
                                           int(nthreads))
    return vx, vy


def vorticity_direct_cutoff(xs, ys, gs, sigmasqr, xt=None, yt=None, nthreads=0):
    """FP64 cutoff-kernel induced vorticity; restates ``ww2par_C_cpu``."""
    xs, ys, gs = _f64(xs), _f64(ys), _f64(gs)
    xt = xs if xt is None else _f64(xt)
    yt = ys if yt is None else _f64(yt)
    w = np.empty(xt.shape[0])
    oracle_lib().or_vorticity_direct_cutoff(xs.shape[0], _p(xs), _p(ys), _p(gs), xt.shape[0],
                                            _p(xt), _p(yt), float(sigmasqr), _p(w), int(nthreads))
    return w


def source_panel_velocity(sigma, xs, ys, xe, ye, cosa, sina, xv, yv, nthreads=0):
    """FP64 source-panel velocity; restates ``_sourcePanel_Cython_cpu.inducedVelocity``."""
    arrs = [_f64(a) for a in (sigma, xs, ys, xe, ye, cosa, sina)]
    xv, yv = _f64(xv), _f64(yv)
    vx = np.empty(xv.shape[0])
    vy = np.empty(xv.shape[0])
    oracle_lib().or_source_panel_velocity(arrs[0].shape[0], *[_p(a) for a in arrs], xv.shape[0],
                                          _p(xv), _p(yv), _p(vx), _p(vy), int(nthreads))
    return vx, vy


def panel_velocity(gamma, xs, ys, xe, ye, cosa, sina, xv, yv, nthreads=0):
    """FP64 vortex-panel velocity; restates ``_vortexPanel_Cython_cpu.inducedVelocity``."""
    arrs = [_f64(a) for a in (gamma, xs, ys, xe, ye, cosa, sina)]
    xv, yv = _f64(xv), _f64(yv)
    vx = np.empty(xv.shape[0])
    vy = np.empty(xv.shape[0])
    oracle_lib().or_panel_velocity(arrs[0].shape[0], *[_p(a) for a in arrs], xv.shape[0],
                                   _p(xv), _p(yv), _p(vx), _p(vy), int(nthreads))
    return vx, vy


def m4prime(x, c=0.0):
    """M4' weights; restates ``m4kernel_1d`` (returns x's shape)."""
    xa = _f64(x)
    flat = xa.reshape(-1)
    w = np.empty_like(flat)
    oracle_lib().or_m4prime(flat.shape[0], _p(flat), float(c), _p(w))
    return w.reshape(xa.shape)


def remesh_left_index(x, b0, h):
    """int64 left index of the 4x4 remesh window (``_regridding.py:157``)."""
    xa = _f64(x)
    out = np.empty(xa.shape[0], dtype=np.int64)
    oracle_lib().or_remesh_left_index(xa.shape[0], _p(xa), float(b0), float(h),
                                      out.ctypes.data_as(_ip))
    return out


def moments(x, y, g):
    """(sum g, sum g*x, sum g*y, sum |g|) in FP64."""
    x, y, g = _f64(x), _f64(y), _f64(g)
    out = np.empty(4)
    oracle_lib().or_moments(x.shape[0], _p(x), _p(y), _p(g), _p(out))
    return out
