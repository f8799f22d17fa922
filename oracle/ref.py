"""Loaders for the reference's own CPU code compiled into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY.  ``make -C oracle ref`` compiles, in place from the
pHyFlow sources, the Cython direct Gauss kernel
(``src/cpp/blobs/cython/vv2parGauss_Cython/vv2parGauss_Cython_cpu.pyx``), the
Cython vortex-panel kernel
(``src/cpp/panels/cython/vortexPanel_Cython/_vortexPanel_Cython_cpu.pyx``) and
the C++ CPU FMM (``src/cpp/blobs/c++/fmm2d_py_cpu_gpu/*.cpp`` behind
``oracle/ref_fmm_driver.cpp``) and the induced-vorticity loop of
``src/cpp/blobs/c/ww2parGauss_C/ww2parGauss_C_cpu.c`` (behind
``oracle/ref_ww2_driver.c``), and the M4' weight loop of
``src/cpp/blobs/c++/interpolation_kernels_1d/_interpolation_kernels_1d.cpp``
(behind ``oracle/ref_m4_driver.cpp``).  The built files travel with the
repository snapshot; the sources they were built from do not.
"""
import ctypes
import importlib.util
import os
import sysconfig

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_SUF = sysconfig.get_config_var("EXT_SUFFIX")
_cache = {}

# constant of the Oseen smoother in the reference FMM binding
# (src/python/blobs/base/induced/_induced.py:239)
FMM_ALPHA = 1.2564312086261696770


def available():
    return all(os.path.exists(p) for p in (
        os.path.join(REF_DIR, "vv2parGauss_Cython_cpu" + _SUF),
        os.path.join(REF_DIR, "_vortexPanel_Cython_cpu" + _SUF),
        os.path.join(REF_DIR, "libreffmm.so")))


def _module(name):
    if name not in _cache:
        path = os.path.join(REF_DIR, name + _SUF)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference exists")
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _cache[name] = mod
    return _cache[name]


def direct_gauss(x, y, g, ksigmasqr):
    """Reference Cython direct sum at the blobs themselves -> (vx, vy)."""
    blobs = np.ascontiguousarray(np.stack([x, y, g], axis=1), dtype=np.float64)
    v = _module("vv2parGauss_Cython_cpu").vv2parGauss_Cython_cpu(blobs, float(ksigmasqr))
    return np.array(v[:, 0]), np.array(v[:, 1])


def panel_velocity(gamma, xs, ys, xe, ye, cosa, sina, xv, yv):
    """Reference Cython vortex-panel induced velocity -> (vx, vy)."""
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in (gamma, xv, yv, xs, ys, xe, ye, cosa, sina)]
    vx, vy = _module("_vortexPanel_Cython_cpu").inducedVelocity(*f)
    return np.array(vx), np.array(vy)


def _fmm_lib():
    if "fmm" not in _cache:
        path = os.path.join(REF_DIR, "libreffmm.so")
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_fmm2d.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, dp, dp, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
        lib.ref_fmm2d.restype = None
        _cache["fmm"] = lib
    return _cache["fmm"]


def fmm_velocity(x, y, g, sigma, k=2.0, xt=None, yt=None, ndirect=35, tol=1e-6, cutoff=None):
    """Reference CPU FMM, mapped to velocities as the reference Python layer
    does (``_induced.py:236-251``): vx = -qi/(2 pi), vy = -qr/(2 pi)."""
    x, y, g = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, g))
    xt = x if xt is None else np.ascontiguousarray(xt, dtype=np.float64)
    yt = y if yt is None else np.ascontiguousarray(yt, dtype=np.float64)
    xopt = np.sqrt(FMM_ALPHA * k * sigma * sigma)
    if cutoff is None:
        cutoff = 5.0 * xopt
    qr = np.zeros(xt.shape[0])
    qi = np.zeros(xt.shape[0])
    dp = ctypes.POINTER(ctypes.c_double)
    p = lambda a: a.ctypes.data_as(dp)
    _fmm_lib().ref_fmm2d(x.shape[0], p(x), p(y), p(g), xt.shape[0], p(xt), p(yt), int(ndirect),
                         float(xopt), float(cutoff), float(tol), p(qr), p(qi))
    return -qi / (2.0 * np.pi), -qr / (2.0 * np.pi)


def vorticity_gauss(x, y, g, ksigmasqr, xt=None, yt=None):
    """The reference's own ww2parGauss_C_cpu loop -> w at (xt, yt) (default:
    the blobs)."""
    if "ww2" not in _cache:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libref_ww2.so"))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_ww2par_gauss.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, dp, dp,
                                         ctypes.c_double, dp]
        lib.ref_ww2par_gauss.restype = None
        _cache["ww2"] = lib
    x, y, g = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, g))
    xt = x if xt is None else np.ascontiguousarray(xt, dtype=np.float64)
    yt = y if yt is None else np.ascontiguousarray(yt, dtype=np.float64)
    w = np.empty(xt.shape[0])
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    _cache["ww2"].ref_ww2par_gauss(x.shape[0], p(x), p(y), p(g), xt.shape[0], p(xt), p(yt),
                                   float(ksigmasqr), p(w))
    return w


def panel_influence(xcp, ycp, xs, ys, xe, ye, cosa, sina):
    """Reference Cython assemble_influenceMatrix -> A (M, M)."""
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in (xcp, ycp, xs, ys, xe, ye, cosa, sina)]
    return np.array(_module("_vortexPanel_Cython_cpu").assemble_influenceMatrix(*f))


def source_panel_available():
    return os.path.exists(os.path.join(REF_DIR, "_sourcePanel_Cython_cpu" + _SUF))


def source_panel_velocity(sigma, xs, ys, xe, ye, cosa, sina, xv, yv):
    """Reference Cython source-panel induced velocity -> (vx, vy)."""
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in (sigma, xv, yv, xs, ys, xe, ye, cosa, sina)]
    vx, vy = _module("_sourcePanel_Cython_cpu").inducedVelocity(*f)
    return np.array(vx), np.array(vy)


def source_panel_influence(xcp, ycp, xs, ys, xe, ye, cosa, sina):
    """Reference Cython source-panel assemble_influenceMatrix -> A (M, M)."""
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in (xcp, ycp, xs, ys, xe, ye, cosa, sina)]
    return np.array(_module("_sourcePanel_Cython_cpu").assemble_influenceMatrix(*f))


def m4_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_m4.so"))


def m4kernel_1d(x, c):
    """The reference's own m4kernel_1d loop (_interpolation_kernels_1d.cpp:
    74-89) -> the M4' weights of the points x (flattened), Wee coefficient c."""
    if "m4" not in _cache:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libref_m4.so"))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_m4kernel_1d.argtypes = [ctypes.c_size_t, dp, ctypes.c_double, dp]
        lib.ref_m4kernel_1d.restype = None
        _cache["m4"] = lib
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
    w = np.empty_like(x)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    _cache["m4"].ref_m4kernel_1d(x.shape[0], p(x), float(c), p(w))
    return w


def cutoff_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_cutoff.so"))


def _cutoff_lib():
    if "cutoff" not in _cache:
        lib = ctypes.CDLL(os.path.join(REF_DIR, "libref_cutoff.so"))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_vv2par_cutoff.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, dp, dp,
                                          ctypes.c_double, dp, dp]
        lib.ref_ww2par_cutoff.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, dp, dp,
                                          ctypes.c_double, dp]
        lib.ref_vv2par_cutoff.restype = None
        lib.ref_ww2par_cutoff.restype = None
        _cache["cutoff"] = lib
    return _cache["cutoff"]


def _targets(x, y, g, xt, yt):
    x, y, g = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, g))
    xt = x if xt is None else np.ascontiguousarray(xt, dtype=np.float64)
    yt = y if yt is None else np.ascontiguousarray(yt, dtype=np.float64)
    return x, y, g, xt, yt


def velocity_cutoff(x, y, g, sigmasqr, xt=None, yt=None):
    """The reference's own cutoff-kernel velocity loop (vv2par_C_cpu.c:133-151)
    -> (vx, vy) at the targets (the blobs if None)."""
    x, y, g, xt, yt = _targets(x, y, g, xt, yt)
    vx, vy = np.empty(xt.shape[0]), np.empty(xt.shape[0])
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    _cutoff_lib().ref_vv2par_cutoff(x.shape[0], p(x), p(y), p(g), xt.shape[0], p(xt), p(yt),
                                    float(sigmasqr), p(vx), p(vy))
    return vx, vy


def vorticity_cutoff(x, y, g, sigmasqr, xt=None, yt=None):
    """The reference's own cutoff-kernel vorticity loop (ww2par_C_cpu.c:130-145)."""
    x, y, g, xt, yt = _targets(x, y, g, xt, yt)
    w = np.empty(xt.shape[0])
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    _cutoff_lib().ref_ww2par_cutoff(x.shape[0], p(x), p(y), p(g), xt.shape[0], p(xt), p(yt),
                                    float(sigmasqr), p(w))
    return w
