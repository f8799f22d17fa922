"""M4' remesh with pHyFlow's ``Regrid`` call surface
(``src/python/blobs/base/regrid/_regridding.py:36-222``)."""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._arrays import Marshal, ptr, require

M4PRIME_INTERPKERNEL = 0


def remesh_device(x, y, g, h, xb0, yb0, c=0.0, capacity=None, with_indices=False, stream=None,
                  population_control=None, tutty_hnu=None):
    """Device-tensor entry.  Returns (x, y, g[, ix, iy]) CUDA tensors of the
    new blobs in (ix, iy) order.  ``capacity`` bounds the output (default
    16 n, the window count); a retry with the exact size follows a capacity
    error.  ``population_control = (gThresholdLocal, gThresholdGlobal)``
    applies PopulationControl to the new blobs in the same pass (dropped cells
    are never written); the threshold used is then appended to the result.
    ``tutty_hnu`` (= sqrt(dt nu)) selects Tutty's diffusive weights instead of
    M4' (``c`` is then unused)."""
    n = x.numel()
    dev = x.device
    require(n, dev, x=x, y=y, g=g)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    ctx = _lib.context(dev.index)
    if capacity is None:
        capacity = 16 * n
    while True:
        xo = torch.empty(capacity, dtype=torch.float64, device=dev)
        yo = torch.empty(capacity, dtype=torch.float64, device=dev)
        go = torch.empty(capacity, dtype=torch.float64, device=dev)
        ixo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
        iyo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
        nout = ctypes.c_int64(0)
        thr = ctypes.c_double(0.0)
        if tutty_hnu is not None:
            if population_control is not None:
                raise ValueError("population_control applies to the M4' remesh only")
            s = _lib.lib.pf_remesh_tutty(ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0),
                                         float(yb0), float(tutty_hnu), capacity, ptr(xo), ptr(yo),
                                         ptr(go), ptr(ixo), ptr(iyo), ctypes.byref(nout), st)
        elif population_control is None:
            s = _lib.lib.pf_remesh(ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0),
                                   float(yb0), float(c), capacity, ptr(xo), ptr(yo), ptr(go),
                                   ptr(ixo), ptr(iyo), ctypes.byref(nout), st)
        else:
            tl, tg = population_control
            s = _lib.lib.pf_remesh_population_control(
                ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0), float(yb0), float(c),
                float(tl), float(tg), capacity, ptr(xo), ptr(yo), ptr(go), ptr(ixo), ptr(iyo),
                ctypes.byref(nout), ctypes.byref(thr), st)
        if s == 6 and nout.value > capacity:  # PF_ERR_CAPACITY
            capacity = nout.value
            continue
        _lib.check(s)
        k = nout.value
        out = (xo[:k], yo[:k], go[:k])
        if with_indices:
            out = out + (ixo[:k], iyo[:k])
        if population_control is not None:
            out = out + (thr.value,)
        return out


def remesh_device_async(x, y, g, h, xb0, yb0, c=0.0, max_base_cells=None, capacity=None,
                        with_indices=False, stream=None):
    """Remesh with the lattice window found on the device and no host
    synchronisation (pf_remesh_async).  Returns (x, y, g[, ix, iy], n_out,
    status, window, moments): outputs of ``capacity`` entries (default: the
    output cells of a window of ``max_base_cells``), and CUDA tensors with the
    output count, the status word (0 = done; 8 = the window exceeded
    ``max_base_cells``: retry with ``window[2] * window[3]``), the window
    {ixmin, iymin, nbx, nby} and the FP64 moments {sum g, sum g x, sum g y,
    sum |g|} of the input blobs then of the new blobs (8 values; see
    ``conservation_error``).  ``max_base_cells`` defaults to 4 n."""
    n = x.numel()
    dev = x.device
    require(n, dev, x=x, y=y, g=g)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    ctx = _lib.context(dev.index)
    mb = int(max_base_cells) if max_base_cells is not None else max(4 * n, 4096)
    if capacity is None:
        capacity = mb + mb // 2 + 65536
    xo = torch.empty(capacity, dtype=torch.float64, device=dev)
    yo = torch.empty(capacity, dtype=torch.float64, device=dev)
    go = torch.empty(capacity, dtype=torch.float64, device=dev)
    ixo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
    iyo = torch.empty(capacity, dtype=torch.int64, device=dev) if with_indices else None
    # written by the call's last kernel, whatever happens on the device
    nout = torch.empty(1, dtype=torch.int64, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    window = torch.empty(4, dtype=torch.int64, device=dev)
    moments = torch.empty(8, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib.pf_remesh_async(ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0),
                                        float(yb0), float(c), mb, capacity, ptr(xo), ptr(yo),
                                        ptr(go), ptr(ixo), ptr(iyo), ptr(nout), ptr(status),
                                        ptr(window), ptr(moments), st))
    out = (xo, yo, go)
    if with_indices:
        out = out + (ixo, iyo)
    return out + (nout, status, window, moments)


def lattice_window(box, h, xb0, yb0):
    """Base-cell window (ixmin, iymin, nbx, nby) holding every blob inside
    box = (xmin, xmax, ymin, ymax): the remesh's window-left index
    ceil((((x - xb0) - 2h) + h/2) / h) - 1 (same rounding as the device) of
    the box corners."""
    h2, h05 = 2.0 * h, 0.5 * h

    def left(v, b0):
        return math.ceil((((v - b0) - h2) + h05) / h) - 1

    ix0, ix1 = left(box[0], xb0), left(box[1], xb0)
    iy0, iy1 = left(box[2], yb0), left(box[3], yb0)
    return ix0, iy0, ix1 - ix0 + 1, iy1 - iy0 + 1


def remesh_window_device(x, y, g, h, xb0, yb0, window, c=0.0, stream=None):
    """Remesh onto a known base-cell window (pf_remesh_window): no host
    synchronisation.  Returns (x, y, g, n_out) where the outputs hold the
    window's (nbx+3)(nby+3) cells and n_out is a 1-element CUDA int64 tensor
    with the number of new blobs (the first n_out entries)."""
    n = x.numel()
    dev = x.device
    require(n, dev, x=x, y=y, g=g)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    ctx = _lib.context(dev.index)
    ixmin, iymin, nbx, nby = (int(v) for v in window)
    cap = (nbx + 3) * (nby + 3)
    xo = torch.empty(cap, dtype=torch.float64, device=dev)
    yo = torch.empty(cap, dtype=torch.float64, device=dev)
    go = torch.empty(cap, dtype=torch.float64, device=dev)
    nout = torch.zeros(1, dtype=torch.int64, device=dev)
    _lib.check(_lib.lib.pf_remesh_window(ctx, n, ptr(x), ptr(y), ptr(g), float(h), float(xb0),
                                         float(yb0), float(c), ixmin, iymin, nbx, nby, cap,
                                         ptr(xo), ptr(yo), ptr(go), None, None, ptr(nout), None,
                                         st))
    return xo, yo, go, nout


def population_control_device(x, y, g, g_threshold_local, g_threshold_global, stream=None):
    """PopulationControl of device tensors: returns (x, y, g, threshold used)
    with the kept blobs in input order (reads the kept count back: one
    synchronisation)."""
    n = x.numel()
    dev = x.device
    require(n, dev, x=x, y=y, g=g)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    ctx = _lib.context(dev.index)
    xo = torch.empty(n, dtype=torch.float64, device=dev)
    yo = torch.empty(n, dtype=torch.float64, device=dev)
    go = torch.empty(n, dtype=torch.float64, device=dev)
    res = torch.empty(2, dtype=torch.float64, device=dev)  # [n_out (int64 bits), threshold]
    _lib.check(_lib.lib.pf_population_control(
        ctx, n, ptr(x), ptr(y), ptr(g), float(g_threshold_local), float(g_threshold_global),
        ptr(xo), ptr(yo), ptr(go), ptr(res), res.data_ptr() + 8, st))
    r = res.cpu()
    k = int(r[:1].view(torch.int64).item())
    return xo[:k], yo[:k], go[:k], float(r[1].item())


def PopulationControl(xBlob, yBlob, wBlob, wThreshold, wTotalThreshold):
    """Drop blobs with |g| below wThreshold, lowering the threshold by decades
    until the dropped circulation is below wTotalThreshold; same arguments and
    results as pHyFlow's ``PopulationControl``
    (``src/python/blobs/base/regrid/_regridding.py:226-330``)."""
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    xn, yn, gn, _ = population_control_device(x, y, g, wThreshold, wTotalThreshold)
    return m.outs(xn, yn, gn)


def Regrid(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, interpKernel=0, c=0.0):
    """Redistribute blobs onto the lattice of spacing h = sigma*overlap.

    Same arguments and results as pHyFlow's ``Regrid``: new (x, y, g) of every
    lattice node touched by a blob's 4x4 M4' window, explicit zeros kept,
    ordered by (ix, iy); ``c`` is the Wee diffusion coefficient.
    """
    if interpKernel != M4PRIME_INTERPKERNEL:
        raise NotImplementedError("pfblob: only the M4' kernel (interpKernel=0) exists")
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if x.numel() < 1:  # the reference returns its inputs unchanged (:143-146)
        return xBlob, yBlob, wBlob
    h = sigma * overlap
    xb0 = float(np.asarray(xBounds)[0]) if not isinstance(xBounds, torch.Tensor) else float(xBounds[0])
    yb0 = float(np.asarray(yBounds)[0]) if not isinstance(yBounds, torch.Tensor) else float(yBounds[0])
    xn, yn, gn = remesh_device(x, y, g, h, xb0, yb0, c)
    return m.outs(xn, yn, gn)


def velocity_and_regrid(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, k=2, method=0,
                        Ndirect=35, tol=1.0e-6, cutoff=None, c=0.0):
    """One blob step's two hot calls from a single upload: the induced
    velocity at the blobs (``velocity(xBlob, yBlob, wBlob, sigma, k, ...,
    method, Ndirect, tol, cutoff)``) and the redistribution
    ``Regrid(xBlob, yBlob, wBlob, sigma, overlap, xBounds, yBounds, 0, c)``
    of the same blobs, as a caller of both would make them (the reference's
    ``Blobs.evaluateVelocity`` then ``Blobs.redistribute``,
    ``src/python/blobs/__blobsClass.py:546-626, 828-897``).  Returns
    ``(vx, vy, x_new, y_new, g_new)``; numpy (or CPU tensor) input is copied to
    the device once, and the results come back with one synchronisation."""
    from .induced import FMM_METHOD, DIRECT_METHOD, fmm_parameters, velocity_device
    if method not in (FMM_METHOD, DIRECT_METHOD):
        raise ValueError(f"pfblob: unknown method {method}")
    m = Marshal(xBlob.device.index if isinstance(xBlob, torch.Tensor) and xBlob.is_cuda else None)
    x, y, g = m.dev(xBlob), m.dev(yBlob), m.dev(wBlob)
    if not (x.numel() == y.numel() == g.numel()):
        raise ValueError("pfblob: xBlob, yBlob, wBlob must have the same length")
    vx, vy = m.empty(x.numel()), m.empty(x.numel())
    ksigmasqr, xopt, cut = fmm_parameters(float(sigma), float(k), cutoff, float(tol))
    velocity_device(x, y, g, ksigmasqr, x, y, vx, vy, method=method, xopt=xopt, cutoff=cut,
                    tol=float(tol), ndirect=int(Ndirect), device=m.index)
    if x.numel() < 1:
        return m.outs(vx, vy, x, y, g)
    h = sigma * overlap
    xb0 = float(np.asarray(xBounds)[0]) if not isinstance(xBounds, torch.Tensor) else float(xBounds[0])
    yb0 = float(np.asarray(yBounds)[0]) if not isinstance(yBounds, torch.Tensor) else float(yBounds[0])
    hv = None
    if m.host:  # the velocities go back on a side stream while the remesh runs
        main = torch.cuda.current_stream(m.device)
        done = torch.cuda.Event()
        done.record(main)
        side = _side_stream(m.device)
        hv = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in (vx, vy)]
        with torch.cuda.stream(side):
            side.wait_event(done)
            for hh, t in zip(hv, (vx, vy)):
                hh.copy_(t, non_blocking=True)
    xn, yn, gn = remesh_device(x, y, g, h, xb0, yb0, c)
    if hv is None:
        return m.outs(vx, vy, xn, yn, gn)
    rest = m.outs(xn, yn, gn)
    side.synchronize()
    return (hv[0].numpy(), hv[1].numpy()) + tuple(rest)


_SIDE = {}


def _side_stream(dev):
    """A second stream per device for copies that overlap the main stream's work."""
    s = _SIDE.get(dev.index)
    if s is None:
        s = _SIDE[dev.index] = torch.cuda.Stream(dev)
    return s
