"""Many independent blob simulations per launch (the C ABI's pf_batch_*).

A ``Batch`` holds device-resident blob sets of uneven sizes.  Its step --
velocity of every set at its own blobs plus an M4' remesh of every set -- is
captured once into a CUDA graph and replayed with one launch: small sets run
together in one persistent direct-sum kernel, larger ones through the FMM,
chosen per set by the autotuner (``tune.Tuner``).
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._arrays import require
from .induced import default_cutoff
from .tune import Tuner



class Batch:
    def __init__(self, sims, tol=1e-6, n_streams=8, remesh=True, tuner=None, device=None,
                 methods=None, leaf_levels=None):
        """sims: list of dicts with CUDA float64 tensors x, y, g and floats
        sigma, k (default 2), overlap (default 0.8), xb0/yb0 (remesh lattice
        origin, default -1.5 h as Blobs.redistribute), c (Wee, default 0)."""
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.tuner = tuner or Tuner(self.device.index)
        self.sims = []
        descs = (_lib.BatchInstance * max(1, len(sims)))()
        xs = [s["x"] for s in sims]
        ys = [s["y"] for s in sims]
        # bounding boxes of every set (one synchronisation at creation)
        if sims:
            mins = torch.stack([torch.stack([a.min(), b.min()]) for a, b in zip(xs, ys)]).cpu().numpy()
            maxs = torch.stack([torch.stack([a.max(), b.max()]) for a, b in zip(xs, ys)]).cpu().numpy()
        for i, s in enumerate(sims):
            x, y, g = s["x"], s["y"], s["g"]
            n = x.numel()
            require(n, self.device, x=x, y=y, g=g)
            sigma = float(s["sigma"])
            k = float(s.get("k", 2.0))
            overlap = float(s.get("overlap", 0.8))
            h = sigma * overlap
            ks = k * sigma * sigma
            cutoff = default_cutoff(ks, tol)
            box = (float(mins[i, 0]), float(maxs[i, 0]), float(mins[i, 1]), float(maxs[i, 1]))
            if methods is not None:
                m, L = int(methods[i]), int(leaf_levels[i]) if leaf_levels is not None else 0
            else:
                m, L = self.tuner.choose(n, ks, box, tol, cutoff, batch=True)
            vx = torch.empty(n, dtype=torch.float64, device=self.device)
            vy = torch.empty(n, dtype=torch.float64, device=self.device)
            d = descs[i]
            d.n = n
            d.x, d.y, d.g = x.data_ptr(), y.data_ptr(), g.data_ptr()
            d.vx, d.vy = vx.data_ptr(), vy.data_ptr()
            d.ksigmasqr = ks
            d.cutoff = cutoff
            for j, v in enumerate(box):
                d.box[j] = v
            d.method = m
            d.leaf_level = L
            d.expansion_terms = 0
            rec = {"n": n, "vx": vx, "vy": vy, "method": m, "leaf_level": L, "keep": (x, y, g)}
            if remesh:
                xb0 = float(s.get("xb0", -1.5 * h))
                yb0 = float(s.get("yb0", -1.5 * h))
                # every output cell lies in the window of the box: an exact bound
                wx = math.ceil((box[1] - box[0]) / h) + 6
                wy = math.ceil((box[3] - box[2]) / h) + 6
                cap = int(min(16 * n, wx * wy))
                xo = torch.empty(cap, dtype=torch.float64, device=self.device)
                yo = torch.empty(cap, dtype=torch.float64, device=self.device)
                go = torch.empty(cap, dtype=torch.float64, device=self.device)
                d.remesh = 1
                d.h, d.xb0, d.yb0, d.c = h, xb0, yb0, float(s.get("c", 0.0))
                d.capacity = cap
                d.x_out, d.y_out, d.g_out = xo.data_ptr(), yo.data_ptr(), go.data_ptr()
                rec.update(x_out=xo, y_out=yo, g_out=go)
            else:
                d.remesh = 0
            self.sims.append(rec)
        self._descs = descs
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.pf_batch_create(_lib.context(self.device.index), len(sims), descs,
                                            float(tol), int(n_streams), ctypes.byref(h)))
        self.handle = h
        meth = (ctypes.c_int32 * max(1, len(sims)))()
        lev = (ctypes.c_int32 * max(1, len(sims)))()
        nodes = ctypes.c_int64(0)
        _lib.check(_lib.lib.pf_batch_info(h, meth, lev, ctypes.byref(nodes)))
        for i, r in enumerate(self.sims):
            r["method"], r["leaf_level"] = int(meth[i]), int(lev[i])
        self.kernel_nodes = nodes.value

    @property
    def n_total(self):
        return sum(r["n"] for r in self.sims)

    def run(self, stream=None):
        st = torch.cuda.current_stream(self.device).cuda_stream if stream is None else stream
        _lib.check(_lib.lib.pf_batch_run(self.handle, ctypes.c_void_p(st)))

    def results(self):
        """Wait for the last run; list of dicts with vx, vy and the remeshed
        x, y, g (views of the device buffers) and a status per set."""
        n = len(self.sims)
        nout = np.zeros(max(1, n), dtype=np.int64)
        status = np.zeros(max(1, n), dtype=np.int32)
        _lib.check(_lib.lib.pf_batch_results(self.handle, nout.ctypes.data_as(ctypes.c_void_p),
                                             status.ctypes.data_as(ctypes.c_void_p)))
        out = []
        for i, r in enumerate(self.sims):
            o = {"vx": r["vx"], "vy": r["vy"], "status": int(status[i]), "method": r["method"],
                 "leaf_level": r["leaf_level"]}
            if "x_out" in r:
                k = int(nout[i])
                o.update(x=r["x_out"][:k], y=r["y_out"][:k], g=r["g_out"][:k])
            out.append(o)
        return out

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib.pf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
