"""Autotuner: direct sum or FMM, and the FMM leaf level, per blob set.

Model-based, with rates measured on the device once (``calibrate``) and kept
in a JSON cache keyed by the GPU name:

* direct sum:  t = n^2 / R_direct                      (pairs/s of the kernel)
* FMM, leaf L: t = pairs(L) / R_p2p + trans(L) (p+1)^2 / R_m2l + n c_blob + T_fixed
  where pairs(L) and trans(L) come from the exact interaction tables of the
  library (``pf_fmm_lists``) for the blob set's box and cutoff, with the
  blobs assumed to fill the box uniformly.

The reference fixes these choices at build or call time (method flag, Ndirect
and p from tol: src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:538-555).
"""
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import _lib
from ._arrays import ptr

CACHE_ENV = "PFBLOB_TUNE_CACHE"
DEFAULT_RATES = {  # B200 measurements, used until calibrate() runs
    "r_direct": 1.4e12, "r_p2p": 8.4e11, "r_m2l": 1.5e13, "c_blob": 2.5e-10,
    "t_fixed": 2.5e-4, "t_fixed_batch": 3e-5,
}


def _tables(L, w0, cutoff, kb=1):
    need = ctypes.c_int64(0)
    _lib.lib.pf_fmm_lists(L, kb, float(w0), float(cutoff), 0.5, None, 0, ctypes.byref(need))
    buf = (ctypes.c_int32 * need.value)()
    _lib.check(_lib.lib.pf_fmm_lists(L, kb, float(w0), float(cutoff), 0.5, buf, need.value,
                                     ctypes.byref(need)))
    a = list(buf)
    pos = 2
    near = []
    for _ in range(L + 1):
        n = a[pos]
        near.append(n)
        pos += 1 + 2 * n
    far_avg = [0.0]
    for _ in range(1, L + 1):
        npos = a[pos]
        pos += 1
        tot = 0
        for _ in range(npos):
            n = a[pos]
            tot += n
            pos += 1 + 2 * n
        far_avg.append(tot / max(npos, 1))
    nq = a[pos]
    return near, far_avg, nq


class Tuner:
    def __init__(self, device=0, rates=None):
        self.device = device
        self.rates = dict(DEFAULT_RATES)
        self._tab = {}
        if rates:
            self.rates.update(rates)
        else:
            self._load()

    # -- persistence -------------------------------------------------------
    def _cache_path(self):
        p = os.environ.get(CACHE_ENV)
        if p:
            return p
        name = torch.cuda.get_device_name(self.device).replace(" ", "_") if torch.cuda.is_available() else "cpu"
        return os.path.join(os.path.expanduser("~"), ".cache", "pfblob", f"tune_{name}.json")

    def _load(self):
        try:
            with open(self._cache_path()) as f:
                self.rates.update(json.load(f))
        except (OSError, ValueError):
            pass

    def save(self):
        p = self._cache_path()
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            json.dump(self.rates, f, indent=1)

    # -- measurement -------------------------------------------------------
    def calibrate(self, save=True):
        """Measure the kernel rates on this device (about a second)."""
        from . import induced
        from . import workloads as wl
        dev = torch.device("cuda", self.device)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        b = wl.uniform_square(n=32768, sigma=0.002, config=2, instance=77)
        x, y, g = T(b.x), T(b.y), T(b.g)
        vx, vy = torch.empty_like(x), torch.empty_like(x)
        ks = b.ksigmasqr
        for _ in range(2):
            induced.velocity_device(x, y, g, ks, x, y, vx, vy, method=induced.DIRECT_METHOD)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            induced.velocity_device(x, y, g, ks, x, y, vx, vy, method=induced.DIRECT_METHOD)
        torch.cuda.synchronize()
        self.rates["r_direct"] = 3 * float(b.n) ** 2 / (time.perf_counter() - t0)
        # FMM phases on a mid-size uniform set
        b = wl.uniform_square(n=262144, sigma=0.002, config=2, instance=78)
        x, y, g = T(b.x), T(b.y), T(b.g)
        vx, vy = torch.empty_like(x), torch.empty_like(x)
        ks, xo, cut = induced.fmm_parameters(b.sigma)
        _lib.fmm_profile(True, self.device)
        try:
            for _ in range(3):
                induced.velocity_device(x, y, g, ks, x, y, vx, vy, method=induced.FMM_METHOD,
                                        xopt=xo, cutoff=cut)
            st = _lib.fmm_last_stats(self.device)
        finally:
            _lib.fmm_profile(False, self.device)
        npt = st["expansion_terms"]
        self.rates["r_p2p"] = st["p2p_pairs"] / (st["ms_p2p"] * 1e-3)
        self.rates["r_m2l"] = st["m2l_translations"] * npt * npt / (st["ms_m2l"] * 1e-3)
        other = (st["ms_total"] - st["ms_p2p"] - st["ms_m2l"]) * 1e-3
        self.rates["c_blob"] = max(other - self.rates["t_fixed"], 0.0) / b.n
        if save:
            try:
                self.save()
            except OSError:
                pass
        return self.rates

    # -- model ----------------------------------------------------------------
    def fmm_cost(self, n, L, w0, cutoff, np_terms=16, batch=False):
        near, far_avg, nq = self._tables_cached(L, w0, cutoff)
        occ = n / 4.0 ** L
        pairs = n * occ * nq
        trans = sum(4.0 ** l * far_avg[l] for l in range(2, L + 1))
        r = self.rates
        fixed = r["t_fixed_batch"] if batch else r["t_fixed"]
        return pairs / r["r_p2p"] + trans * np_terms ** 2 / r["r_m2l"] + n * r["c_blob"] + fixed

    def choose(self, n, ksigmasqr, box, tol=1e-6, cutoff=None, batch=False):
        """(method, leaf_level): method 0 = FMM, 1 = direct.  ``batch``: the set
        runs inside a captured batch, where the FMM's per-call latency (plan
        look-up, bounding-box read-back, launch gaps) overlaps other sets'
        work and only its device time counts."""
        if n < 64 or tol == 0.0:
            return 1, 0
        w0 = max(box[1] - box[0], box[3] - box[2]) or 1.0
        if cutoff is None:
            from .induced import default_cutoff
            cutoff = default_cutoff(ksigmasqr, tol)
        t_direct = float(n) * n / self.rates["r_direct"]
        best = (t_direct, 1, 0)
        L0 = max(3, int(math.ceil(0.5 * math.log2(max(n, 2) / 35.0))))
        for L in range(max(3, L0 - 2), min(11, L0 + 2) + 1):
            near, far_avg, nq = self._tables_cached(L, w0, cutoff)
            if nq > 1024:
                continue
            t = self.fmm_cost(n, L, w0, cutoff, batch=batch)
            if t < best[0]:
                best = (t, 0, L)
        return best[1], best[2]

    def _tables_cached(self, L, w0, cutoff):
        key = (L, round(cutoff / w0, 12))
        if key not in self._tab:
            self._tab[key] = _tables(L, 1.0, cutoff / w0)
        return self._tab[key]
