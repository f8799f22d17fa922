"""Serving loop: velocity + remesh steps of resident simulations, continuously
batched on one GPU.

Simulations stay on the device (x, y, g as CUDA tensors).  A request asks for
one step of one simulation: the velocity at its blobs (direct sum or FMM, as
the autotuner chose for that simulation) and an M4' remesh of its blobs
(optionally after a forward-Euler move by dt, the reference's
``_convection_fe``; optionally replacing the resident state).

Execution: ``n_slots`` worker threads, each with its own CUDA stream and its
own library context (scratch arena).  A dispatcher admits waiting requests in
arrival order as soon as a slot is free and the device has room: a request's
scratch need is estimated from its blob count, and a slot may only grow its
arena into free HBM (``torch.cuda.mem_get_info``, minus a reserve) that no other
admitted request has claimed.  Requests that arrive while others run are
admitted as slots and memory free up, so their kernels overlap on the device.
Every kernel is deterministic, so a request's result does not depend on what
runs beside it.

With ``step_graphs=True`` the server also captures, at ``warmup()``, one
StepGraph per resident simulation (its pf_blob_step with a private context
and output buffers; see stepgraph.py), as long as free HBM holds them.  A
plain step request (no move, no kept result, no state update) then costs one
graph launch on the slot's stream instead of the step's ~30 kernel launches;
its moments are copied to the request's row.  The graphs hold their scratch
from warm-up on, so such a request claims no arena growth.  Two requests for
the same simulation take its graph one after the other (a per-simulation
lock: CUDA orders launches of one executable graph anyway, the lock also
orders the moment copies).

The reference has no counterpart (one blob set per call, synchronous).
"""
import ctypes
import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .induced import DIRECT_METHOD, FMM_METHOD, fmm_parameters, velocity_device
from .regrid import lattice_window, remesh_device, remesh_device_async
from .tune import Tuner

# scratch bytes per blob of one step (FMM arrays + remesh arrays), measured
# from the library's scratch layouts, plus a per-cell term for the window
# (remesh sums, flags and slots, and the three output arrays)
BYTES_PER_BLOB = 260
BYTES_PER_CELL = 48


@dataclass
class Simulation:
    x: torch.Tensor
    y: torch.Tensor
    g: torch.Tensor
    sigma: float
    k: float = 2.0
    overlap: float = 0.8
    c: float = 0.0
    method: int = -1
    leaf_level: int = 0
    box: tuple = None     # (xmin, xmax, ymin, ymax) of the resident blobs, None = unknown
    window: tuple = None  # remesh base-cell window of `box`

    @property
    def n(self):
        return self.x.numel()

    @property
    def h(self):
        return self.sigma * self.overlap


@dataclass
class Request:
    sim: int
    t_arrival: float
    dt: float = 0.0
    update: bool = False
    t_start: float = 0.0
    t_done: float = 0.0
    n: int = 0
    slot: int = -1
    claim: int = 0
    result: dict = field(default_factory=dict)
    moments: object = None  # FP64 {sum g, sum g x, sum g y, sum |g|} before, after (device)
    idx: int = 0            # position in its trace (row of the server's moment pool)
    error: str = ""

    @property
    def latency_ms(self):
        return (self.t_done - self.t_arrival) * 1e3


class Server:
    def __init__(self, sims, n_slots=8, tol=1e-6, tuner=None, hbm_reserve=2 << 30,
                 free_hbm=None, keep_results=False, device=None, step_graphs=False):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.sims = list(sims)
        self.tol = tol
        self.keep = keep_results
        self.tuner = tuner or Tuner(self.device.index)
        self.reserve = hbm_reserve
        self.free_hbm = free_hbm or (lambda: torch.cuda.mem_get_info(self.device)[0])
        for s in self.sims:
            self._box(s)
            if s.method < 0:
                s.method, s.leaf_level = self.tuner.choose(s.n, s.k * s.sigma * s.sigma, s.box, tol)
        self.n_slots = n_slots
        self._need = {}
        for i in range(len(self.sims)):
            self.need_bytes(i)
        self._lock = threading.Condition()
        self._slot_free = [True] * n_slots
        self._slot_bytes = [0] * n_slots    # arena bytes a slot may already hold
        self._claimed = 0                    # bytes of growth claimed by admitted requests
        self._queues = [queue.Queue() for _ in range(n_slots)]
        self._done = []
        # per-slot device buffers of the lean path (one pf_blob_step per
        # request): velocity and remesh outputs sized for the largest
        # simulation, the count and status words; step descriptors per
        # (slot, simulation), built on first use
        self._slot_buf = [None] * n_slots
        self._desc = {}
        self._mom = torch.zeros((0, 8), dtype=torch.float64, device=self.device)
        self.step_graphs = step_graphs
        self._graphs = {}  # sim -> (x pointer, n, StepGraph)
        self._sim_locks = [threading.Lock() for _ in self.sims]
        self.graph_replays = 0
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True)
                         for i in range(n_slots)]
        for t in self._threads:
            t.start()

    def warmup(self, every_sim=True, timeout=None):
        """Grow every slot's arena to the largest request and build every
        simulation's FMM plan before serving, so that no request pays for an
        allocation or a plan build (both synchronise the device)."""
        big = max(range(len(self.sims)), key=lambda i: self.need_bytes(i))
        self.run_trace([(0.0, big)] * self.n_slots, timeout=timeout)
        if every_sim:
            self.run_trace([(0.0, i) for i in range(len(self.sims))], timeout=timeout)
        if self.step_graphs:
            self.build_graphs()

    def build_graphs(self):
        """Capture the step of every resident simulation that has none (or
        whose state was replaced), while free HBM (less the reserve) holds the
        graph's scratch and outputs; the rest keep the kernel-by-kernel path.
        Each capture synchronises the device: call it while no request runs.
        Returns the number of simulations with a current graph."""
        from .stepgraph import StepGraph
        for i, s in enumerate(self.sims):
            if not s.n:
                continue
            old = self._graphs.get(i)
            if old is not None and old[:2] == (s.x.data_ptr(), s.n):
                continue
            if old is not None:
                old[2].close()
                del self._graphs[i]
            cap = self._bound(s, False) * 3 // 2 + 65536
            if self.need_bytes(i) + 24 * cap + 16 * s.n > self.free_hbm() - self.reserve:
                continue
            ks, xo, cut = fmm_parameters(s.sigma, s.k, tol=self.tol)
            h = s.h
            g = StepGraph(s.x, s.y, s.g, ks, xo, cut, self.tol, self._box(s), h, -1.5 * h,
                          -1.5 * h, c=s.c, method=s.method,
                          leaf_level=s.leaf_level if s.method == FMM_METHOD else 0,
                          max_base_cells=self._bound(s, False), capacity=cap)
            self._graphs[i] = (s.x.data_ptr(), s.n, g)
        return len(self._graphs)

    def _graph(self, req):
        """The step graph that serves `req`, or None (moved, kept or updating
        requests, and simulations without a current graph, take the kernel-by-
        kernel path)."""
        if req.dt != 0.0 or self.keep or req.update:
            return None
        e = self._graphs.get(req.sim)
        if e is None:
            return None
        s = self.sims[req.sim]
        return e[2] if e[:2] == (s.x.data_ptr(), s.n) else None

    # -- memory model -----------------------------------------------------------
    def need_bytes(self, sim):
        """Scratch estimate of one step of simulation `sim` (cached per state)."""
        s = self.sims[sim]
        key = (sim, s.n, s.x.data_ptr())
        v = self._need.get(key)
        if v is None:
            b = self._box(s)
            span = max(b[1] - b[0], b[3] - b[2]) if s.n else 0.0
            cells = (span / s.h + 8.0) ** 2 if s.n else 0.0
            v = int(BYTES_PER_BLOB * s.n + BYTES_PER_CELL * cells) + (1 << 20)
            self._need[key] = v
        return v

    @staticmethod
    def _box(s):
        """Bounding box of a simulation's blobs (one synchronisation; cached
        until the state is replaced)."""
        if s.box is None and s.n:
            b = torch.stack([s.x.min(), s.x.max(), s.y.min(), s.y.max()]).cpu().tolist()
            s.box = tuple(b)
            h = s.h
            s.window = lattice_window(s.box, h, -1.5 * h, -1.5 * h)
        return s.box

    # -- workers ------------------------------------------------------------------
    def _worker(self, slot):
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(self.device)
        while True:
            req = self._queues[slot].get()
            if req is None:
                return
            try:
                with torch.cuda.stream(stream):
                    self._step(req)
                stream.synchronize()
            except Exception as e:  # reported on the request, the server keeps going
                req.error = f"{type(e).__name__}: {e}"
            req.t_done = time.perf_counter()
            with self._lock:
                self._slot_free[slot] = True
                self._claimed -= req.claim  # now allocated, hence seen by free_hbm()
                self._done.append(req)
                self._lock.notify_all()

    def _bound(self, s, moved):
        nbx, nby = s.window[2], s.window[3]
        b = (nbx + 16) * (nby + 16)
        return 4 * b if moved else b

    def _slot_buffers(self, slot, need_n=0, need_cap=0):
        """The slot's buffers, (re)allocated when a simulation outgrows them.
        Called by the slot's own worker between requests (its stream idle),
        so replaced buffers are no longer in use; the slot's descriptors
        pointing at them are dropped."""
        b = self._slot_buf[slot]
        if b is not None and (len(b["vx"]) < need_n or b["cap"] < need_cap):
            for key in [k for k in self._desc if k[0] == slot]:
                self._desc.pop(key, None)
            b = None
        if b is None:
            nmax = max(max(s.n for s in self.sims), need_n)
            cmax = max(max(self._bound(s, False) * 3 // 2 + 65536 for s in self.sims if s.n),
                       need_cap)
            f64 = dict(dtype=torch.float64, device=self.device)
            b = {"vx": torch.empty(nmax, **f64), "vy": torch.empty(nmax, **f64),
                 "out": torch.empty((3, cmax), **f64), "cap": cmax,
                 "nout": torch.zeros(1, dtype=torch.int64, device=self.device),
                 "status": torch.zeros(1, dtype=torch.int32, device=self.device)}
            self._slot_buf[slot] = b
        return b

    def _descriptor(self, slot, sim):
        """pf_step of simulation `sim` on slot `slot` (cached; rebuilt when
        the simulation's state is replaced)."""
        s = self.sims[sim]
        b = self._slot_buffers(slot, s.n, self._bound(s, False) * 3 // 2 + 65536)
        key = (slot, sim, s.x.data_ptr(), s.n)
        d = self._desc.get(key)
        if d is None:
            ks, xo, cut = fmm_parameters(s.sigma, s.k, tol=self.tol)
            h = s.h
            d = _lib.Step()
            d.n, d.x, d.y, d.g = s.n, s.x.data_ptr(), s.y.data_ptr(), s.g.data_ptr()
            d.ksigmasqr, d.xopt, d.cutoff, d.tol = ks, xo, cut, self.tol
            d.method, d.leaf_level = s.method, s.leaf_level if s.method == FMM_METHOD else 0
            for i, v in enumerate(self._box(s)):
                d.box[i] = v
            d.vx, d.vy = b["vx"].data_ptr(), b["vy"].data_ptr()
            d.h, d.xb0, d.yb0, d.c = h, -1.5 * h, -1.5 * h, s.c
            d.max_base_cells, d.capacity = self._bound(s, False), b["cap"]
            o = b["out"]
            d.x_out, d.y_out, d.g_out = o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr()
            d.n_out_dev, d.status_dev = b["nout"].data_ptr(), b["status"].data_ptr()
            self._desc[key] = d
        return d

    def _step(self, req):
        """Enqueue one step on the current stream.  With the blob box known
        (resident state, no move) nothing here waits for the device: the FMM
        takes the cached box and the remesh finds its window on the device;
        such a step is one pf_blob_step call into slot buffers."""
        s = self.sims[req.sim]
        g = self._graph(req)
        if g is not None:
            stream = torch.cuda.current_stream(self.device)
            with self._sim_locks[req.sim]:
                g.launch(stream.cuda_stream)
                self._mom[req.idx].copy_(g.moments, non_blocking=True)
                stream.synchronize()  # the graph's buffers are free for the next request
            req.n = s.n
            req.moments = self._mom[req.idx]
            with self._lock:
                self.graph_replays += 1
            return
        if req.dt == 0.0 and not (self.keep or req.update) and s.n:
            d = self._descriptor(req.slot, req.sim)
            d.moments_dev = self._mom[req.idx].data_ptr()
            st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
            _lib.check(_lib.lib.pf_blob_step(_lib.context(self.device.index), ctypes.byref(d), st))
            req.n = s.n
            req.moments = self._mom[req.idx]
            return
        ks, xo, cut = fmm_parameters(s.sigma, s.k, tol=self.tol)
        vx = torch.empty_like(s.x)
        vy = torch.empty_like(s.x)
        box = self._box(s)
        if s.method == FMM_METHOD:
            _lib.fmm_set_tuning(s.leaf_level, 0, 1)
        velocity_device(s.x, s.y, s.g, ks, s.x, s.y, vx, vy, method=s.method, xopt=xo, cutoff=cut,
                        tol=self.tol, box=box)
        h = s.h
        xm, ym = s.x, s.y
        if req.dt != 0.0:
            xm = s.x + req.dt * vx
            ym = s.y + req.dt * vy
        # remesh with the window found on the device (bounded by the resident
        # set's window with a margin for moved blobs) and the FP64 moments of
        # the blobs before and after (the step's circulation and impulse check)
        xn, yn, gn, nout, status, win, mom = remesh_device_async(
            xm, ym, s.g, h, -1.5 * h, -1.5 * h, s.c, max_base_cells=self._bound(s, req.dt != 0.0))
        if req.dt != 0.0 or self.keep or req.update:
            k, st = int(nout.item()), int(status.item())
            if st:  # moved past the bound: the synchronous remesh finds any window
                xn, yn, gn = remesh_device(xm, ym, s.g, h, -1.5 * h, -1.5 * h, s.c)
                mom = None
            else:
                xn, yn, gn = xn[:k], yn[:k], gn[:k]
        req.n = s.n
        req.moments = mom
        if self.keep:
            req.result = {"vx": vx, "vy": vy, "x": xn, "y": yn, "g": gn}
        if req.update:
            with self._sim_locks[req.sim]:
                e = self._graphs.pop(req.sim, None)
                if e is not None:
                    e[2].close()
                s.x, s.y, s.g = xn, yn, gn
                s.box = s.window = None

    # -- dispatcher ---------------------------------------------------------------
    def _try_admit(self, req):
        """Admit `req` to a free slot if memory allows; returns True if started."""
        # a step graph holds its own scratch: nothing to claim
        need = 0 if self._graph(req) is not None else self.need_bytes(req.sim)
        free_slots = [i for i in range(self.n_slots) if self._slot_free[i]]
        if not free_slots:
            return False
        # prefer a slot whose arena already holds the need (no growth)
        fit = [i for i in free_slots if self._slot_bytes[i] >= need]
        slot = fit[0] if fit else max(free_slots, key=lambda i: self._slot_bytes[i])
        growth = max(0, need - self._slot_bytes[slot])
        if growth > 0 and growth + self._claimed > self.free_hbm() - self.reserve:
            return False
        self._slot_free[slot] = False
        self._slot_bytes[slot] = max(self._slot_bytes[slot], need)
        self._claimed += growth
        req.claim = growth
        req.slot = slot
        req.t_start = time.perf_counter()
        self._queues[slot].put(req)
        return True

    def run_trace(self, trace, dt=0.0, update=False, timeout=None):
        """Replay (t_offset_seconds, sim_id) arrivals in real time; returns the
        completed requests in completion order."""
        trace = sorted(trace)
        if self._mom.shape[0] < len(trace):  # a moment row per request of the trace
            self._mom = torch.zeros((len(trace), 8), dtype=torch.float64, device=self.device)
        t0 = time.perf_counter()
        pending = []
        reqs = []
        i = 0
        with self._lock:
            self._done = []
        deadline = None if timeout is None else t0 + timeout
        while True:
            now = time.perf_counter()
            while i < len(trace) and t0 + trace[i][0] <= now:
                r = Request(sim=int(trace[i][1]), t_arrival=t0 + trace[i][0], dt=dt, update=update,
                            idx=i)
                pending.append(r)
                reqs.append(r)
                i += 1
            with self._lock:
                while pending and self._try_admit(pending[0]):
                    pending.pop(0)
                if i >= len(trace) and not pending and len(self._done) == len(reqs):
                    break
                if deadline is not None and now > deadline:
                    raise TimeoutError("serving trace did not finish in time")
                wait = 0.002
                if i < len(trace):
                    wait = min(wait, max(0.0, t0 + trace[i][0] - now))
                self._lock.wait(timeout=wait)
        with self._lock:
            return list(self._done)

    def close(self):
        for q in self._queues:
            q.put(None)
        for t in self._threads:
            t.join(timeout=10)
        for e in self._graphs.values():
            e[2].close()
        self._graphs = {}


def poisson_trace(n_requests, rate, n_sims, seed=0):
    """Arrival offsets (s) of a Poisson process of `rate` requests/s, each for a
    uniformly chosen simulation."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    sims = rng.integers(0, n_sims, n_requests)
    return list(zip(t.tolist(), sims.tolist()))


def conservation(done, sims):
    """Largest relative circulation and linear-impulse change over the served
    steps (FP64 moments from the remesh, read after the trace; impulse
    normalised by sum |g| times the largest coordinate of the blobs)."""
    circ = imp = 0.0
    checked = 0
    for r in done:
        if r.error or r.moments is None:
            continue
        m = r.moments.cpu().tolist()
        den = m[3] if m[3] > 0 else 1.0
        sc = max(abs(v) for v in sims[r.sim].box) if sims[r.sim].box else 1.0
        circ = max(circ, abs(m[4] - m[0]) / den)
        imp = max(imp, max(abs(m[5] - m[1]), abs(m[6] - m[2])) / (den * (sc or 1.0)))
        checked += 1
    return {"circulation": circ, "linear_impulse": imp, "steps_checked": checked}


def summarize(done, t_span=None):
    lat = np.array([r.latency_ms for r in done if not r.error])
    n = sum(r.n for r in done if not r.error)
    if t_span is None and done:
        t_span = max(r.t_done for r in done) - min(r.t_arrival for r in done)
    return {"requests": len(done), "errors": sum(1 for r in done if r.error),
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else math.nan,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else math.nan,
            "evals_per_s": n / t_span if t_span else math.nan, "blobs": n, "span_s": t_span}
