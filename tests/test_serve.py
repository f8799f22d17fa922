"""Serving loop: trace generation, summaries and the admission policy (CPU),
and on the GPU: results are the same alone and in the mix, admission follows
free HBM, a simulated out-of-memory device makes requests wait and the loop
report it."""
import numpy as np
import pytest
import torch


def test_poisson_trace_and_summary_cpu():
    from pfblob.serve import Request, poisson_trace, summarize
    tr = poisson_trace(1000, 500.0, 7, seed=3)
    t = np.array([a for a, _ in tr])
    assert np.all(np.diff(t) > 0) and abs(t[-1] - 2.0) < 0.3
    assert {s for _, s in tr} <= set(range(7))
    reqs = [Request(sim=0, t_arrival=0.0, t_done=0.001 * (i + 1), n=100) for i in range(100)]
    s = summarize(reqs, t_span=1.0)
    assert abs(s["p50_ms"] - 50.5) < 1e-9 and s["evals_per_s"] == 10000


def _admission_only_server(n_slots, free, reserve, needs):
    """A Server with its admission state and no device or worker threads: the
    policy of _try_admit on the host, with a fake free-HBM reading."""
    import queue
    from pfblob.serve import Server
    s = Server.__new__(Server)
    s.n_slots = n_slots
    s._slot_free = [True] * n_slots
    s._slot_bytes = [0] * n_slots
    s._claimed = 0
    s._queues = [queue.Queue() for _ in range(n_slots)]
    s.keep = False
    s._graphs = {}
    s.reserve = reserve
    s.free_hbm = lambda: free[0]
    s.need_bytes = lambda sim: needs[sim]
    return s


def test_admission_policy_cpu():
    from pfblob.serve import Request
    GB = 1 << 30
    free = [10 * GB]
    s = _admission_only_server(2, free, reserve=2 * GB, needs={0: 3 * GB, 1: 6 * GB, 2: 1 * GB})
    a = Request(sim=0, t_arrival=0.0)
    assert s._try_admit(a) and a.claim == 3 * GB and s._claimed == 3 * GB
    # 6 GB more would exceed free - reserve - claimed = 5 GB: waits
    b = Request(sim=1, t_arrival=0.0)
    assert not s._try_admit(b) and b.slot == -1
    # a request that fits in the remaining room is admitted to the other slot
    c = Request(sim=2, t_arrival=0.0)
    assert s._try_admit(c) and c.slot != a.slot and c.claim == 1 * GB
    # no free slot: waits whatever the memory
    assert not s._try_admit(Request(sim=2, t_arrival=0.0))
    # slot of `a` done (its growth now allocated, so no longer claimed); a
    # request that fits the 3 GB arena of that slot needs no growth
    s._slot_free[a.slot] = True
    s._claimed -= a.claim
    free[0] = 7 * GB
    d = Request(sim=0, t_arrival=0.0)
    assert s._try_admit(d) and d.slot == a.slot and d.claim == 0
    assert s._queues[a.slot].qsize() == 2 and s._queues[c.slot].qsize() == 1


def test_admission_prefers_the_slot_that_already_fits_cpu():
    from pfblob.serve import Request
    GB = 1 << 30
    s = _admission_only_server(3, [100 * GB], reserve=0, needs={0: 4 * GB})
    s._slot_bytes = [1 * GB, 5 * GB, 2 * GB]
    r = Request(sim=0, t_arrival=0.0)
    assert s._try_admit(r) and r.slot == 1 and r.claim == 0
    # slot 1 is busy now: no free slot fits, so the largest free arena grows
    # (the least growth)
    r2 = Request(sim=0, t_arrival=0.0)
    assert s._try_admit(r2) and r2.slot == 2 and r2.claim == 2 * GB


def _sims(sizes, config=5):
    from pfblob import workloads as wl
    from pfblob.serve import Simulation
    dev = torch.device("cuda", 0)
    out = []
    for i, n in enumerate(sizes):
        b = wl.mixed_instance(int(n), config=config, instance=i)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        out.append(Simulation(T(b.x), T(b.y), T(b.g), sigma=b.sigma))
    return out


@pytest.mark.gpu
def test_same_result_alone_and_in_the_mix():
    from pfblob.serve import Server, poisson_trace
    sizes = [1500, 6000, 20000, 50000, 120000, 3000, 9000, 70000]
    trace = poisson_trace(24, 20000.0, len(sizes), seed=1)  # arrivals faster than service
    mix = Server(_sims(sizes), n_slots=6, keep_results=True)
    done_mix = mix.run_trace(trace, timeout=120)
    mix.close()
    alone = Server(_sims(sizes), n_slots=1, keep_results=True)
    done_alone = alone.run_trace(trace, timeout=120)
    alone.close()
    assert len(done_mix) == len(done_alone) == 24
    assert not any(r.error for r in done_mix + done_alone)
    # requests overlapped in the mix
    iv = sorted((r.t_start, r.t_done) for r in done_mix)
    assert any(b[0] < a[1] for a, b in zip(iv, iv[1:]))
    key = lambda r: (r.t_arrival, r.sim)
    for a, b in zip(sorted(done_mix, key=key), sorted(done_alone, key=key)):
        assert a.sim == b.sim
        for k in ("vx", "vy", "x", "y", "g"):
            assert torch.equal(a.result[k], b.result[k]), k
        assert torch.equal(a.moments, b.moments)


@pytest.mark.gpu
def test_served_steps_conserve_circulation_and_impulse():
    """Every served step carries the FP64 moments of its blobs before and
    after the remesh; circulation and linear impulse are conserved to 1e-12,
    with and without a forward-Euler move."""
    from pfblob.serve import Server, conservation, poisson_trace
    sims = _sims([1500, 6000, 20000, 50000, 120000])
    srv = Server(sims, n_slots=4)
    done = srv.run_trace(poisson_trace(20, 5000.0, len(sims), seed=4), timeout=120)
    c = conservation(done, srv.sims)
    assert c["steps_checked"] == 20 and c["circulation"] <= 1e-12 and c["linear_impulse"] <= 1e-12
    moved = srv.run_trace(poisson_trace(10, 5000.0, len(sims), seed=5), dt=1e-3, timeout=120)
    c = conservation(moved, srv.sims)
    assert c["steps_checked"] == 10 and c["circulation"] <= 1e-12 and c["linear_impulse"] <= 1e-12
    srv.close()


@pytest.mark.gpu
def test_admission_follows_free_hbm_and_reports_oom():
    from pfblob.serve import Server, poisson_trace
    sims = _sims([30000, 30000, 30000, 30000])
    # a device with room for one request's scratch growth at a time
    srv = Server(sims, n_slots=4, hbm_reserve=0)
    one = max(srv.need_bytes(i) for i in range(4))
    srv.free_hbm = lambda: one + 1
    done = srv.run_trace(poisson_trace(4, 1e6, 4, seed=2), timeout=120)
    grown = sorted((r.t_start, r.t_done) for r in done if r.claim > 0)
    assert len(done) == 4 and all(b[0] >= a[1] for a, b in zip(grown, grown[1:]))
    srv.close()
    # no room at all: the request waits, the loop reports instead of hanging
    srv = Server(_sims([40000]), n_slots=2, hbm_reserve=0, free_hbm=lambda: 0)
    with pytest.raises(TimeoutError):
        srv.run_trace([(0.0, 0)], timeout=1.0)
    srv.close()


@pytest.mark.gpu
def test_update_replaces_resident_state():
    from pfblob.serve import Server
    sims = _sims([5000])
    srv = Server(sims, n_slots=1, keep_results=True)
    done = srv.run_trace([(0.0, 0)], update=True, timeout=60)
    assert sims[0].n == done[0].result["x"].numel() != 5000
    srv.close()


@pytest.mark.gpu
def test_step_graph_serving_matches_kernel_by_kernel_serving():
    """A server that replays one captured step per simulation gives, request
    by request, bitwise the FP64 moments of the kernel-by-kernel server
    (before and after each remesh), conserves them, launches one graph per
    request, and its velocities agree with the kept results of a plain run."""
    from pfblob.serve import Server, conservation, poisson_trace
    sizes = [1500, 6000, 20000, 50000, 120000, 3000]
    trace = poisson_trace(30, 20000.0, len(sizes), seed=7)
    gsrv = Server(_sims(sizes), n_slots=4, step_graphs=True)
    gsrv.warmup()
    assert len(gsrv._graphs) == len(sizes)
    r0 = gsrv.graph_replays
    done_g = gsrv.run_trace(trace, timeout=120)
    assert gsrv.graph_replays - r0 == 30 and not any(r.error for r in done_g)
    c = conservation(done_g, gsrv.sims)
    assert c["steps_checked"] == 30 and c["circulation"] <= 1e-12 and c["linear_impulse"] <= 1e-12
    esrv = Server(_sims(sizes), n_slots=4)
    done_e = esrv.run_trace(trace, timeout=120)
    esrv.close()
    key = lambda r: r.idx
    for a, b in zip(sorted(done_g, key=key), sorted(done_e, key=key)):
        assert a.sim == b.sim and torch.equal(a.moments, b.moments)
    # the velocity of each graph's last replay against the kept result of a
    # kernel-by-kernel step of the same resident set
    ksrv = Server(_sims(sizes), n_slots=1, keep_results=True)
    kept = {r.sim: r for r in ksrv.run_trace([(0.0, i) for i in range(len(sizes))], timeout=120)}
    ksrv.close()
    for i, (_, n, g) in gsrv._graphs.items():
        vx, vy = kept[i].result["vx"], kept[i].result["vy"]
        err = torch.sqrt(((g.vx - vx) ** 2 + (g.vy - vy) ** 2).sum() / (vx ** 2 + vy ** 2).sum())
        assert float(err) <= 1e-9, (i, n, float(err))
    # a state update drops that simulation's graph; its next plain request
    # takes the kernel-by-kernel path
    gsrv.run_trace([(0.0, 0)], update=True, timeout=60)
    assert 0 not in gsrv._graphs
    r1 = gsrv.graph_replays
    assert not gsrv.run_trace([(0.0, 0)], timeout=60)[0].error and gsrv.graph_replays == r1
    gsrv.close()
