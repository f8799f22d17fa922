"""Benchmark of the vortex-blob hot path on B200: blob-velocity evaluations/s.

Workload (default): single large instance -- N = 2^20 blobs uniform in the
unit square (seeded), g ~ N(0,1)/N, sigma = 0.002; one step = the blob
velocity at every blob (FMM when built, else the direct sum; FP32-compensated)
plus one M4' remesh (h = 0.8 sigma).  evals/s = N / step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--method auto|fmm|direct]

One JSON line on rank 0.  Under torchrun every rank runs its own replica of
the workload (independent simulations, no collective: "replicas only");
value = sum over ranks of N / (max over ranks of the step time).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "phyflow2.0_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

L2_BYTES = 126 * 2 ** 20
MUFU_PER_SM_CLK = 16
MUFU_PER_INTERACTION = 2  # ex2 + rcp
FP32_PER_SM_CLK = 128
FP32_OPS_FULL, FP32_OPS_FAR = 14, 7  # FP32 lane ops of one pair: full / far (no ex2, one-float coordinates)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "sm_max_mhz": d.get("sm_max_mhz", 1965.0),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "source": "fallback"}


def profiled_traffic():
    """Per-launch DRAM bytes of kernels from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    return json.load(open(p)) if os.path.exists(p) else {}


# ---------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [c.strip() for c in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = [s for s in sm if s >= 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def gpu_id_for_smi(torch):
    try:
        u = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        return vis or "0"


# ---------------------------------------------------------------------------
N_DEFAULT = 1 << 20


def workload_c2(n=None):
    """C2 blobs; a smaller n (profiling cases) keeps sigma and the domain."""
    from pfblob import workloads as wl
    return wl.uniform_square(n=n or N_DEFAULT, sigma=0.002, overlap=0.8, config=2, instance=0)


def pick_method(arg):
    import pfblob
    if arg != "auto":
        return arg
    ok = True
    try:
        import torch
        x = torch.rand(64, dtype=torch.float64, device="cuda")
        v = torch.empty_like(x)
        pfblob.velocity_device(x, x, x, 1e-4, x, x, v, v, method=pfblob.FMM_METHOD, tol=1e-6)
        torch.cuda.synchronize()
    except Exception:
        ok = False
    return "fmm" if ok else "direct"


def reduce_max(value, dev, world):
    """Max over ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world):
    import torch
    import pfblob
    from pfblob import _lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    b = workload_c2(args.n)
    n = b.n
    method = pick_method(args.method)
    meth_id = pfblob.FMM_METHOD if method == "fmm" else pfblob.DIRECT_METHOD
    ks, xopt, cut = pfblob.fmm_parameters(b.sigma, b.k, tol=1e-6)
    xb, yb = b.bounds()
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x, y, g = T(b.x), T(b.y), T(b.g)
    vx = torch.empty(n, dtype=torch.float64, device=dev)
    vy = torch.empty_like(vx)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=meth_id, xopt=xopt, cutoff=cut,
                               tol=1e-6, ndirect=args.ndirect)
        if ev is not None:
            ev[1].record(stream)
        out = pfblob.remesh_device(x, y, g, b.h, xb[0], yb[0], 0.0, capacity=8 * n)
        if ev is not None:
            ev[2].record(stream)
        return out

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    nout = step()[0].numel()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    fmm_stats = []
    if method == "fmm":
        _lib.fmm_profile(True, dev.index)
    l0 = _lib.kernel_launches()
    with ClockSampler(gpu_id_for_smi(torch)) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush between timed steps (outside the events)
            step(evs[k])
            if method == "fmm":  # the remesh already synchronised the stream
                fmm_stats.append(_lib.fmm_last_stats(dev.index))
        torch.cuda.synchronize()
    launches = _lib.kernel_launches() - l0
    if method == "fmm":
        _lib.fmm_profile(False, dev.index)
    if world > 1:
        torch.distributed.barrier()
    vel_ms = [e[0].elapsed_time(e[1]) for e in evs]
    rm_ms = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = sum(vel_ms + rm_ms) / args.steps
    t_max = reduce_max(step_ms, dev, world)
    value = world * n / (t_max * 1e-3)

    # end to end through the public API with host (numpy) buffers
    e2e = None
    if not args.no_e2e:
        hx, hy, hg = b.x, b.y, b.g
        e2e_ms = []
        for k in range(max(2, min(args.steps, 5)) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ux, uy = pfblob.velocity(hx, hy, hg, b.sigma, k=b.k, hardware=1, method=meth_id,
                                     Ndirect=args.ndirect, tol=1e-6)
            rxn, ryn, rgn = pfblob.Regrid(hx, hy, hg, b.sigma, b.overlap, xb, yb)
            torch.cuda.synchronize()
            if k > 0:
                e2e_ms.append((time.perf_counter() - t0) * 1e3)
        em = reduce_max(statistics.median(e2e_ms), dev, world)
        e2e = {"value": world * n / (em * 1e-3), "unit": "evals/s", "ms_per_step": em,
               "h2d_bytes_per_step": 2 * 24 * n, "d2h_bytes_per_step": 16 * n + 24 * rxn.shape[0]}

    pk = peaks()
    vel_avg = statistics.mean(vel_ms)
    rm_avg = statistics.mean(rm_ms)
    traffic = profiled_traffic()
    if method == "direct":
        inter = float(n) * n
        ach = inter / (vel_avg * 1e-3)
        peak = (pk["sm_max_mhz"] * 1e6 * MUFU_PER_SM_CLK * torch.cuda.get_device_properties(dev)
                .multi_processor_count / MUFU_PER_INTERACTION)
        roof = {"bound": "mufu", "kernel": "k_direct_gauss", "achieved": ach / 1e9,
                "peak": peak / 1e9, "unit": "Ginteractions/s", "frac": ach / peak,
                "traffic": traffic.get("k_direct_gauss"),
                "peak_source": f"{MUFU_PER_SM_CLK} MUFU/SM/clk x SMs x sm_max_mhz "
                               f"({pk['source']}) / {MUFU_PER_INTERACTION} MUFU per interaction",
                "per_unit": "1 interaction = 2 MUFU (ex2, rcp) + 14 FP32 flops"}
    else:
        st0 = fmm_stats[-1]
        ms_p2p = statistics.mean(f["ms_p2p"] for f in fmm_stats)
        pairs = st0["p2p_pairs"]
        far = st0["p2p_pairs_far"]
        ach = pairs / (ms_p2p * 1e-3)
        # two-pipe roofline: the launch cannot beat the busier of the MUFU and
        # FP32 pipes; pairs in tiles beyond the Gaussian's reach skip the ex2
        sm_clk = pk["sm_max_mhz"] * 1e6 * torch.cuda.get_device_properties(dev).multi_processor_count
        t_mufu = (MUFU_PER_INTERACTION * pairs - far) / (MUFU_PER_SM_CLK * sm_clk)
        t_fp32 = (FP32_OPS_FULL * (pairs - far) + FP32_OPS_FAR * far) / (FP32_PER_SM_CLK * sm_clk)
        peak = pairs / max(t_mufu, t_fp32)
        roof = {"bound": "mufu" if t_mufu >= t_fp32 else "fp32", "kernel": "k_p2p (FMM near field)",
                "achieved": ach / 1e9, "peak": peak / 1e9, "unit": "Ginteractions/s",
                "frac": ach / peak, "traffic": traffic.get("k_p2p"), "pairs_per_launch": pairs,
                "pairs_far": far, "launch_ms": ms_p2p,
                "pipe_ms": {"mufu": t_mufu * 1e3, "fp32": t_fp32 * 1e3},
                "peak_source": f"pairs / max(MUFU ops / ({MUFU_PER_SM_CLK} MUFU/SM/clk), FP32 lane "
                               f"ops / ({FP32_PER_SM_CLK} FP32/SM/clk)) x SMs x sm_max_mhz "
                               f"({pk['source']})",
                "per_unit": f"pair within the Gaussian's reach: 2 MUFU (ex2, rcp) + {FP32_OPS_FULL} "
                            f"FP32 ops; pair with a source beyond it from the whole target group "
                            f"(pairs_far): 1 MUFU (rcp) + {FP32_OPS_FAR} FP32 ops"}
        npt = st0["expansion_terms"]
        ms_m2l = statistics.mean(f["ms_m2l"] for f in fmm_stats)
        m2l_flops = st0["m2l_translations"] * 8.0 * npt * npt
        fp64_peak = 148 * 64 * 2 * pk["sm_max_mhz"] * 1e6
        roof_m2l = {"bound": "fp64", "kernel": "k_m2l", "achieved": m2l_flops / (ms_m2l * 1e-3) / 1e12,
                    "peak": fp64_peak / 1e12, "unit": "TFLOP/s",
                    "frac": m2l_flops / (ms_m2l * 1e-3) / fp64_peak,
                    "per_unit": "8 (p+1)^2 FP64 flops per translation",
                    "translations": st0["m2l_translations"],
                    "peak_source": "148 SMs x 64 FP64 FMA/clk x 2 x sm_max_mhz (nominal)"}
        fmm_info = {"leaf_level": st0["leaf_level"], "expansion_terms": npt,
                    "block_level_drop": st0["block_level_drop"], "p2p_pairs": pairs,
                    "p2p_pairs_far": far,
                    "m2l_translations": st0["m2l_translations"],
                    "phase_ms": {k[3:]: statistics.mean(f[k] for f in fmm_stats)
                                 for k in ("ms_sort", "ms_upward", "ms_m2l", "ms_downward",
                                           "ms_p2p", "ms_l2p", "ms_total")},
                    "roofline_m2l": roof_m2l}
    alg_bytes = 24 * n + 24 * nout
    roof_rm = {"bound": "hbm", "kernel": "remesh (all passes)", "achieved": alg_bytes / (rm_avg * 1e-3) / 1e9,
               "peak": pk["hbm_gbs"], "unit": "GB/s",
               "frac": alg_bytes / (rm_avg * 1e-3) / 1e9 / pk["hbm_gbs"],
               "traffic": traffic.get("remesh"), "algorithmic_bytes": alg_bytes}
    line = {
        "metric": "blob velocity evals/s at <=1e-6 rel err vs FP64 (velocity + M4' remesh step)",
        "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-compensated velocity, f64 remesh",
        "data": "synthetic (seeded U[0,1)^2 blobs, g~N(0,1)/N)",
        "config": {"workload": f"single large instance: N={n} blobs U[0,1)^2, sigma=0.002, "
                               f"velocity at all blobs ({method}) + M4' remesh h=0.8 sigma",
                   "n_blobs": n, "method": method, "sigma": b.sigma, "n_out_remesh": nout,
                   "l2": "flushed between timed steps (256 MB write outside the step events)",
                   "parallelism": f"replicas x{world}"},
        "phase_ms": {"velocity": vel_avg, "remesh": rm_avg},
        "gpu_launches": launches, "roofline": roof, "roofline_remesh": roof_rm,
        "fmm": fmm_info if method == "fmm" else None,
        "clocks": clk.summary(), "e2e": e2e,
    }
    return line


# ---------------------------------------------------------------------------
# CPU side: the reference's own CPU code (oracle/_ref) on a bounded sample
def cpu_reference_step(method, rng_seed=0):
    """One bounded sample of the workload on the host with the reference's CPU
    implementation.  Returns (evals/s scaled to the full workload, description,
    threads)."""
    import oracle
    from oracle import ref
    b = workload_c2()
    threads = os.cpu_count() or 1
    if method == "direct":
        # 1/8 x 1/8 sub-square: same density; direct cost scales as N^2
        sel = (b.x < 0.125) & (b.y < 0.125)
        xs, ys, gs = b.x[sel], b.y[sel], b.g[sel]
        ns = xs.shape[0]
        t0 = time.perf_counter()
        if ref.available():
            ref.direct_gauss(xs, ys, gs, b.ksigmasqr)
            kind = "reference"
        else:
            oracle.velocity_direct(xs, ys, gs, b.ksigmasqr, nthreads=threads)
            kind = "port"
        tv = time.perf_counter() - t0
        rate = float(ns) * ns / tv  # interactions/s
        xb, yb = b.bounds()
        t0 = time.perf_counter()
        oracle.regrid(xs, ys, gs, b.sigma, b.overlap, xb, yb)
        tr = (time.perf_counter() - t0) / ns  # s per blob
        t_full = float(b.n) * b.n / rate + tr * b.n
        desc = (f"{ns} blobs of the 1/8 x 1/8 sub-square (same density): reference Cython direct "
                f"(OpenMP, {threads} threads) scaled to N^2 pairs + numpy/scipy Regrid per blob")
        return b.n / t_full, desc, threads, kind
    # FMM path: 1/4 x 1/4 sub-square, reference C++ FMM (single thread) + Regrid
    sel = (b.x < 0.25) & (b.y < 0.25)
    xs, ys, gs = b.x[sel], b.y[sel], b.g[sel]
    ns = xs.shape[0]
    t0 = time.perf_counter()
    if ref.available():
        ref.fmm_velocity(xs, ys, gs, b.sigma, k=b.k, tol=1e-6, ndirect=35)
        kind = "reference"
    else:
        oracle.velocity_direct(xs, ys, gs, b.ksigmasqr, nthreads=threads)
        kind = "port"
    xb, yb = b.bounds()
    oracle.regrid(xs, ys, gs, b.sigma, b.overlap, xb, yb)
    t = time.perf_counter() - t0
    desc = (f"{ns} blobs of the 1/4 x 1/4 sub-square (same density): reference C++ CPU FMM "
            f"(tol 1e-6, Ndirect 35, single-threaded as built) + numpy/scipy Regrid")
    return ns / t, desc, (1 if kind == "reference" else threads), kind


def run_reference(args):
    method = "fmm" if args.method in ("auto", "fmm") else "direct"
    for _ in range(args.warmup):
        cpu_reference_step(method)
    vals = []
    desc = threads = kind = None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, desc, threads, kind = cpu_reference_step(method)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    n = 1 << 20
    return {
        "impl": "reference",
        "metric": "blob velocity evals/s at <=1e-6 rel err vs FP64 (velocity + M4' remesh step)",
        "value": value, "unit": "evals/s", "n_gpus": args.gpus, "device": "host cores",
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": n / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"single large instance: N={n} blobs U[0,1)^2, sigma=0.002, "
                               f"velocity at all blobs ({method}) + M4' remesh h=0.8 sigma",
                   "n_blobs": n, "method": method},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }


# ---------------------------------------------------------------------------
# Batched (config 4) and served (config 5) sections: same metric, many blob sets
def _sims_on_device(sizes, config, dev):
    import torch
    from pfblob import workloads as wl
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = []
    for i, n in enumerate(sizes):
        b = wl.mixed_instance(int(n), config=config, instance=i)
        out.append((b, T(b.x), T(b.y), T(b.g)))
    return out


def run_batched(dev, n_sims=256, steps=5):
    """256 simulations, N log-uniform in [2048, 262144]: one CUDA-graph launch
    per step vs one simulation per launch sequence (same methods and trees)."""
    import torch
    import pfblob
    from pfblob import _lib, workloads as wl
    from pfblob.batch import Batch
    from pfblob.tune import Tuner
    sizes = wl.log_uniform_sizes(n_sims, 2048, 262144, config=4)
    sims = _sims_on_device(sizes, 4, dev)
    tun = Tuner(dev.index)
    tun.calibrate(save=False)
    bt = Batch([{"x": x, "y": y, "g": g, "sigma": b.sigma} for b, x, y, g in sims], tol=1e-6,
               n_streams=8, tuner=tun)
    for _ in range(3):
        bt.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tb = []
    for _ in range(steps):
        e0.record()
        bt.run()
        e1.record()
        torch.cuda.synchronize()
        tb.append(e0.elapsed_time(e1))
    res = bt.results()
    ntot = int(sizes.sum())

    def plain_step():
        for (b, x, y, g), r in zip(sims, bt.sims):
            ks, xo, cut = pfblob.fmm_parameters(b.sigma)
            if r["method"] == 0:
                _lib.fmm_set_tuning(r["leaf_level"], 0, 1)
            pfblob.velocity_device(x, y, g, ks, x, y, r["vx"], r["vy"], method=r["method"],
                                   xopt=xo, cutoff=cut, tol=1e-6)
            xb, yb = b.bounds()
            pfblob.remesh_device(x, y, g, b.h, xb[0], yb[0])
        _lib.fmm_set_tuning(0, 0, 1)

    plain_step()
    torch.cuda.synchronize()
    tp = []
    for _ in range(3):
        t0 = time.perf_counter()
        plain_step()
        torch.cuda.synchronize()
        tp.append((time.perf_counter() - t0) * 1e3)
    out = {"workload": f"{n_sims} simulations, N log-uniform [2048, 262144] (sum {ntot}), "
                       "Lamb-Oseen + uniform mix in [-1,1]^2, sigma U[0.002, 0.01]; "
                       "velocity (autotuned direct/FMM) + M4' remesh per simulation",
           "n_blobs": ntot, "batched_ms": statistics.median(tb),
           "batched_evals_per_s": ntot / (statistics.median(tb) * 1e-3),
           "plain_ms": statistics.median(tp), "plain_evals_per_s": ntot / (statistics.median(tp) * 1e-3),
           "ratio": statistics.median(tp) / statistics.median(tb),
           "n_direct": sum(1 for r in res if r["method"] == 1),
           "n_fmm": sum(1 for r in res if r["method"] == 0), "graph_kernel_nodes": bt.kernel_nodes,
           "launches_per_step": 1}
    bt.close()
    return out


def run_served(dev, n_sims=1024, n_req=400, rates=(100, 1000, 5000), slots=8):
    """1024 resident simulations, N log-uniform in [1024, 2^20]; Poisson arrivals
    of velocity+remesh requests; continuous batching over `slots` worker streams
    vs one request at a time."""
    from pfblob import workloads as wl
    from pfblob.serve import Server, Simulation, poisson_trace, summarize
    sizes = wl.log_uniform_sizes(n_sims, 1024, 1 << 20, config=5)
    sims = [Simulation(x, y, g, sigma=b.sigma) for b, x, y, g in _sims_on_device(sizes, 5, dev)]
    out = {"workload": f"{n_sims} resident simulations, N log-uniform [1024, 1048576] "
                       f"(sum {int(sizes.sum())}); Poisson arrivals, {n_req} requests per rate",
           "slots": slots, "rates": {}}
    srv = Server(sims, n_slots=slots)
    srv.warmup()
    for rate in rates:
        out["rates"][str(rate)] = summarize(srv.run_trace(poisson_trace(n_req, rate, n_sims, seed=rate)))
    srv.close()
    one = Server(sims, n_slots=1)
    one.warmup(every_sim=False)
    sat = max(rates)
    out["plain_one_at_a_time"] = summarize(one.run_trace(poisson_trace(n_req, sat, n_sims, seed=sat)))
    one.close()
    out["ratio_at_saturation"] = (out["rates"][str(sat)]["evals_per_s"] /
                                  out["plain_one_at_a_time"]["evals_per_s"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="auto", choices=["auto", "fmm", "direct"])
    ap.add_argument("--ndirect", type=int, default=35)
    ap.add_argument("--n", type=int, default=None,
                    help="blob count (default 2^20; smaller only for profiling captures)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (256 simulations) and served (1024 simulations) sections")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    import torch
    if world > 1:
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_ours(args, rank, world)
    if rank == 0 and world == 1 and not args.no_extras and args.n is None:
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        line["batched"] = run_batched(dev)
        line["served"] = run_served(dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, desc, threads, kind = cpu_reference_step(line["config"]["method"])
        line["cpu_baseline"] = {"value": v, "unit": "evals/s", "cores": threads, "kind": kind,
                                "sample": desc}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
