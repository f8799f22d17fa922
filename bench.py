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


def workloads():
    """The seeded generators (pfblob/workloads.py), loaded by file so that the
    reference arm never imports pfblob (whose import loads libpfblob.so)."""
    import importlib.util
    name = "pfblob_workloads_file"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(ROOT, "phyflow2.0_b200", "pfblob", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


def workload_c2(n=None):
    """C2 blobs; a smaller n (profiling cases) keeps sigma and the domain."""
    return workloads().uniform_square(n=n or N_DEFAULT, sigma=0.002, overlap=0.8, config=2,
                                      instance=0)


METRIC = "blob velocity evals/s at <=1e-6 rel err vs FP64 (velocity + M4' remesh step)"


def workload_config(n, method, sigma, world):
    """The config object both arms print (identical for the same workload)."""
    return {"workload": f"single large instance: N={n} blobs U[0,1)^2, sigma=0.002, "
                        f"velocity at all blobs ({method}) + M4' remesh h=0.8 sigma",
            "n_blobs": n, "method": method, "sigma": sigma,
            "l2": "GPU arm: L2 flushed between timed steps (256 MB write outside the step "
                  "events); the step's inputs are 24 MB",
            "parallelism": f"replicas x{world}"}


def host_info():
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count() or 1, "cpu_model": model}


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
    from pfblob.regrid import remesh_device_async

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
    # the remesh scratch bound of a resident blob set: its previous window
    # plus 25% (found by the first warm-up step)
    mb = [max(4 * n, 4096)]

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=meth_id, xopt=xopt, cutoff=cut,
                               tol=1e-6, ndirect=args.ndirect)
        if ev is not None:
            ev[1].record(stream)
        out = remesh_device_async(x, y, g, b.h, xb[0], yb[0], 0.0, max_base_cells=mb[0],
                                  with_indices=True)
        if ev is not None:
            ev[2].record(stream)
        return out

    def settle(out):
        """Host side of a step's remesh, after the device work: the output
        count, the status word (8 = window beyond the bound: raise it), the
        window."""
        k, st_, w = int(out[5].item()), int(out[6].item()), out[7].cpu().tolist()
        if st_ & 8:
            mb[0] = int(w[2] * w[3] * 5 // 4) + 1
        elif st_:
            raise RuntimeError(f"remesh status {st_}")
        return k, st_, w

    for _ in range(args.warmup):
        o = step()
        settle(o)
        w = o[7].cpu().tolist()
        mb[0] = int(w[2] * w[3] * 5 // 4) + 1
    torch.cuda.synchronize()
    last = step()
    nout, _, win = settle(last)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # eager pass: the step issued call by call (velocity_device, which finds
    # the tree box on the device and reads it back, then remesh_device_async),
    # with events between the two calls and the FMM's own phase events; it
    # gives the phase split and the kernel rooflines
    fmm_stats = []
    if method == "fmm":
        _lib.fmm_profile(True, dev.index)
    l0 = _lib.kernel_launches()
    outs = []
    for k in range(args.steps):
        flush.fill_(float(k))  # L2 flush between timed steps (outside the events)
        # keep only the step's small status tensors: the output blobs are
        # released, so the allocator reuses their blocks step after step
        outs.append(step(evs[k])[5:8])
        if method == "fmm":  # reads the FMM's events: synchronises after the step
            fmm_stats.append(_lib.fmm_last_stats(dev.index))
    torch.cuda.synchronize()
    eager_launches = _lib.kernel_launches() - l0
    if method == "fmm":
        _lib.fmm_profile(False, dev.index)
    for o in outs:  # every timed step completed its remesh on the first try
        kk, st_ = int(o[0].item()), int(o[1].item())
        assert st_ == 0 and kk == nout, (kk, st_, nout)
    vel_ms = [e[0].elapsed_time(e[1]) for e in evs]
    rm_ms = [e[1].elapsed_time(e[2]) for e in evs]
    eager_ms = sum(vel_ms + rm_ms) / args.steps
    last = step()  # the eager step's results (with indices) for the check
    torch.cuda.synchronize()

    # the headline: the same step as ONE graph launch (pfblob.StepGraph, the
    # captured pf_blob_step: FMM on the set's bounding box, remesh with its
    # window found on the device), inputs resident, L2 flushed between steps
    box = (float(b.x.min()), float(b.x.max()), float(b.y.min()), float(b.y.max()))
    sg = pfblob.StepGraph(x, y, g, ks, xopt, cut, 1e-6, box, b.h, xb[0], yb[0], 0.0,
                          method=meth_id, max_base_cells=mb[0])
    for _ in range(3):
        sg.launch()
    torch.cuda.synchronize()
    gev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    chk = torch.zeros((args.steps, 2), dtype=torch.int64, device=dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = _lib.kernel_launches()
    with ClockSampler(gpu_id_for_smi(torch)) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush between timed steps (outside the events)
            gev[k][0].record(stream)
            sg.launch(stream.cuda_stream)
            gev[k][1].record(stream)
            chk[k, 0].copy_(sg.n_out[0])  # outside the events
            chk[k, 1].copy_(sg.status[0])
        torch.cuda.synchronize()
    launches = _lib.kernel_launches() - l0
    for kk, st_ in chk.cpu().tolist():
        assert st_ == 0 and kk == nout, (kk, st_, nout)
    if world > 1:
        torch.distributed.barrier()
    graph_ms = [e[0].elapsed_time(e[1]) for e in gev]
    step_ms = sum(graph_ms) / args.steps
    t_max = reduce_max(step_ms, dev, world)
    value = world * n / (t_max * 1e-3)
    graph_info = {"kernels_per_launch": sg.kernels,
                  "ms_per_step_median": statistics.median(graph_ms),
                  "equals_eager_bitwise": bool(
                      torch.equal(sg.vx, vx) and torch.equal(sg.vy, vy) and
                      all(torch.equal(sg.out[i, :nout], last[i][:nout]) for i in range(3)))}
    eager_info = {"ms_per_step": eager_ms, "value": world * n / (reduce_max(eager_ms, dev, world)
                                                                  * 1e-3),
                  "gpu_launches": eager_launches,
                  "issue": "velocity_device (tree box found on the device and read back) then "
                           "remesh_device_async, kernel by kernel"}

    # end to end through the public API with host (numpy) buffers: one upload
    # of x, y, g, velocity and remesh, results read back
    e2e = None
    if not args.no_e2e:
        # the step's inputs in pinned host memory (as a caller staging them)
        hx, hy, hg = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                      for a in (b.x, b.y, b.g))
        e2e_ms = []
        for k in range(max(2, min(args.steps, 5)) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ux, uy, rxn, ryn, rgn = pfblob.velocity_and_regrid(
                hx, hy, hg, b.sigma, b.overlap, xb, yb, k=b.k, method=meth_id,
                Ndirect=args.ndirect, tol=1e-6)
            torch.cuda.synchronize()
            if k > 0:
                e2e_ms.append((time.perf_counter() - t0) * 1e3)
        em = reduce_max(statistics.median(e2e_ms), dev, world)
        e2e = {"value": world * n / (em * 1e-3), "unit": "evals/s", "ms_per_step": em,
               "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 16 * n + 24 * rxn.shape[0],
               "api": "pfblob.velocity_and_regrid (pinned host tensors in, numpy out)"}

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
        fmm_info = None
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
        # executed FP64 work of one translation: the real binomial matrix times
        # the complex vector (4 (p+1)^2, on the FP64 tensor cores) and the
        # scalings by the operator's powers before and after (16 (p+1))
        m2l_flops = st0["m2l_translations"] * (4.0 * npt * npt + 16.0 * npt)
        fp64_peak = 148 * 64 * 2 * pk["sm_max_mhz"] * 1e6
        roof_m2l = {"bound": "fp64", "kernel": "k_m2l", "achieved": m2l_flops / (ms_m2l * 1e-3) / 1e12,
                    "peak": fp64_peak / 1e12, "unit": "TFLOP/s",
                    "frac": m2l_flops / (ms_m2l * 1e-3) / fp64_peak,
                    "per_unit": "4 (p+1)^2 + 16 (p+1) FP64 flops per translation (real binomial "
                                "matrix x complex vector on the FP64 tensor cores, scalings by the "
                                "operator's powers)",
                    "translations": st0["m2l_translations"],
                    "peak_source": "148 SMs x 64 FP64 FMA/clk x 2 x sm_max_mhz (nominal; the FP64 "
                                   "tensor-core rate is the same)"}
        fmm_info = {"leaf_level": st0["leaf_level"], "expansion_terms": npt,
                    "block_level_drop": st0["block_level_drop"], "p2p_pairs": pairs,
                    "p2p_pairs_far": far,
                    "m2l_translations": st0["m2l_translations"],
                    "phase_ms": {k[3:]: statistics.mean(f[k] for f in fmm_stats)
                                 for k in ("ms_sort", "ms_upward", "ms_m2l", "ms_downward",
                                           "ms_p2p", "ms_l2p", "ms_total")},
                    "roofline_m2l": roof_m2l}
    alg_bytes = 24 * n + 24 * nout
    roof_rm = {"bound": "hbm", "kernel": "remesh (all passes, pf_remesh_async)",
               "achieved": alg_bytes / (rm_avg * 1e-3) / 1e9, "peak": pk["hbm_gbs"], "unit": "GB/s",
               "frac": alg_bytes / (rm_avg * 1e-3) / 1e9 / pk["hbm_gbs"],
               "traffic": traffic.get("remesh"), "algorithmic_bytes": alg_bytes,
               "per_unit": "24 B per input blob (x, y, g read) + 24 B per output blob (x, y, g "
                           "written)"}
    cfg = workload_config(n, method, b.sigma, world)
    cfg["n_out_remesh"] = nout
    line = {
        "metric": METRIC,
        "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-compensated velocity, f64 remesh",
        "data": "synthetic (seeded U[0,1)^2 blobs, g~N(0,1)/N)",
        "config": cfg,
        "phase_ms": {"velocity": vel_avg, "remesh": rm_avg,
                     "velocity_median": statistics.median(vel_ms),
                     "remesh_median": statistics.median(rm_ms), "remesh_max": max(rm_ms)},
        "gpu_launches": launches, "roofline": roof, "roofline_remesh": roof_rm,
        "fmm": fmm_info,
        "clocks": clk.summary(), "e2e": e2e,
        "step_issue": "one CUDA graph launch per step (pfblob.StepGraph: pf_blob_step "
                      "captured; FMM on the set's bounding box, remesh window found on the "
                      "device); phase_ms and the rooflines are from the eager pass",
        "graph": graph_info, "eager": eager_info,
    }
    if rank == 0 and not args.no_check:
        line["err_vs_fp64"] = check_step(
            b, sg.vx, sg.vy, (sg.out[0], sg.out[1], sg.out[2], last[3], last[4]), nout)
        line["err_vs_fp64"]["checked"] = ("the graph's velocity and new blobs (their lattice "
                                          "indices from the eager step, which the graph equals "
                                          "bitwise)")
    sg.close()
    return line


def check_step(b, vx, vy, out, nout, n_targets=4096):
    """Accuracy of the timed step's results, outside the timed region: the
    velocity against the FP64 oracle direct sum on a seeded subset of targets
    (normwise: max |dv| / max |v_ref|), the remesh against the oracle Regrid
    (indices and coordinates bit-exact, values normwise), and conservation."""
    import oracle
    t0 = time.perf_counter()
    rng = np.random.default_rng(20261203)
    sub = np.sort(rng.choice(b.n, size=min(n_targets, b.n), replace=False))
    rx, ry = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, b.x[sub].copy(), b.y[sub].copy(),
                                    nthreads=os.cpu_count() or 1)
    gx, gy = vx.cpu().numpy()[sub], vy.cpu().numpy()[sub]
    d = np.sqrt((gx - rx) ** 2 + (gy - ry) ** 2)
    vref = np.sqrt(rx ** 2 + ry ** 2)
    strong = vref >= 1e-3 * vref.max()
    xb, yb = b.bounds()
    ox, oy, og, oix, oiy = oracle.regrid(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
    k = nout
    rx_, ry_, rg_, rix, riy = (t[:k].cpu().numpy() for t in out[:5])
    m0 = oracle.moments(b.x, b.y, b.g)
    m1 = oracle.moments(rx_, ry_, rg_)
    xs = float(max(np.abs(b.x).max(), np.abs(b.y).max()))
    return {"velocity_normwise": float(d.max() / vref.max()),
            "velocity_pointwise_max": float((d[strong] / vref[strong]).max()),
            "targets": int(sub.size), "gate": 1e-6,
            "remesh_indices_bit_exact": bool(k == oix.size and np.array_equal(rix, oix)
                                             and np.array_equal(riy, oiy)),
            "remesh_coords_bit_exact": bool(k == ox.size and np.array_equal(rx_, ox)
                                            and np.array_equal(ry_, oy)),
            "remesh_values_normwise": float(np.abs(rg_ - og).max() / np.abs(og).max())
            if k == og.size else None,
            "circulation": float(abs(m1[0] - m0[0]) / m0[3]),
            "linear_impulse": float(max(abs(m1[1] - m0[1]), abs(m1[2] - m0[2])) / (m0[3] * xs)),
            "oracle": "FP64 direct Gauss sum (C restatement of vv2parGauss) on a seeded target "
                      "subset; numpy/scipy Regrid restatement",
            "check_s": time.perf_counter() - t0}


# ---------------------------------------------------------------------------
# CPU side: the reference's own CPU code (oracle/_ref) on the same workload.
# The reference FMM (fmm2dInteract, fmm.cpp:88-304) is single-threaded as
# built; its API takes targets apart from sources, so each host process runs
# it with all sources on a contiguous share of the targets, and the Regrid
# (numpy + scipy restatement of _regridding.py:107-222, pinned bit-exact to
# the reference's own function) runs in the parent meanwhile.
_REF_STATE = {}


def _ref_worker_init(x, y, g, sigma, k):
    from oracle import ref
    _REF_STATE.update(x=x, y=y, g=g, sigma=sigma, k=k, ref=ref)


def _ref_worker_chunk(lohi):
    lo, hi = lohi
    st = _REF_STATE
    vx, vy = st["ref"].fmm_velocity(st["x"], st["y"], st["g"], st["sigma"], k=st["k"],
                                    xt=st["x"][lo:hi].copy(), yt=st["y"][lo:hi].copy(),
                                    tol=1e-6, ndirect=35)
    return lo, vx, vy


class ReferenceStep:
    """One step of the workload on the host with the reference's CPU code:
    FMM velocity at every blob + Regrid of every blob."""

    def __init__(self, b, procs=None):
        import multiprocessing as mp
        from oracle import ref
        self.b = b
        self.kind = "reference" if ref.available() else "port"
        self.procs = procs or max(1, min(os.cpu_count() or 1, 64))
        self.pool = None
        if self.kind == "reference":
            ctx = mp.get_context("spawn")  # no fork of a process that may hold a GPU context
            self.pool = ctx.Pool(self.procs, initializer=_ref_worker_init,
                                 initargs=(b.x, b.y, b.g, b.sigma, b.k))
        edges = np.linspace(0, b.n, self.procs + 1).astype(np.int64)
        self.chunks = [(int(edges[i]), int(edges[i + 1])) for i in range(self.procs)]

    def run(self):
        import oracle
        b = self.b
        xb, yb = b.bounds()
        vx = np.empty(b.n)
        vy = np.empty(b.n)
        if self.pool is not None:
            pending = self.pool.map_async(_ref_worker_chunk, self.chunks)
            rx, ry, rg, _, _ = oracle.regrid(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
            for lo, cx, cy in pending.get():
                vx[lo:lo + cx.shape[0]] = cx
                vy[lo:lo + cy.shape[0]] = cy
        else:  # reference not compiled here: the oracle port, all cores
            vx, vy = oracle.velocity_direct(b.x, b.y, b.g, b.ksigmasqr, nthreads=self.procs)
            rx, ry, rg, _, _ = oracle.regrid(b.x, b.y, b.g, b.sigma, b.overlap, xb, yb)
        return vx, vy, rx.shape[0]

    def describe(self):
        hi = host_info()
        if self.kind == "reference":
            what = (f"reference C++ CPU FMM (tol 1e-6, Ndirect 35; single-threaded as built) on "
                    f"all {self.b.n} blobs as sources, targets split over {self.procs} host "
                    f"processes, + numpy/scipy Regrid of all blobs in the parent meanwhile")
        else:
            what = (f"oracle FP64 direct sum ({self.procs} threads) + numpy/scipy Regrid, all "
                    f"{self.b.n} blobs")
        return f"full workload every step: {what}; host {hi['nproc']} x {hi['cpu_model']}"

    def close(self):
        if self.pool is not None:
            self.pool.close()
            self.pool.join()


def run_reference(args):
    b = workload_c2(args.n)
    rs = ReferenceStep(b)
    try:
        nout = None
        for _ in range(args.warmup):
            _, _, nout = rs.run()
        times = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            t1 = time.perf_counter()
            _, _, nout = rs.run()
            times.append(time.perf_counter() - t1)
        wall = time.perf_counter() - t0
    finally:
        rs.close()
    ms = statistics.mean(times) * 1e3
    value = b.n / (ms * 1e-3)
    cfg = workload_config(b.n, "fmm", b.sigma, args.gpus)
    cfg["n_out_remesh"] = nout
    hi = host_info()
    return {
        "impl": "reference", "metric": METRIC,
        "value": value, "unit": "evals/s", "n_gpus": args.gpus, "device": "host cores",
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded U[0,1)^2 "
        "blobs, g~N(0,1)/N)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": rs.procs, "kind": rs.kind,
                         "sample": rs.describe(), "nproc": hi["nproc"], "cpu_model": hi["cpu_model"]},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }


def kernel_baselines():
    """The reference's compiled Cython kernels on this host's cores (OpenMP,
    every host thread): the direct Gauss sum on the C1 Lamb-Oseen lattice
    (10,000 blobs, all 1e8 pairs) and the vortex-panel velocity on 16,384
    seeded points of the near-wall set x 512 panels.  Pairs per second."""
    from oracle import ref
    if not ref.available():
        return None
    wl = workloads()
    out = {"threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))}
    c1 = wl.lamb_oseen_lattice()
    ref.direct_gauss(c1.x[:64], c1.y[:64], c1.g[:64], c1.ksigmasqr)  # load the module
    t0 = time.perf_counter()
    ref.direct_gauss(c1.x, c1.y, c1.g, c1.ksigmasqr)
    t = time.perf_counter() - t0
    out["direct_c1"] = {"pairs_per_s": float(c1.n) ** 2 / t, "ms": t * 1e3, "n": c1.n,
                        "kernel": "vv2parGauss_Cython_cpu (reference Cython, OpenMP)"}
    sl = wl.shear_layer(n=1 << 22)
    ps = wl.cylinder_panels(512)
    idx = np.sort(np.random.default_rng(7).choice(sl.n, 16384, replace=False))
    args = (ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina)
    ref.panel_velocity(*args, sl.x[idx[:64]], sl.y[idx[:64]])
    t0 = time.perf_counter()
    ref.panel_velocity(*args, sl.x[idx], sl.y[idx])
    t = time.perf_counter() - t0
    out["panels_c3_sample"] = {"pairs_per_s": 16384 * 512 / t, "ms": t * 1e3, "points": 16384,
                               "panels": 512,
                               "kernel": "_vortexPanel_Cython_cpu.inducedVelocity (reference Cython)"}
    return out


def cpu_baseline(n=None):
    """One full step of the reference's CPU path on this host (rank 0, N=1),
    plus the reference's Cython direct and panel kernels on their own."""
    b = workload_c2(n)
    rs = ReferenceStep(b)
    try:
        t0 = time.perf_counter()
        rs.run()
        t = time.perf_counter() - t0
    finally:
        rs.close()
    hi = host_info()
    return {"value": b.n / t, "unit": "evals/s", "cores": rs.procs, "kind": rs.kind,
            "sample": "one step, " + rs.describe(), "ms_per_step": t * 1e3, "nproc": hi["nproc"],
            "cpu_model": hi["cpu_model"], "kernels": kernel_baselines()}


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


def run_batched(dev, n_sims=256, steps=5, n_streams=8):
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
               n_streams=n_streams, tuner=tun)
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


def run_c3(dev, n=1 << 22, steps=5, warmup=2):
    """The near-wall shear-layer configuration at its stated size: N = 2^22
    blobs (n) in the annulus 1 <= r <= 1.5 plus 512 vortex panels on the unit
    circle.  One step = FMM blob velocity + panel velocity added on top + the
    M4' remesh (window found on the device).  CUDA events per phase."""
    import torch
    import pfblob
    from pfblob import _lib
    from pfblob.regrid import remesh_device_async
    wl = workloads()
    b = wl.shear_layer(n=n)
    ps = wl.cylinder_panels(512)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x, y, g = T(b.x), T(b.y), T(b.g)
    pan = [T(a) for a in (ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina)]
    vx, vy = torch.empty_like(x), torch.empty_like(x)
    ks, xo, cut = pfblob.fmm_parameters(b.sigma)
    xb, yb = b.bounds()
    mb = int((3.1 / b.h) ** 2)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)

    def step(ev=None):
        if ev:
            ev[0].record(st)
        pfblob.velocity_device(x, y, g, ks, x, y, vx, vy, method=pfblob.FMM_METHOD, xopt=xo,
                               cutoff=cut)
        if ev:
            ev[1].record(st)
        pfblob.panel_velocity_device(*pan, x, y, vx, vy, accumulate=True)
        if ev:
            ev[2].record(st)
        out = remesh_device_async(x, y, g, b.h, xb[0], yb[0], max_base_cells=mb)
        if ev:
            ev[3].record(st)
        return out

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    _lib.fmm_profile(True, dev.index)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    stats, out = [], None
    for k in range(steps):
        flush.fill_(float(k))
        # the previous step's outputs are released first, so the allocator
        # reuses their blocks (no device allocation inside the timed steps)
        out = None
        out = step(evs[k])
        stats.append(_lib.fmm_last_stats(dev.index))
    torch.cuda.synchronize(dev)
    _lib.fmm_profile(False, dev.index)
    outs = [out]
    ph = {name: statistics.mean(e[i].elapsed_time(e[i + 1]) for e in evs)
          for i, name in enumerate(("fmm", "panels", "remesh"))}
    ms = sum(ph.values())
    st0 = stats[-1]
    ms_p2p = statistics.mean(f["ms_p2p"] for f in stats)
    pk = peaks()
    sm_clk = pk["sm_max_mhz"] * 1e6 * torch.cuda.get_device_properties(dev).multi_processor_count
    pairs, far = st0["p2p_pairs"], st0["p2p_pairs_far"]
    t_mufu = (MUFU_PER_INTERACTION * pairs - far) / (MUFU_PER_SM_CLK * sm_clk)
    t_fp32 = (FP32_OPS_FULL * (pairs - far) + FP32_OPS_FAR * far) / (FP32_PER_SM_CLK * sm_clk)
    ppairs = 512.0 * b.n
    k_out, status = int(outs[-1][3].item()), int(outs[-1][4].item())
    mom = outs[-1][6].cpu().numpy()
    circ, imp = pfblob.conservation_error(mom[:4], mom[4:], float(np.abs(b.x).max()))
    rm_bytes = 24 * b.n + 24 * k_out
    return {"workload": f"near-wall shear layer: N={b.n} blobs in 1<=r<=1.5 (h={b.h:.4e}, "
                        "sigma=h/0.8), 512 vortex panels on the unit circle; FMM blob velocity + "
                        "panel velocity + M4' remesh per step",
            "n_blobs": b.n, "ms_per_step": ms, "evals_per_s": b.n / (ms * 1e-3), "phase_ms": ph,
            "roofline_p2p": {"achieved": pairs / (ms_p2p * 1e-3) / 1e9,
                             "peak": pairs / max(t_mufu, t_fp32) / 1e9, "unit": "Ginteractions/s",
                             "frac": max(t_mufu, t_fp32) / (ms_p2p * 1e-3), "pairs": pairs,
                             "pairs_far": far, "launch_ms": ms_p2p},
            "panel_pairs_per_s": ppairs / (ph["panels"] * 1e-3),
            "remesh": {"n_out": k_out, "status": status, "circulation": circ,
                       "linear_impulse": imp},
            "roofline_remesh": {"bound": "hbm", "achieved": rm_bytes / (ph["remesh"] * 1e-3) / 1e9,
                                "peak": pk["hbm_gbs"], "unit": "GB/s",
                                "frac": rm_bytes / (ph["remesh"] * 1e-3) / 1e9 / pk["hbm_gbs"],
                                "algorithmic_bytes": rm_bytes,
                                "per_unit": "24 B per input blob + 24 B per output blob"},
            "l2": "flushed between timed steps"}


def run_c1(dev, steps=20, warmup=3):
    """The reference's CPU-runnable configuration: the 100 x 100 Lamb-Oseen
    lattice (N = 10,000, h = 0.02), direct-sum velocity at every blob and one
    M4' remesh, timed per phase with CUDA events on inputs already on the GPU."""
    import torch
    import pfblob
    from pfblob.regrid import remesh_device_async
    b = workloads().lamb_oseen_lattice()
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x, y, g = T(b.x), T(b.y), T(b.g)
    vx, vy = torch.empty_like(x), torch.empty_like(x)
    xb, yb = b.bounds()
    st = torch.cuda.current_stream(dev)
    mb = max(4 * b.n, 4096)

    def step(ev=None):
        if ev:
            ev[0].record(st)
        pfblob.velocity_device(x, y, g, b.ksigmasqr, x, y, vx, vy, method=pfblob.DIRECT_METHOD)
        if ev:
            ev[1].record(st)
        out = remesh_device_async(x, y, g, b.h, xb[0], yb[0], max_base_cells=mb)
        if ev:
            ev[2].record(st)
        return out

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    out = None
    for k in range(steps):
        out = None
        out = step(evs[k])
    torch.cuda.synchronize(dev)
    vel = statistics.median(e[0].elapsed_time(e[1]) for e in evs)
    rm = statistics.median(e[1].elapsed_time(e[2]) for e in evs)
    # the same step captured once (pfblob.StepGraph) and replayed
    box = (float(b.x.min()), float(b.x.max()), float(b.y.min()), float(b.y.max()))
    sg = pfblob.StepGraph(x, y, g, b.ksigmasqr, 0.0, 0.0, 1e-6, box, b.h, xb[0], yb[0],
                          method=pfblob.DIRECT_METHOD, max_base_cells=mb)
    for _ in range(warmup):
        sg.launch()
    gev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    torch.cuda.synchronize(dev)
    for e in gev:
        e[0].record(st)
        sg.launch()
        e[1].record(st)
    torch.cuda.synchronize(dev)
    gms = statistics.median(e[0].elapsed_time(e[1]) for e in gev)
    k = int(out[3].item())
    same = (torch.equal(sg.vx, vx) and torch.equal(sg.vy, vy) and int(sg.n_out.item()) == k
            and torch.equal(sg.out[2, :k], out[2][:k]))
    graph = {"ms_per_step": gms, "kernels_per_launch": sg.kernels, "equals_eager_bitwise": same}
    sg.close()
    return {"workload": "C1 Lamb-Oseen lattice: N=10000 (h=0.02, sigma=h/0.8), direct velocity at "
                        "every blob + M4' remesh", "n_blobs": b.n, "ms_per_step": vel + rm,
            "phase_ms": {"velocity": vel, "remesh": rm},
            "direct_pairs_per_s": float(b.n) ** 2 / (vel * 1e-3),
            "n_out": k, "status": int(out[4].item()), "graph": graph,
            "timing": "medians of CUDA-event phases; inputs resident, L2 not flushed (the set is "
                      "0.24 MB); graph: the step as one StepGraph launch, median of its launches"}


def run_evolve(dev, steps=10, warmup=2):
    """A moving blob set: ``Blobs.evolve`` on the C2 blobs (forward-Euler
    convection by the FMM velocity, redistribution and population control
    every step, as the reference's defaults do; a free stream moves the set),
    so the FMM box and the remesh window drift every step.  Reports the step
    time and the FMM plans built per step after warm-up."""
    import torch
    import pfblob
    from pfblob import _lib
    b = workload_c2()
    bl = pfblob.Blobs((b.x, b.y, b.g), vInf=[0.3, -0.2], nu=0.0, deltaTc=1e-3, h=b.h,
                      overlap=b.overlap, timeIntegrationParams={'method': 'euler'},
                      velocityComputationParams={'method': 'fmm', 'hardware': 'gpu'},
                      device=dev.index)
    for _ in range(warmup):
        bl.evolve()
    torch.cuda.synchronize(dev)
    n0 = bl.numBlobs
    p0 = _lib.fmm_plan_builds()
    t0 = time.perf_counter()
    for _ in range(steps):
        bl.evolve()
    torch.cuda.synchronize(dev)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    return {"workload": "Blobs.evolve of the C2 set after construction-time redistribution "
                        f"({n0} lattice blobs): FE convection (FMM velocity, free stream (0.3, -0.2), "
                        "dt 1e-3) + redistribution + population control every step",
            "n_blobs": int(n0), "ms_per_step": ms, "evals_per_s": n0 / (ms * 1e-3),
            "plan_builds_per_step": (_lib.fmm_plan_builds() - p0) / steps, "steps": steps,
            "timing": "host wall clock around evolve(), synchronised (evolve reads counts back)"}


def run_served(dev, n_sims=1024, n_req=400, rates=(100, 1000, 5000), slots=8):
    """1024 resident simulations, N log-uniform in [1024, 2^20]; Poisson arrivals
    of velocity+remesh requests; continuous batching over `slots` worker streams
    vs one request at a time."""
    import torch
    from pfblob import workloads as wl
    from pfblob.serve import Server, Simulation, conservation, poisson_trace, summarize
    sizes = wl.log_uniform_sizes(n_sims, 1024, 1 << 20, config=5)
    sims = [Simulation(x, y, g, sigma=b.sigma) for b, x, y, g in _sims_on_device(sizes, 5, dev)]
    out = {"workload": f"{n_sims} resident simulations, N log-uniform [1024, 1048576] "
                       f"(sum {int(sizes.sum())}); Poisson arrivals, {n_req} requests per rate",
           "slots": slots, "rates": {}}
    sat = max(rates)
    srv = Server(sims, n_slots=slots)
    srv.warmup()
    worst = {"circulation": 0.0, "linear_impulse": 0.0, "steps_checked": 0}
    for rate in rates:
        done = srv.run_trace(poisson_trace(n_req, rate, n_sims, seed=rate))
        out["rates"][str(rate)] = summarize(done)
        c = conservation(done, srv.sims)
        worst = {k: (max(worst[k], c[k]) if k != "steps_checked" else worst[k] + c[k])
                 for k in worst}
    out["conservation"] = dict(worst, gate=1e-12,
                               note="FP64 moments of every served step, before and after its "
                                    "remesh (fused into the remesh kernels)")
    srv.close()
    # the same slots replaying one captured step per simulation, and the
    # device time of the saturation trace's steps replayed back to back on one
    # stream (the work the device has to do, whatever the host side)
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    srv = Server(sims, n_slots=slots, step_graphs=True)
    t0 = time.perf_counter()
    srv.warmup()
    torch.cuda.synchronize(dev)
    sg = {"graphs": len(srv._graphs), "warmup_s": time.perf_counter() - t0,
          "device_gb_held": (free0 - torch.cuda.mem_get_info(dev)[0]) / 1e9}
    trace = poisson_trace(n_req, sat, n_sims, seed=sat)
    r0 = srv.graph_replays
    sg["served_at_saturation"] = summarize(srv.run_trace(trace))
    sg["replayed_requests"] = srv.graph_replays - r0
    if len(srv._graphs) == n_sims:
        st = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(2):  # the second pass is the one kept
            torch.cuda.synchronize(dev)
            e0.record(st)
            for _, i in trace:
                srv._graphs[i][2].launch(st.cuda_stream)
            e1.record(st)
            torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        sg["serial_device_ms"] = ms
        sg["serial_device_evals_per_s"] = sum(sims[i].n for _, i in trace) / (ms * 1e-3)
    srv.close()
    out["step_graphs"] = sg
    one = Server(sims, n_slots=1)
    one.warmup(every_sim=False)
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
    ap.add_argument("--no-check", action="store_true",
                    help="skip the accuracy check of the timed step against the FP64 oracle")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (256 simulations) and served (1024 simulations) sections")
    ap.add_argument("--only", default=None, choices=["c1", "c3", "evolve", "batched", "served"],
                    help="run one extra section alone and print its JSON (profiling captures)")
    ap.add_argument("--c3-n", type=int, default=1 << 22,
                    help="blobs of the near-wall section (default 2^22; smaller for captures)")
    ap.add_argument("--c3-steps", type=int, default=5)
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
    if args.only is not None:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        sec = {"c1": lambda: run_c1(dev), "c3": lambda: run_c3(dev, n=args.c3_n, steps=args.c3_steps),
               "evolve": lambda: run_evolve(dev), "batched": lambda: run_batched(dev),
               "served": lambda: run_served(dev)}[args.only]()
        print(json.dumps({"section": args.only, **sec}), flush=True)
        return
    line = run_ours(args, rank, world)
    if rank == 0 and world == 1 and not args.no_extras and args.n is None:
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        line["c1"] = run_c1(dev)
        line["c3"] = run_c3(dev, n=args.c3_n, steps=args.c3_steps)
        line["evolve"] = run_evolve(dev)
        line["batched"] = run_batched(dev)
        line["served"] = run_served(dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
