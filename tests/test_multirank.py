"""Multi-process paths of bench.py on CPU (gloo, world size 2): the job time is
the max over ranks, and the reference arm runs on rank 0 only."""
import os
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    v = bench.reduce_max(1.5 + rank, torch.device("cpu"), world)
    out[rank] = v
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.get_context("spawn").Manager() as m:  # no fork of a threaded process
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        assert out[0] == out[1] == 2.5


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_on_rank0():
    """Rank 0 prints one JSON line with the contract's keys; its metric and
    config workload are those of the GPU arm's line."""
    import json
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "evals/s" and d["higher_is_better"]
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["n_blobs"] == 1 << 20
    assert "velocity at all blobs" in d["config"]["workload"]


def test_reference_arm_does_not_load_the_library():
    """The reference arm's workload comes from the generator file alone: the
    pfblob package (whose import loads libpfblob.so) is never imported."""
    code = ("import sys; sys.argv=['bench.py']; import bench; b = bench.workload_c2(4096); "
            "assert b.n == 4096; assert 'pfblob' not in sys.modules, sorted(sys.modules)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
