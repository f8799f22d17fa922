"""Build libpfblob.so (sm_100a) in-tree.

    python phyflow2.0_b200/build.py [--force] [--verbose-ptxas] [--checked]

Compiles every csrc/*.cu with nvcc for sm_100a only and links the shared
library into pfblob/libpfblob.so, next to the Python host package that loads
it.  Objects go to _build/ (git-ignored).  Incremental: a source is rebuilt
when it or any csrc header is newer than its object.

--checked builds the bounds-checked variant instead (-DPF_BOUNDS_CHECK,
objects in _build_checked/, pfblob/libpfblob_checked.so; selected at import
by PFBLOB_CHECKED=1).
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "pfblob", "libpfblob.so")
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
OUT_CHECKED = os.path.join(HERE, "pfblob", "libpfblob_checked.so")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
                 "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, force, ptxas_v, checked=False):
    obj = os.path.join(BUILD_CHECKED if checked else BUILD, os.path.basename(src)[:-3] + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header())):
        return obj, None
    cmd = ([NVCC] + CFLAGS + (["-DPF_BOUNDS_CHECK"] if checked else [])
           + (["-Xptxas", "-v"] if ptxas_v else []) + ["-c", src, "-o", obj])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, (r.stderr if ptxas_v else None)


def build(force=False, ptxas_v=False, checked=False):
    out = OUT_CHECKED if checked else OUT
    os.makedirs(BUILD_CHECKED if checked else BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        res = list(ex.map(lambda s: _compile(s, force, ptxas_v, checked), srcs))
    objs = [o for o, _ in res]
    if ptxas_v:
        for _, log in res:
            if log:
                sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(out) or os.path.getmtime(out) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--checked", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose_ptxas, a.checked))
