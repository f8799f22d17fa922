"""The GPU suite once more on the bounds-checked build (libpfblob_checked.so,
-DPF_BOUNDS_CHECK): every data-dependent index the kernels test (counting-sort
slots of the FMM and the remesh, P2P source runs and target groups, L2P
scatter, remesh records and output slots) stays inside its buffer in every
GPU test, and the results still pass the same parity gates.  A failed test
records its site and skips the access (no trap); pf_check_bounds, called after
every library call in this build, turns it into an error."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_gpu_suite_on_the_checked_build():
    lib = os.path.join(ROOT, "phyflow2.0_b200", "pfblob", "libpfblob_checked.so")
    assert os.path.exists(lib), "libpfblob_checked.so not built (build.py --checked)"
    env = dict(os.environ, PFBLOB_CHECKED="1")
    cmd = [sys.executable, "-m", "pytest", os.path.join(ROOT, "tests"), "-m", "gpu", "-x", "-q",
           "-p", "no:cacheprovider", "-k", "not test_gpu_suite_on_the_checked_build"]
    r = subprocess.run(cmd, env=env, cwd=ROOT, capture_output=True, text=True, timeout=1200)
    tail = (r.stdout + r.stderr)[-3000:]
    assert r.returncode == 0, tail
    assert " passed" in r.stdout, tail


def test_loaded_variant_matches_environment():
    """Runs in both suites: the library loaded is the one PFBLOB_CHECKED asks
    for (the checked run above really runs the checked kernels)."""
    import pfblob._lib as L
    assert L.lib.pf_bounds_checked() == int(L.CHECKED)
    assert os.path.basename(L.LIB_PATH) == ("libpfblob_checked.so" if L.CHECKED else "libpfblob.so")
