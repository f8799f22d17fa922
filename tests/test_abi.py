"""The C ABI library loads and exports every symbol include/pfblob.h declares
(no compute: these run without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pfblob.h")
LIB = os.path.join(ROOT, "phyflow2.0_b200", "pfblob", "libpfblob.so")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("pf_create", "pf_destroy", "pf_last_error", "pf_velocity_direct", "pf_velocity_fmm",
              "pf_panel_velocity", "pf_remesh", "pf_moments"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libpfblob.so lacks {missing}"


def test_checked_library_exports_every_declared_symbol():
    """The bounds-checked build (-DPF_BOUNDS_CHECK) has the same ABI and says
    which build it is; the normal build says it is not checked, and its
    pf_check_bounds is a no-op that needs no GPU."""
    path = os.path.join(ROOT, "phyflow2.0_b200", "pfblob", "libpfblob_checked.so")
    if not os.path.exists(path):
        pytest.skip("libpfblob_checked.so not built (build.py --checked)")
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libpfblob_checked.so lacks {missing}"
    assert lib.pf_bounds_checked() == 1
    plain = ctypes.CDLL(LIB)
    assert plain.pf_bounds_checked() == 0
    assert plain.pf_check_bounds(-1) == 0


def test_python_prototypes_cover_header():
    import pfblob._lib as L
    assert set(declared_symbols()) <= set(L.PROTOTYPES)


def test_version_and_error_string_without_gpu():
    import pfblob._lib as L
    assert L.lib.pf_version() >= 10000
    assert isinstance(L.lib.pf_last_error(), bytes)


def test_create_reports_missing_device_as_status():
    import torch
    import pfblob._lib as L
    if torch.cuda.is_available():
        pytest.skip("host without a GPU only")
    p = ctypes.c_void_p()
    s = L.lib.pf_create(0, ctypes.byref(p))
    assert s in (1, 3)  # PF_ERR_INVALID_ARG (0 devices) or PF_ERR_CUDA
    assert L.lib.pf_last_error()


def test_null_context_is_rejected_without_gpu():
    import pfblob._lib as L
    s = L.lib.pf_velocity_direct(None, 10, None, None, None, 10, None, None, 1.0, None, None, None)
    assert s == 1
    assert b"NULL context" in L.lib.pf_last_error()


NO_STATUS = {"pf_last_error", "pf_version", "pf_kernel_launches", "pf_fmm_plan_builds",
             "pf_bounds_checked"}
NULL_IS_NOOP = {"pf_destroy", "pf_batch_destroy", "pf_step_graph_destroy"}  # like free(NULL)
# pf_fmm_set_tuning: 0 = automatic choice of every knob; pf_check_bounds: a
# no-op in the normal build
ZEROS_VALID = {"pf_fmm_set_tuning", "pf_check_bounds"}


def test_every_entry_point_rejects_null_arguments_without_gpu():
    """NULL handles and arrays with zero sizes and parameters: every entry
    point returns PF_ERR_INVALID_ARG with a message naming it, never crashes
    and never reaches the device."""
    import pfblob._lib as L
    for name, argtypes in L.PROTOTYPES.items():
        if name in NO_STATUS:
            continue
        args = [0.0 if t is ctypes.c_double else
                0 if t in (ctypes.c_int, ctypes.c_int32, ctypes.c_int64) else None
                for t in argtypes]
        s = getattr(L.lib, name)(*args)
        if name in NULL_IS_NOOP or name in ZEROS_VALID:
            assert s == 0, name
            continue
        assert s == 1, (name, s)
        msg = L.lib.pf_last_error().decode()
        assert msg.startswith(name.replace("_tutty", "")), (name, msg)


@pytest.mark.parametrize("bad", ["xb0", "yb0", "c"])
def test_window_remeshes_reject_non_finite_bounds_without_gpu(bad):
    """The window remeshes check their scalar arguments before any device
    work: a NaN or infinite bound or Wee coefficient is an invalid argument."""
    import pfblob._lib as L
    vals = {"xb0": 0.0, "yb0": 0.0, "c": 0.0}
    for v in (float("nan"), float("inf")):
        vals[bad] = v
        dummy = ctypes.c_void_p(16)  # never dereferenced: the checks fail first
        s = L.lib.pf_remesh_window_noalloc(0, None, None, None, 0.01, vals["xb0"], vals["yb0"],
                                           vals["c"], 0, 0, 1, 1, 0, None, None, None, None,
                                           None, dummy, None, None)
        assert s == 1 and b"finite" in L.lib.pf_last_error()
        s = L.lib.pf_remesh_window(dummy, 0, None, None, None, 0.01, vals["xb0"], vals["yb0"],
                                   vals["c"], 0, 0, 1, 1, 0, None, None, None, None, None, dummy,
                                   None, None)
        assert s == 1 and b"finite" in L.lib.pf_last_error()


def _batch_instance(**kw):
    import pfblob._lib as L
    d = L.BatchInstance()
    d.n = 0
    d.ksigmasqr = 8e-6
    d.cutoff = 0.01
    for i, v in enumerate((0.0, 1.0, 0.0, 1.0)):
        d.box[i] = v
    d.method = 0
    d.h = 0.0016
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("field,value,words", [
    ("expansion_terms", 17, "expansion terms"),
    ("expansion_terms", 64, "expansion terms"),
    ("cutoff", float("nan"), "bad cutoff"),
    ("cutoff", -1.0, "bad cutoff"),
    ("ksigmasqr", 0.0, "bad ksigmasqr"),
    ("method", 7, "method"),
    ("leaf_level", 2, "leaf level"),
])
def test_batch_rejects_bad_instances_without_gpu(field, value, words):
    """pf_batch_create checks every instance before it touches the device
    (the FMM's coefficient arrays are sized by the expansion terms, so an
    uninstantiated size must never reach the kernels)."""
    import pfblob._lib as L
    dummy_ctx = ctypes.c_void_p(16)  # never dereferenced: the checks fail first
    inst = (L.BatchInstance * 1)(_batch_instance(**{field: value}))
    out = ctypes.c_void_p()
    s = L.lib.pf_batch_create(dummy_ctx, 1, inst, 1e-6, 1, ctypes.byref(out))
    assert s == 1 and out.value is None
    assert words in L.lib.pf_last_error().decode()


@pytest.mark.parametrize("field", ["h", "xb0", "yb0", "c"])
def test_batch_rejects_non_finite_remesh_arguments_without_gpu(field):
    import pfblob._lib as L
    dummy_ctx = ctypes.c_void_p(16)
    inst = (L.BatchInstance * 1)(_batch_instance(remesh=1, **{field: float("inf")}))
    out = ctypes.c_void_p()
    assert L.lib.pf_batch_create(dummy_ctx, 1, inst, 1e-6, 1, ctypes.byref(out)) == 1
    assert "bad remesh arguments" in L.lib.pf_last_error().decode()


def test_noalloc_rejects_window_whose_cell_count_overflows_without_gpu():
    """Each window side below 2^30 but (nbx + 3)(nby + 3) far above 2^31: the
    scratch size would wrap; the argument check rejects the window before any
    CUDA call."""
    import pfblob._lib as L
    dummy = ctypes.c_void_p(16)  # never dereferenced: the checks fail first
    s = L.lib.pf_remesh_window_noalloc(4, dummy, dummy, dummy, 0.01, 0.0, 0.0, 0.0, 0, 0,
                                       847355459, 143221333, 0, None, None, None, None, None,
                                       dummy, None, None)
    assert s == 1 and b"bad window" in L.lib.pf_last_error()
    s = L.lib.pf_remesh_window(dummy, 4, dummy, dummy, dummy, 0.01, 0.0, 0.0, 0.0, 0, 0,
                               847355459, 143221333, 0, None, None, None, None, None, dummy,
                               None, None)
    assert s == 1 and b"bad window" in L.lib.pf_last_error()


def test_async_remesh_checks_its_bound_without_gpu():
    import pfblob._lib as L
    dummy = ctypes.c_void_p(16)
    for mb in (0, 1 << 30):
        s = L.lib.pf_remesh_async(dummy, 4, dummy, dummy, dummy, 0.01, 0.0, 0.0, 0.0, mb, 0, None,
                                  None, None, None, None, dummy, None, None, None, None)
        assert s == 1 and b"max_base_cells" in L.lib.pf_last_error()


@pytest.mark.parametrize("struct,mirror", [("pf_step", "Step"),
                                           ("pf_batch_instance", "BatchInstance"),
                                           ("pf_fmm_stats", "FmmStats")])
def test_struct_mirrors_match_the_header_layout(tmp_path, struct, mirror):
    """The ctypes mirrors have the header's size and field offsets (checked by
    compiling the header with the host C compiler)."""
    import shutil
    import subprocess
    import pfblob._lib as L
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    m = getattr(L, mirror)
    fields = [f for f, _ in m._fields_]
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pfblob.h"', 'int main(void) {',
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ['  return 0;', '}']
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    inc = ["-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include"]
    r = subprocess.run([cc, *inc, str(src), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("header does not compile with the host compiler here: " + r.stderr[-300:])
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(m)
    assert out[1:] == [getattr(m, f).offset for f in fields]
