"""ctypes binding of libpfblob.so (the C ABI declared in include/pfblob.h).

The library is required: importing this module raises if the shared object
is missing or fails to load.  There is no CPU path behind it.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# PFBLOB_CHECKED=1 selects the bounds-checked build (libpfblob_checked.so):
# every call is then followed by pf_check_bounds, which synchronises.
CHECKED = os.environ.get("PFBLOB_CHECKED", "0") not in ("", "0")
LIB_PATH = os.path.join(_HERE, "libpfblob_checked.so" if CHECKED else "libpfblob.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"pfblob: {LIB_PATH} is not built; run `python phyflow2.0_b200/build.py"
        f"{' --checked' if CHECKED else ''}` (the package has no CPU fallback)")

lib = ctypes.CDLL(LIB_PATH)

_c = ctypes
_vp = _c.c_void_p
_i64 = _c.c_int64
_dbl = _c.c_double
_int = _c.c_int

PF_OK = 0
STATUS_NAMES = {0: "PF_OK", 1: "PF_ERR_INVALID_ARG", 2: "PF_ERR_OOM", 3: "PF_ERR_CUDA",
                4: "PF_ERR_TIMEOUT", 5: "PF_ERR_NAN_INPUT", 6: "PF_ERR_CAPACITY",
                7: "PF_ERR_NOT_BUILT"}

# (name, argtypes) for every entry point declared in include/pfblob.h
PROTOTYPES = {
    "pf_create": [_int, _c.POINTER(_vp)],
    "pf_destroy": [_vp],
    "pf_last_error": [],
    "pf_mem_usage": [_vp, _c.POINTER(_c.c_size_t)],
    "pf_trim": [_vp],
    "pf_version": [],
    "pf_kernel_launches": [],
    "pf_bounds_checked": [],
    "pf_check_bounds": [_int],
    "pf_velocity_direct": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _vp, _vp, _vp],
    "pf_velocity_direct_cutoff": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _vp, _vp, _vp],
    "pf_vorticity_direct": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _vp, _vp],
    "pf_vorticity_direct_cutoff": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _vp, _vp],
    "pf_velocity_fmm": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _int,
                        _vp, _vp, _vp],
    "pf_velocity_fmm_box": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _dbl, _dbl, _dbl, _dbl,
                            _int, _c.POINTER(_dbl), _vp, _vp, _vp],
    "pf_panel_velocity": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp,
                          _int, _vp],
    "pf_source_panel_velocity": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp,
                          _int, _vp],
    "pf_remesh": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _i64, _vp, _vp, _vp, _vp, _vp,
                  _c.POINTER(_i64), _vp],
    "pf_remesh_tutty": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _i64, _vp, _vp, _vp,
                        _vp, _vp, _c.POINTER(_i64), _vp],
    "pf_moments": [_vp, _i64, _vp, _vp, _vp, _vp, _vp],
    "pf_panel_influence_matrix": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_source_panel_influence_matrix": [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_dense_lu_factor": [_vp, _i64, _vp, _vp, _vp, _vp],
    "pf_dense_lu_solve": [_vp, _i64, _vp, _vp, _vp, _vp],
    "pf_population_control": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_remesh_population_control": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl,
                                     _i64, _vp, _vp, _vp, _vp, _vp, _c.POINTER(_i64),
                                     _c.POINTER(_dbl), _vp],
    "pf_remesh_window": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _i64, _i64, _i64, _i64,
                         _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_remesh_async": [_vp, _i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _i64, _i64, _vp, _vp,
                        _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_blob_step": [_vp, _vp, _vp],
    "pf_step_graph_create": [_vp, _vp, _c.POINTER(_vp)],
    "pf_step_graph_launch": [_vp, _vp],
    "pf_step_graph_kernels": [_vp, _c.POINTER(_i64)],
    "pf_step_graph_destroy": [_vp],
    "pf_remesh_window_noalloc": [_i64, _vp, _vp, _vp, _dbl, _dbl, _dbl, _dbl, _i64, _i64, _i64,
                                 _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pf_fmm_lists": [_int, _int, _dbl, _dbl, _dbl, _vp, _i64, _c.POINTER(_i64)],
    "pf_fmm_set_tuning": [_int, _int, _int],
    "pf_fmm_plan_builds": [],
    "pf_batch_create": [_vp, _c.c_int32, _vp, _dbl, _c.c_int32, _c.POINTER(_vp)],
    "pf_batch_run": [_vp, _vp],
    "pf_batch_results": [_vp, _vp, _vp],
    "pf_batch_info": [_vp, _vp, _vp, _vp],
    "pf_batch_destroy": [_vp],
    "pf_fmm_profile": [_vp, _int],
    "pf_fmm_last_stats": [_vp, _vp],
    "pf_fmm_tree_keys": [_vp, _i64, _vp, _vp, _dbl, _dbl, _dbl, _int, _vp, _vp],
}

for _name, _args in PROTOTYPES.items():
    if not hasattr(lib, _name):
        continue  # optional entry points are checked by the symbol test
    f = getattr(lib, _name)
    f.argtypes = _args
    f.restype = _int
lib.pf_last_error.restype = _c.c_char_p
lib.pf_version.restype = _int
lib.pf_kernel_launches.restype = _c.c_uint64
lib.pf_fmm_plan_builds.restype = _c.c_uint64


class PfError(RuntimeError):
    """A libpfblob call returned a status other than PF_OK."""

    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


class CapacityError(PfError):
    def __init__(self, status, msg, needed):
        self.needed = needed
        super().__init__(status, msg)


def check(status):
    if status == PF_OK and CHECKED:
        status = lib.pf_check_bounds(-1)
    if status != PF_OK:
        msg = lib.pf_last_error()
        raise PfError(status, msg.decode() if msg else "")


_ctx_lock = threading.Lock()
_ctx = {}


def context(device=0):
    """Per-(device, thread) pf_ctx handle (contexts are not shared between
    host threads)."""
    key = (device, threading.get_ident())
    with _ctx_lock:
        h = _ctx.get(key)
        if h is None:
            p = _vp()
            check(lib.pf_create(int(device), _c.byref(p)))
            h = p.value
            _ctx[key] = h
    return h


def mem_usage(device=0):
    n = _c.c_size_t()
    check(lib.pf_mem_usage(context(device), _c.byref(n)))
    return n.value


def version():
    return lib.pf_version()


def fmm_plan_builds():
    """Process-wide number of FMM plans built so far."""
    return int(lib.pf_fmm_plan_builds())


def kernel_launches():
    """Process-wide number of library kernel launches so far."""
    return int(lib.pf_kernel_launches())


class FmmStats(_c.Structure):
    """Mirror of pf_fmm_stats (include/pfblob.h)."""
    _fields_ = [("leaf_level", _c.c_int32), ("expansion_terms", _c.c_int32),
                ("block_level_drop", _c.c_int32), ("used_direct", _c.c_int32),
                ("n_src", _c.c_int64), ("n_tgt", _c.c_int64), ("p2p_pairs", _c.c_int64),
                ("m2l_translations", _c.c_int64), ("ms_sort", _c.c_float),
                ("ms_upward", _c.c_float), ("ms_m2l", _c.c_float), ("ms_downward", _c.c_float),
                ("ms_p2p", _c.c_float), ("ms_l2p", _c.c_float), ("ms_total", _c.c_float),
                ("reserved", _c.c_float), ("p2p_pairs_far", _c.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


def fmm_profile(enable, device=0):
    check(lib.pf_fmm_profile(context(device), int(bool(enable))))


def fmm_last_stats(device=0):
    s = FmmStats()
    check(lib.pf_fmm_last_stats(context(device), _c.byref(s)))
    return s.as_dict()


def fmm_set_tuning(leaf_level=0, expansion_terms=0, block_level_drop=1):
    check(lib.pf_fmm_set_tuning(int(leaf_level), int(expansion_terms), int(block_level_drop)))


class BatchInstance(_c.Structure):
    """Mirror of pf_batch_instance (include/pfblob.h)."""
    _fields_ = [("n", _c.c_int64), ("x", _vp), ("y", _vp), ("g", _vp), ("vx", _vp), ("vy", _vp),
                ("ksigmasqr", _c.c_double), ("cutoff", _c.c_double), ("box", _c.c_double * 4),
                ("method", _c.c_int32), ("leaf_level", _c.c_int32),
                ("expansion_terms", _c.c_int32), ("remesh", _c.c_int32), ("h", _c.c_double),
                ("xb0", _c.c_double), ("yb0", _c.c_double), ("c", _c.c_double),
                ("capacity", _c.c_int64), ("x_out", _vp), ("y_out", _vp), ("g_out", _vp)]


class Step(_c.Structure):
    """Mirror of pf_step (include/pfblob.h)."""
    _fields_ = [("n", _c.c_int64), ("x", _vp), ("y", _vp), ("g", _vp),
                ("ksigmasqr", _c.c_double), ("xopt", _c.c_double), ("cutoff", _c.c_double),
                ("tol", _c.c_double), ("method", _c.c_int32), ("leaf_level", _c.c_int32),
                ("box", _c.c_double * 4), ("vx", _vp), ("vy", _vp), ("h", _c.c_double),
                ("xb0", _c.c_double), ("yb0", _c.c_double), ("c", _c.c_double),
                ("max_base_cells", _c.c_int64), ("capacity", _c.c_int64), ("x_out", _vp),
                ("y_out", _vp), ("g_out", _vp), ("n_out_dev", _vp), ("status_dev", _vp),
                ("moments_dev", _vp)]
