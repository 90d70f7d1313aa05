"""Loads libjurassic_b200.so and declares the C-ABI of
include/jurassic_b200.h.  There is no fallback: if the library is missing
the import fails with instructions to build it."""
import ctypes as C
import os

from . import structs as S

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libjurassic_b200.so")

# Every symbol the public header declares.
EXPORTS = [
    "formod", "brightness", "planck", "jsc_status_string", "jsc_last_status",
    "jsc_set_exit_on_error", "jsc_last_error_message", "jsc_release_cache",
    "jsc_launch_count", "jsc_model_create", "jsc_model_destroy",
    "jsc_model_table_bytes", "jsc_batch_create", "jsc_batch_destroy",
    "jsc_batch_upload", "jsc_batch_run", "jsc_batch_download",
    "jsc_formod_batch", "jsc_batch_set_timing", "jsc_batch_kernel_ms",
    "jsc_batch_counters", "jsc_batch_set_digest", "jsc_batch_index_digest",
    "jsc_batch_autotune", "jsc_batch_variant", "jsc_batch_variant_ms",
    "jsc_batch_set_aero", "jsc_formod_batch_noalloc", "jsc_batch_set_nalpha",
    "jsc_batch_set_variant", "jsc_surrogate_create", "jsc_surrogate_destroy",
    "jsc_surrogate_param_count", "jsc_surrogate_get_params", "jsc_surrogate_set_params",
    "jsc_surrogate_loss_grad", "jsc_surrogate_train", "jsc_surrogate_predict",
    "jsc_batch_scatter_samples", "jsc_batch_set_surrogate", "jsc_batch_surrogate_stats",
    "jsc_batch_set_fixed", "jsc_batch_download_async", "jsc_batch_async_status",
    "jsc_batch_graph_capture", "jsc_batch_graph_launch", "jsc_surrogate_set_tensor_path",
    "jsc_atm2x", "jsc_x2atm", "jsc_obs2y", "jsc_kernel", "jsc_read_aero", "jsc_get_opt_prop",
    "formod_pencil", "formod_fov", "read_shape", "read_tbl", "srcfunc_planck",
    "formod_continua", "intpol_tbl", "intpol_tbl_eps", "intpol_tbl_u", "locate_tbl",
    "jsc_srcfunc_sca", "jsc_batch_scatter_points", "jsc_surrogate_get_scaling",
    "jsc_batch_set_nalpha_depth", "jsc_batch_set_wait_budget", "jsc_scan_selftest",
    "jsc_batch_set_fixed_points", "jsc_batch_set_surrogate_depth",
    "jsc_batch_scatter_samples_depth", "jsc_batch_surrogate_stats_depth",
]


class BatchInput(C.Structure):
    _fields_ = [
        ("n_atm", C.c_int), ("n_levels", C.c_int),
        ("atm_off", C.POINTER(C.c_int)),
        ("z", C.POINTER(C.c_double)), ("lon", C.POINTER(C.c_double)),
        ("lat", C.POINTER(C.c_double)), ("p", C.POINTER(C.c_double)),
        ("t", C.POINTER(C.c_double)),
        ("q", C.POINTER(C.c_double)), ("k", C.POINTER(C.c_double)),
        ("n_rays", C.c_int),
        ("ray_atm", C.POINTER(C.c_int)),
        ("time", C.POINTER(C.c_double)),
        ("obsz", C.POINTER(C.c_double)), ("obslon", C.POINTER(C.c_double)),
        ("obslat", C.POINTER(C.c_double)),
        ("vpz", C.POINTER(C.c_double)), ("vplon", C.POINTER(C.c_double)),
        ("vplat", C.POINTER(C.c_double)),
    ]


class BatchOutput(C.Structure):
    _fields_ = [
        ("rad", C.POINTER(C.c_double)), ("tau", C.POINTER(C.c_double)),
        ("tpz", C.POINTER(C.c_double)), ("tplon", C.POINTER(C.c_double)),
        ("tplat", C.POINTER(C.c_double)), ("nlos", C.POINTER(C.c_int)),
    ]


_lib = None


def load():
    """The library handle, loaded once with the C-ABI signatures set."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libjurassic_b200.so not found at %s; build it with "
            "'python jurassic-scatter_b200/build.py' (or __graft_entry__.build())"
            % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    P = C.POINTER
    sig = {
        "formod": (None, [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT)]),
        "brightness": (d, [d, d]),
        "planck": (d, [d, d]),
        "jsc_status_string": (C.c_char_p, [i]),
        "jsc_last_status": (i, []),
        "jsc_set_exit_on_error": (None, [i]),
        "jsc_read_aero": (i, [C.c_char_p, C.c_char_p, P(S.CtlT), P(S.AeroT)]),
        "jsc_get_opt_prop": (i, [P(S.CtlT), P(S.AeroT)]),
        "jsc_atm2x": (C.c_size_t, [P(S.CtlT), P(S.AtmT), P(S.AeroT), vp, vp, vp]),
        "jsc_x2atm": (None, [P(S.CtlT), vp, P(S.AtmT), P(S.AeroT)]),
        "jsc_obs2y": (C.c_size_t, [P(S.CtlT), P(S.ObsT), vp, vp, vp]),
        "jsc_kernel": (i, [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT), vp, C.c_size_t,
                           C.c_size_t, C.c_size_t]),
        "jsc_last_error_message": (C.c_char_p, []),
        "jsc_release_cache": (None, []),
        "jsc_launch_count": (C.c_uint64, []),
        "jsc_model_create": (i, [P(S.CtlT), i, P(vp)]),
        "jsc_model_destroy": (None, [vp]),
        "jsc_model_table_bytes": (C.c_size_t, [vp]),
        "jsc_batch_create": (i, [vp, P(S.CtlT), i, i, i, C.c_int64, P(vp)]),
        "jsc_batch_destroy": (None, [vp]),
        "jsc_batch_upload": (i, [vp, P(BatchInput), vp]),
        "jsc_batch_run": (i, [vp, vp]),
        "jsc_batch_download": (i, [vp, P(BatchOutput), vp]),
        "jsc_formod_batch": (i, [vp, P(S.CtlT), P(BatchInput), P(BatchOutput), vp]),
        "jsc_batch_set_timing": (None, [vp, i]),
        "jsc_batch_kernel_ms": (d, [vp, C.c_char_p]),
        "jsc_batch_counters": (i, [vp, P(C.c_int64), P(C.c_int64)]),
        "jsc_batch_set_digest": (i, [vp, i]),
        "jsc_batch_index_digest": (i, [vp, P(C.c_uint64)]),
        "jsc_batch_autotune": (i, [vp, vp]),
        "jsc_batch_variant": (i, [vp, P(i), P(i), P(i)]),
        "jsc_batch_variant_ms": (d, [vp, i]),
        "jsc_batch_set_aero": (i, [vp, P(S.AeroT)]),
        "jsc_batch_set_nalpha": (i, [vp, i]),
        "jsc_batch_set_variant": (i, [vp, i]),
        "jsc_batch_set_fixed": (i, [vp, i]),
        "jsc_batch_download_async": (i, [vp, P(BatchOutput), vp]),
        "jsc_batch_async_status": (i, [vp]),
        "jsc_batch_graph_capture": (i, [vp, P(BatchInput), P(BatchOutput), vp]),
        "jsc_batch_graph_launch": (i, [vp, vp]),
        "jsc_surrogate_create": (i, [i, i, C.c_uint64, P(vp)]),
        "jsc_surrogate_destroy": (None, [vp]),
        "jsc_surrogate_param_count": (i, [vp]),
        "jsc_surrogate_get_params": (i, [vp, P(C.c_float)]),
        "jsc_surrogate_set_params": (i, [vp, P(C.c_float)]),
        "jsc_surrogate_loss_grad": (i, [vp, P(C.c_float), P(C.c_float), i, P(C.c_float),
                                        P(C.c_float)]),
        "jsc_surrogate_train": (i, [vp, P(C.c_float), P(d), C.c_int64, i, i, C.c_float,
                                    C.c_uint64, P(C.c_float)]),
        "jsc_surrogate_predict": (i, [vp, P(C.c_float), i, P(d)]),
        "jsc_surrogate_set_tensor_path": (i, [vp, i]),
        "jsc_batch_scatter_samples": (i, [vp, P(C.c_float), P(d), C.c_int64, P(C.c_int64)]),
        "jsc_batch_set_surrogate": (i, [vp, vp, d, i]),
        "jsc_batch_surrogate_stats": (i, [vp, P(C.c_int64), P(C.c_int64), P(C.c_int64), P(d),
                                          P(i)]),
        "jsc_formod_batch_noalloc": (i, [vp, P(S.CtlT), P(BatchInput), P(BatchOutput), vp]),
        "formod_pencil": (None, [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT), i, i]),
        "formod_fov": (None, [P(S.CtlT), P(S.ObsT)]),
        "read_shape": (None, [C.c_char_p, P(d), P(d), P(i)]),
        "read_tbl": (None, [P(S.CtlT), vp]),
        "srcfunc_planck": (None, [P(S.CtlT), d, P(d)]),
        "formod_continua": (None, [P(S.CtlT), P(S.LosT), i, P(d)]),
        "intpol_tbl": (None, [P(S.CtlT), vp, P(S.LosT), i, P(d), P(d)]),
        "intpol_tbl_eps": (d, [vp, i, i, i, i, d]),
        "intpol_tbl_u": (d, [vp, i, i, i, i, d]),
        "locate_tbl": (i, [P(C.c_float), i, d]),
        "jsc_srcfunc_sca": (i, [P(S.CtlT), P(S.AtmT), P(S.AeroT), i, P(d), P(d), P(i), P(d), i,
                                P(d)]),
        "jsc_batch_scatter_points": (i, [vp, i, P(d), P(d), P(i), P(d), P(i), P(d), vp]),
        "jsc_surrogate_get_scaling": (i, [vp, P(C.c_float), P(C.c_float), P(C.c_float),
                                          P(C.c_float)]),
        "jsc_batch_set_nalpha_depth": (i, [vp, i, i]),
        "jsc_batch_set_wait_budget": (i, [vp, C.c_uint]),
        "jsc_scan_selftest": (i, [i, i, C.c_uint, i]),
        "jsc_batch_set_fixed_points": (i, [vp, C.c_int64]),
        "jsc_batch_set_surrogate_depth": (i, [vp, i, vp, d, i]),
        "jsc_batch_scatter_samples_depth": (i, [vp, i, P(C.c_float), P(d), C.c_int64,
                                                P(C.c_int64)]),
        "jsc_batch_surrogate_stats_depth": (i, [vp, i, P(C.c_int64), P(C.c_int64),
                                                P(C.c_int64), P(d), P(d), P(i)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class JscError(RuntimeError):
    def __init__(self, status, where=""):
        lib = load()
        msg = lib.jsc_last_error_message().decode(errors="replace")
        super().__init__("%s: %s (%s)" % (where, lib.jsc_status_string(status).decode(), msg))
        self.status = status


def check(status, where=""):
    if status != 0:
        raise JscError(status, where)
