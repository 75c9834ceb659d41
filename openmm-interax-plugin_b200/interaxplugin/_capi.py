"""ctypes binding of the C ABI in include/interax_b200.h (libinterax_b200.so, built in-tree)."""
import ctypes
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent.parent
# IX_B200_LIBRARY names another build of the library (the autotuner's candidates); the default is the in-tree build
LIB_PATH = Path(os.environ.get("IX_B200_LIBRARY", str(_PKG / "libinterax_b200.so")))

IX_OK = 0
IX_POSQ_FLOAT4, IX_POSQ_FLOAT4_CORRECTED, IX_POSQ_DOUBLE4 = 0, 1, 2
P = ctypes.c_void_p


class PairSettings(ctypes.Structure):
    _fields_ = [("nonbonded_method", ctypes.c_int), ("cutoff", ctypes.c_double),
                ("use_switching_function", ctypes.c_int), ("switching_distance", ctypes.c_double),
                ("softcore_radius", ctypes.c_double), ("force_group", ctypes.c_int),
                ("alchemical_parameter", ctypes.c_char_p), ("num_exclusions", ctypes.c_int),
                ("exclusions", P)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_longlong) for k in ("submitted", "admitted", "completed", "failed", "contexts", "cohorts",
                                                  "pending", "running")] + \
               [(k, ctypes.c_double) for k in ("budget_bytes", "reserved_bytes", "peak_reserved_bytes", "arena_bytes",
                                               "peak_arena_bytes")] + [("worker_seconds", ctypes.c_double * 12)] + \
               [("contexts_reused", ctypes.c_longlong)]


_lib = None


def lib():
    """Load the CUDA library.  There is no fallback: a missing library is an error."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(the InteraxFF B200 path has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        sig = {
            "ix_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, P, ctypes.POINTER(P)]),
            "ix_ctx_destroy": (None, [P]),
            "ix_last_error": (ctypes.c_char_p, [P]),
            "ix_add_dispersion": (ctypes.c_int, [P, ctypes.POINTER(PairSettings), P, P, ctypes.c_double, ctypes.c_int]),
            "ix_add_exchange": (ctypes.c_int, [P, ctypes.POINTER(PairSettings), P, P, ctypes.c_int]),
            "ix_add_short_range": (ctypes.c_int, [P, ctypes.POINTER(PairSettings), P, P, ctypes.c_int]),
            "ix_add_three_body": (ctypes.c_int, [P, ctypes.c_int, P, P, P, P, P, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 ctypes.c_char_p, ctypes.c_int]),
            "ix_update_dispersion": (ctypes.c_int, [P, P, ctypes.c_double]),
            "ix_update_exchange": (ctypes.c_int, [P, P, ctypes.c_int]),
            "ix_update_short_range": (ctypes.c_int, [P, P, ctypes.c_int]),
            "ix_update_three_body": (ctypes.c_int, [P, P, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "ix_set_parameter": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_double]),
            "ix_dispersion_long_range_correction": (ctypes.c_int, [ctypes.c_int, P, P, ctypes.POINTER(PairSettings),
                                                                   ctypes.c_double, ctypes.c_int, P, P]),
            "ix_set_positions": (ctypes.c_int, [P, P, P]),
            "ix_compute": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]),
            "ix_compute_device": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.c_int, P]),
            "ix_compute_device_f64": (ctypes.c_int, [P, ctypes.c_int, P, P, P, P]),
            "ix_compute_device_posq": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, P, P, P, P, ctypes.c_int, P,
                                                      P]),
            "ix_get_device_status": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int)]),
            "ix_set_list_capacity": (ctypes.c_int, [P, ctypes.c_longlong, ctypes.c_int]),
            "ix_get_list_stats": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_longlong)]),
            "ix_set_counting": (ctypes.c_int, [P, ctypes.c_int]),
            "ix_get_counts": (ctypes.c_int, [P, P, P]),
            "ix_md_set_masses": (ctypes.c_int, [P, P]),
            "ix_md_run": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, P, P, P]),
            "ix_md_set_constraints": (ctypes.c_int, [P, ctypes.c_int, P, P, ctypes.c_double]),
            "ix_get_stream": (P, [P]),
            "ix_synchronize": (ctypes.c_int, [P]),
            "ix_version": (ctypes.c_char_p, []),
            "ix_measure_fp32_peak": (ctypes.c_int, [ctypes.c_int, P]),
            "ix_md_steps_async": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double]),
            "ix_md_finish": (ctypes.c_int, [P, P, P, P]),
            "ix_set_profiling": (ctypes.c_int, [P, ctypes.c_int]),
            "ix_get_kernel_times": (ctypes.c_int, [P, P, P]),
            "ix_get_launch_count": (ctypes.c_int, [P, P]),
            "ix_set_graphs": (ctypes.c_int, [P, ctypes.c_int]),
            "ix_compute_windows": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_int, P, P, P]),
            "ix_compute_windows_device": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_int, P, P, P]),
            "ix_three_body_noalloc": (ctypes.c_int, [ctypes.c_int, P, P, ctypes.c_int, P, P, P, P, P, ctypes.c_double,
                                                     ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_int, ctypes.c_double, P, P, P]),
            "ix_three_body_noalloc_overflow": (ctypes.c_int, [P]),
            "ix_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(P)]),
            "ix_batch_destroy": (None, [P]),
            "ix_batch_last_error": (ctypes.c_char_p, [P]),
            "ix_batch_add_system": (ctypes.c_int, [P, ctypes.c_int, P]),
            "ix_batch_add_dispersion": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(PairSettings), P, P,
                                                       ctypes.c_double, ctypes.c_int]),
            "ix_batch_add_exchange": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(PairSettings), P, P,
                                                     ctypes.c_int]),
            "ix_batch_add_short_range": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(PairSettings), P, P,
                                                        ctypes.c_int]),
            "ix_batch_add_three_body": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, P, P, P, P, ctypes.c_double,
                                                       ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                       ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
            "ix_batch_set_parameter": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_double]),
            "ix_batch_num_particles": (ctypes.c_int, [P, P, P]),
            "ix_batch_compute": (ctypes.c_int, [P, P, P, P]),
            "ix_batch_compute_device": (ctypes.c_int, [P, P, P, P]),
            "ix_batch_get_counts": (ctypes.c_int, [P, P, P]),
            "ix_batch_get_stream": (P, [P]),
            "ix_batch_md_run": (ctypes.c_int, [P, P, ctypes.c_double, P, P, P, P, P]),
            "ix_request_create": (ctypes.c_int, [ctypes.c_int, P, ctypes.POINTER(P)]),
            "ix_request_set_state": (ctypes.c_int, [P, P, P, P]),
            "ix_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(P)]),
            "ix_server_set_batching": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
            "ix_server_destroy": (None, [P]),
            "ix_server_last_error": (ctypes.c_char_p, [P]),
            "ix_server_submit": (ctypes.c_int, [P, P, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]),
            "ix_server_poll": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.POINTER(ctypes.c_int)]),
            "ix_server_wait": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_int, P, ctypes.POINTER(ctypes.c_int)]),
            "ix_server_result": (ctypes.c_int, [P, ctypes.c_longlong, P, P, P, P, ctypes.POINTER(ctypes.c_double)]),
            "ix_server_stats_get": (ctypes.c_int, [P, ctypes.POINTER(ServerStats)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)
