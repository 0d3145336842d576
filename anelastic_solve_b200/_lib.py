"""Loader of the sm_100a library libanel.so (ctypes).

The product path has no CPU fallback: if the library is missing or does not
load, every call raises.  Build it with ``python -m anelastic_solve_b200.build``
or ``__graft_entry__.build()``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import abi

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libanel.so"
_LIB = None

# every symbol declared in include/anel.h, with (restype, argtypes)
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
SIGNATURES = {
    "anel_last_error": (C.c_char_p, []),
    "anel_version": (C.c_int, []),
    "anel_kernel_launch_count": (C.c_int64, []),
    "anel_tuning_report": (C.c_int32, [C.c_char_p, C.c_int32]),
    "anel_mg_init": (C.c_int, [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams)]),
    "anel_mg_set_density": (C.c_int, [_DP]),
    "anel_mg_solve": (None, [_DP, _DP, _IP, _DP]),
    "anel_mg_finalize": (C.c_int, []),
    "anel_mg_create": (_P, [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams), C.c_int32, _IP]),
    "anel_mg_destroy": (None, [_P]),
    "anel_mg_ctx_set_density": (C.c_int, [_P, _DP, C.c_int32]),
    "anel_mg_ctx_solve": (C.c_int, [_P, _DP, _DP, C.c_int32, _P, C.POINTER(abi.MGReport)]),
    "anel_mg_ctx_solve_batch": (C.c_int, [_P, C.c_int32, C.POINTER(_DP), C.POINTER(_DP), _P,
                                          C.POINTER(abi.MGReport)]),
    "anel_mg_ctx_levels": (C.c_int, [_P, _IP, C.c_int32]),
    "anel_mg_ctx_set_profiling": (C.c_int, [_P, C.c_int32]),
    "anel_mg_ctx_debug_pass": (C.c_int, [_P, C.c_int32, _DP, _DP, _P]),
    "anel_ns_create": (_P, [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams),
                            C.POINTER(abi.NSParams), C.c_int32, _IP]),
    "anel_ns_destroy": (None, [_P]),
    "anel_ns_set_fields": (C.c_int, [_P, C.POINTER(abi.Fields), C.c_int32]),
    "anel_ns_get_fields": (C.c_int, [_P, C.POINTER(abi.Fields), C.c_int32]),
    "anel_ns_ctx_substep": (C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _P, _IP, _DP]),
    "anel_ns_ctx_step": (C.c_int, [_P, C.c_int32, _P, C.POINTER(abi.StepReport)]),
    "anel_ns_ctx_step_cohort": (C.c_int, [C.POINTER(_P), C.c_int32, C.c_int32, _P, _P,
                                          C.POINTER(abi.StepReport)]),
    "anel_ns_ctx_set_clock": (C.c_int, [_P, C.c_double, C.c_int32]),
    "anel_ns_ctx_set_profiling": (C.c_int, [_P, C.c_int32]),
    "anel_ns_ctx_project": (C.c_int, [_P, _IP, _DP]),
    "anel_ns_ctx_divergence": (C.c_int, [_P, _DP]),
    "anel_ns_ctx_step_host": (C.c_int, [_P, C.POINTER(abi.Fields), C.POINTER(abi.Fields), C.c_int32, _P,
                                        C.POINTER(abi.StepReport)]),
    "anel_ns_ctx_set_diagnostics": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "anel_ns_ctx_compute_diagnostics": (C.c_int, [_P, _P]),
    "anel_ns_ctx_get_diagnostics": (C.c_int, [_P, _DP, C.c_int32]),
    "anel_restart_write": (C.c_int, [C.c_char_p, C.c_int32, _P, C.c_int32, C.c_int32, C.c_int32,
                                     C.POINTER(_DP)]),
    "anel_restart_read": (C.c_int, [C.c_char_p, C.c_int32, _P, C.c_int32, C.c_int32, C.c_int32,
                                    C.POINTER(_DP)]),
    "anel_ns_ctx_write_restart": (C.c_int, [_P, C.c_char_p, C.c_int32, _P]),
    "anel_ns_ctx_read_restart": (C.c_int, [_P, C.c_char_p, C.c_int32, C.c_int32, _P]),
    "anel_serve_create": (_P, [C.c_int32, C.c_int64, C.c_int32, _IP]),
    "anel_serve_submit": (C.c_int, [_P, C.POINTER(abi.Request), C.POINTER(C.c_int64)]),
    "anel_serve_poll": (C.c_int, [_P, C.POINTER(abi.Result), C.c_int32, _IP, C.c_int32]),
    "anel_serve_drain": (C.c_int, [_P]),
    "anel_serve_stats_get": (C.c_int, [_P, C.POINTER(abi.ServeStats)]),
    "anel_serve_destroy": (None, [_P]),
    "anel_divergence_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _DP, _DP, _DP, _DP, _DP,
                                          _DP, _DP, _P]),
    "anel_ns_init": (C.c_int, [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams),
                               C.POINTER(abi.NSParams)]),
    "anel_bind_fields": (C.c_int, [C.POINTER(abi.Fields)]),
    "anel_rk_substep": (None, [_DP, _DP, _DP, _DP, _DP, _DP, _IP, _IP]),
    "anel_ns_finalize": (C.c_int, []),
}


class AnelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"anel error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load libanel.so once; raise if it is absent (no CPU fallback)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run python -m anelastic_solve_b200.build")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def last_error() -> str:
    return (lib().anel_last_error() or b"").decode()


def check(code: int, allow=(abi.OK,)) -> int:
    if code not in allow:
        raise AnelError(code, last_error())
    return code


def launch_count() -> int:
    return int(lib().anel_kernel_launch_count())


def tuning_report() -> str:
    """The autotuner's choices so far (anel_tuning_report)."""
    n = int(lib().anel_tuning_report(None, 0))
    buf = C.create_string_buffer(n + 1)
    lib().anel_tuning_report(buf, n + 1)
    return buf.value.decode()
