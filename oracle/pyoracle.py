"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, as the checker.  The product package
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from anelastic_solve_b200 import abi

_HERE = Path(__file__).resolve().parent
_LIB = None


def build() -> Path:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _HERE / "liboracle.so"


def lib():
    global _LIB
    if _LIB is None:
        so = _HERE / "liboracle.so"
        if not so.exists():
            build()
        L = C.CDLL(str(so))
        L.orc_mg_create.restype = C.c_void_p
        L.orc_mg_create.argtypes = [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams),
                                    C.POINTER(C.c_int)]
        L.orc_mg_destroy.argtypes = [C.c_void_p]
        L.orc_mg_set_density.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_mg_solve.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_mg_debug_pass.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        L.orc_mg_levels.restype = C.c_int
        L.orc_mg_levels.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.orc_mg_true_resid.restype = C.c_double
        L.orc_mg_true_resid.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_mg_apply.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _LIB = L
    return _LIB


def _f(a: np.ndarray) -> np.ndarray:
    if not (a.dtype == np.float64 and a.flags.f_contiguous):
        raise TypeError("oracle fields must be Fortran-ordered float64 arrays")
    return a


class OracleMG:
    """mg_read_params + MG_init + mg_solver of the reference, on the CPU."""

    def __init__(self, grid, params: abi.MGParams):
        self._desc, self._keep = abi.make_grid_desc(grid)
        self.params = params
        st = C.c_int(0)
        self._h = lib().orc_mg_create(C.byref(self._desc), C.byref(params), C.byref(st))
        self.stat = st.value
        self.grid = grid
        if self.stat != 0:
            lib().orc_mg_destroy(self._h)
            self._h = None
            raise ValueError(f"oracle MG_init failed, stat={self.stat}")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_mg_destroy(self._h)
            self._h = None

    def set_density(self, r: np.ndarray):
        lib().orc_mg_set_density(self._h, abi.dptr(_f(r)))

    def solve(self, phi: np.ndarray, rhs: np.ndarray):
        """In place on phi (and clobbers rhs, like the reference)."""
        it = C.c_int(0)
        rm = C.c_double(0)
        lib().orc_mg_solve(self._h, abi.dptr(_f(phi)), abi.dptr(_f(rhs)), C.byref(it), C.byref(rm))
        return it.value, rm.value

    def debug_pass(self, which: int, phi: np.ndarray, src: np.ndarray):
        lib().orc_mg_debug_pass(self._h, which, abi.dptr(_f(phi)), abi.dptr(_f(src)))

    def levels(self) -> np.ndarray:
        out = (C.c_int * (12 * abi.MAX_LEVELS))()
        n = lib().orc_mg_levels(self._h, out, abi.MAX_LEVELS)
        return np.array(out[: 12 * n], dtype=np.int64).reshape(n, 12)

    def true_resid(self, phi, f) -> float:
        return lib().orc_mg_true_resid(self._h, abi.dptr(_f(phi)), abi.dptr(_f(f)))

    def apply(self, phi) -> np.ndarray:
        out = np.zeros_like(phi, order="F")
        lib().orc_mg_apply(self._h, abi.dptr(_f(phi)), abi.dptr(out))
        return out


def _ns_lib():
    L = lib()
    if not hasattr(L, "_ns_ready"):
        L.orc_ns_create.restype = C.c_void_p
        L.orc_ns_create.argtypes = [C.POINTER(abi.GridDesc), C.POINTER(abi.MGParams),
                                    C.POINTER(abi.NSParams), C.POINTER(C.c_int)]
        L.orc_ns_destroy.argtypes = [C.c_void_p]
        L.orc_ns_bind.argtypes = [C.c_void_p, C.POINTER(abi.Fields)]
        L.orc_ns_set_clock.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.orc_ns_substep.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_ns_step.argtypes = [C.c_void_p, C.POINTER(abi.StepReport)]
        L.orc_ns_project.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_ns_divergence.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_ns_ghost.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        L.orc_ns_rhs.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.orc_ns_cn.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                C.c_double, C.c_int]
        L.orc_ns_les_update.argtypes = [C.c_void_p]
        L.orc_ns_diagnostics.restype = C.c_int
        L.orc_ns_diagnostics.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L._ns_ready = True
    return L


class OracleNS:
    """rk_ss / NSsolver of the reference on the CPU, in place on a dict of
    Fortran-ordered host fields (names of abi.FIELD_NAMES)."""

    def __init__(self, grid, mgp: abi.MGParams, nsp: abi.NSParams, fields: dict):
        L = _ns_lib()
        self._desc, self._keep = abi.make_grid_desc(grid)
        st = C.c_int(0)
        self._h = L.orc_ns_create(C.byref(self._desc), C.byref(mgp), C.byref(nsp), C.byref(st))
        if st.value != 0:
            raise ValueError(f"oracle NS init failed, stat={st.value}")
        self.fields = fields
        fs = abi.Fields()
        for n in abi.FIELD_NAMES:
            a = fields.get(n)
            if a is not None:
                setattr(fs, n, abi.dptr(_f(a)))
        self._fs = fs
        L.orc_ns_bind(self._h, C.byref(fs))

    def __del__(self):
        if getattr(self, "_h", None):
            _ns_lib().orc_ns_destroy(self._h)
            self._h = None

    def set_clock(self, time: float, nstep: int):
        _ns_lib().orc_ns_set_clock(self._h, time, nstep)

    def substep(self, a1, a2, a3, dt_rk, dt):
        it = C.c_int(0)
        rm = C.c_double(0)
        _ns_lib().orc_ns_substep(self._h, a1, a2, a3, dt_rk, dt, C.byref(it), C.byref(rm))
        return it.value, rm.value

    def step(self) -> abi.StepReport:
        rep = abi.StepReport()
        _ns_lib().orc_ns_step(self._h, C.byref(rep))
        return rep

    def project(self):
        it = C.c_int(0)
        rm = C.c_double(0)
        _ns_lib().orc_ns_project(self._h, C.byref(it), C.byref(rm))
        return it.value, rm.value

    def divergence(self):
        out = (C.c_double * 2)()
        _ns_lib().orc_ns_divergence(self._h, out)
        return out[0], out[1]

    def ghost(self, a, vt: int):
        _ns_lib().orc_ns_ghost(self._h, abi.dptr(_f(a)), vt)

    def crank_nicolson(self, q: np.ndarray, u: np.ndarray, a3: float, rkdt: float, var: int) -> np.ndarray:
        """var_advance_CN_PL(q, u, 1, a3, 1, rkdt, var) on copies: the
        solved, ghosted field (var 1 u, 2 v, 3 w, 5 rho, 8 scal1)."""
        out = np.array(u, dtype=np.float64, order="F", copy=True)
        qq = np.array(q, dtype=np.float64, order="F", copy=True)
        _ns_lib().orc_ns_cn(self._h, abi.dptr(qq), abi.dptr(out), a3, rkdt, var)
        return out

    def les_update(self):
        """The model coefficients and SGSdiff's nuT, kappaT, nappaT from the
        current fields (into the bound arrays)."""
        _ns_lib().orc_ns_les_update(self._h)

    RHS = ("u", "v", "w", "rho", "scal1")

    def rhs(self, name: str) -> np.ndarray:
        """The explicit right-hand side of one field (u1_rhs .. scal1_rhs)
        on the current fields, ghosted as the routine leaves it."""
        out = np.zeros_like(self.fields["u"], order="F")
        _ns_lib().orc_ns_rhs(self._h, self.RHS.index(name), abi.dptr(out))
        return out

    def diagnostics(self, mode: int = abi.DIAG_LITERAL, stretched=(0, 0, 1)) -> dict:
        """The driver's per-step plane statistics (NSsolver.F90:288-395) on
        the current fields: {name: profile of nz+2 values} for
        abi.DIAG_NAMES."""
        Z = self._desc.nz + 2
        out = np.zeros(16 * Z)
        st = (C.c_int * 3)(*[int(v) for v in stretched])
        r = _ns_lib().orc_ns_diagnostics(self._h, int(mode == abi.DIAG_CORRECTED), st,
                                         out.ctypes.data_as(C.POINTER(C.c_double)))
        if r != 0:
            raise ValueError("a stretched axis needs at least 4 cells")
        return {n: out[q * Z:(q + 1) * Z].copy() for q, n in enumerate(abi.DIAG_NAMES)}
