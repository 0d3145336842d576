"""Python mirror of the reference time stepper (NSsolver / rk_ss).

The reference advances its module fields with ``rk_ss(a1, a2, a3, ec,
dt_rk, dt, psolve, stat)`` three times per ``NSsolver`` step
(ANELASTIC_SL/dns/NSsolver.F90:63-583).  :class:`NSSolver` keeps the fields
on one GPU and exposes the same sub-step and step, running the sm_100a
kernels of libanel.so (no CPU fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import AnelError, check, lib
from .mg import _ptr

__all__ = ["NSSolver", "RK3"]

# Williamson low-storage RK3 coefficients (a1, a2, a3, ec, dt_rk/dt),
# NSsolver.F90:198-261
RK3 = ((0.0, 1.0, 1.0 / 3.0, -1.0 / 6.0, 1.0 / 3.0),
       (-5.0 / 9.0, 1.0, 15.0 / 16.0, -10.0 / 3.0, 5.0 / 12.0),
       (-153.0 / 128.0, 1.0, 8.0 / 15.0, 15.0 / 8.0, 1.0 / 4.0))


class NSSolver:
    def __init__(self, grid, mgp: abi.MGParams, nsp: abi.NSParams, device: int = 0):
        self._desc, self._keep = abi.make_grid_desc(grid)
        self.grid, self.mgp, self.nsp = grid, mgp, nsp
        st = C.c_int32(0)
        self._h = lib().anel_ns_create(C.byref(self._desc), C.byref(mgp), C.byref(nsp), int(device),
                                       C.byref(st))
        if not self._h:
            raise AnelError(st.value, lib().anel_last_error().decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().anel_ns_destroy(self._h)
            self._h = None

    __del__ = close

    def _fields(self, d: dict):
        fs = abi.Fields()
        mem = None
        for name, a in d.items():
            if a is None:
                continue
            p, m = _ptr(a)
            if mem is not None and m != mem:
                raise TypeError("all fields of one call must live in the same memory space")
            mem = m
            setattr(fs, name, p)
        return fs, (abi.MEM_HOST if mem is None else mem)

    def set_fields(self, d: dict):
        fs, mem = self._fields(d)
        check(lib().anel_ns_set_fields(self._h, C.byref(fs), mem))

    def get_fields(self, names=("u", "v", "w", "p", "rho", "scal1")) -> dict:
        out = {n: np.zeros(self.grid.ghosted, order="F") for n in names}
        fs, mem = self._fields(out)
        check(lib().anel_ns_get_fields(self._h, C.byref(fs), mem))
        return out

    def get_into(self, d: dict):
        fs, mem = self._fields(d)
        check(lib().anel_ns_get_fields(self._h, C.byref(fs), mem))

    def substep(self, a1, a2, a3, dt_rk, dt, stream=None):
        it = C.c_int32(0)
        rm = C.c_double(0)
        s = C.c_void_p(int(stream)) if stream is not None else None
        check(lib().anel_ns_ctx_substep(self._h, a1, a2, a3, dt_rk, dt, s, C.byref(it), C.byref(rm)))
        return it.value, rm.value

    def step(self, n: int = 1, stream=None) -> abi.StepReport:
        rep = abi.StepReport()
        s = C.c_void_p(int(stream)) if stream is not None else None
        check(lib().anel_ns_ctx_step(self._h, int(n), s, C.byref(rep)))
        return rep

    @staticmethod
    def step_cohort(members, n: int = 1, batch=None, stream=None):
        """n steps of every NSSolver in members together, the pressure
        solves of each sub-step batched (anel_ns_ctx_step_cohort); batch: an
        MGSolver of the members' grid and multigrid parameters, or None for
        the first member's own.  Returns the members' reports."""
        k = len(members)
        hs = (C.c_void_p * k)(*[m._h for m in members])
        reps = (abi.StepReport * k)()
        s = C.c_void_p(int(stream)) if stream is not None else None
        b = batch._h if batch is not None else None
        check(lib().anel_ns_ctx_step_cohort(hs, k, int(n), b, s, reps))
        return list(reps)

    def step_host(self, fields_in: dict, fields_out: dict, n: int = 1, stream=None) -> abi.StepReport:
        """n steps from host arrays fields_in to host arrays fields_out (may
        be the same dict), copies overlapped with the step where the data
        allow it (anel_ns_ctx_step_host).  Use pinned arrays for
        asynchronous copies."""
        fi, mi = self._fields(fields_in)
        fo, mo = self._fields(fields_out)
        if mi != abi.MEM_HOST or mo != abi.MEM_HOST:
            raise TypeError("step_host takes host arrays")
        rep = abi.StepReport()
        s = C.c_void_p(int(stream)) if stream is not None else None
        check(lib().anel_ns_ctx_step_host(self._h, C.byref(fi), C.byref(fo), int(n), s, C.byref(rep)))
        return rep

    def set_profiling(self, on: bool):
        check(lib().anel_ns_ctx_set_profiling(self._h, 1 if on else 0))

    def set_clock(self, time: float, nstep: int):
        check(lib().anel_ns_ctx_set_clock(self._h, float(time), int(nstep)))

    def project(self):
        it = C.c_int32(0)
        rm = C.c_double(0)
        check(lib().anel_ns_ctx_project(self._h, C.byref(it), C.byref(rm)))
        return it.value, rm.value

    def divergence(self):
        out = (C.c_double * 2)()
        check(lib().anel_ns_ctx_divergence(self._h, out))
        return out[0], out[1]

    def set_diagnostics(self, on: bool = True, mode: int = abi.DIAG_LITERAL, stretched=(0, 0, 1)):
        """Run the driver's per-step plane statistics (NSsolver.F90:288-395)
        after every step(); ``stretched[d]`` marks the axes whose grid file
        says 'stretched'."""
        st = (C.c_int32 * 3)(*[int(v) for v in stretched])
        check(lib().anel_ns_ctx_set_diagnostics(self._h, 1 if on else 0, int(mode), st))

    def compute_diagnostics(self):
        """One pass of the plane statistics on the current fields."""
        check(lib().anel_ns_ctx_compute_diagnostics(self._h, None))

    def write_restart(self, path, hdr: abi.RestartHeader, layout: int = abi.RESTART_SMALL):
        """The context's u, v, w, p, rho, scal1 to a restart file in the
        reference's layout (Restart.F90)."""
        import os

        check(lib().anel_ns_ctx_write_restart(self._h, os.fsencode(path), int(layout), C.byref(hdr)))

    def read_restart(self, path, layout: int = abi.RESTART_SMALL, icparam: bool = True):
        """Load a restart file into the context (fields ghosted as the
        reference's start_small/start_big do); with icparam the clock
        (time, nstep) comes from the file.  Returns the header."""
        import os

        h = abi.RestartHeader()
        check(lib().anel_ns_ctx_read_restart(self._h, os.fsencode(path), int(layout), 1 if icparam else 0,
                                             C.byref(h)))
        return h

    def diagnostics(self) -> dict:
        """{name: profile of nz+2 values (k = 1..nz+2)} for abi.DIAG_NAMES."""
        Z = self._desc.nz + 2
        out = np.zeros(16 * Z)
        check(lib().anel_ns_ctx_get_diagnostics(self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                                abi.MEM_HOST))
        return {n: out[q * Z:(q + 1) * Z].copy() for q, n in enumerate(abi.DIAG_NAMES)}
