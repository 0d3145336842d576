"""Python mirror of the reference multigrid interface (mgMK).

The reference drives its solver through ``mg_read_params(ini, stat)``,
``MG_init(stat)``, ``mg_solver(phif, rhsf, iter, relmax)`` and
``mg_end(ierr)`` (ANELASTIC_SL/mgMK/mg_read_params.F90, mg_init.F90,
mg_solver.F90, mg_end.F90).  :class:`MGSolver` keeps those names and
argument meanings on top of the C-ABI context calls of include/anel.h; the
arithmetic runs in the sm_100a kernels of libanel.so (no CPU fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import AnelError, check, lib

__all__ = ["MGSolver", "AnelError"]


def _is_torch_cuda(t) -> bool:
    return type(t).__module__.startswith("torch") and getattr(t, "is_cuda", False)


def _ptr(a):
    """(pointer, mem) for a Fortran-ordered float64 numpy array or a
    contiguous float64 CUDA torch tensor holding a Fortran-ordered field."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.f_contiguous:
            raise TypeError("host fields must be Fortran-ordered float64 numpy arrays")
        return a.ctypes.data_as(C.POINTER(C.c_double)), abi.MEM_HOST
    if _is_torch_cuda(a):
        import torch

        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("device fields must be contiguous float64 CUDA tensors")
        return C.cast(C.c_void_p(a.data_ptr()), C.POINTER(C.c_double)), abi.MEM_DEVICE
    if isinstance(a, int):
        return C.cast(C.c_void_p(a), C.POINTER(C.c_double)), abi.MEM_DEVICE
    raise TypeError(f"unsupported field type {type(a)}")


class MGSolver:
    """One multigrid context (the state MG_init builds) on one GPU.

    ``grid`` is an :class:`anelastic_solve_b200.grid.Grid`; ``params`` an
    :class:`anelastic_solve_b200.abi.MGParams` (see ``abi.make_mg_params``).
    """

    def __init__(self, grid, params: abi.MGParams, device: int = 0):
        self._desc, self._keep = abi.make_grid_desc(grid)
        self.params = params
        self.grid = grid
        st = C.c_int32(0)
        self._h = lib().anel_mg_create(C.byref(self._desc), C.byref(params), int(device), C.byref(st))
        if not self._h:
            raise AnelError(st.value, lib().anel_last_error().decode())
        self.last_report = abi.MGReport()

    def close(self):
        if getattr(self, "_h", None):
            lib().anel_mg_destroy(self._h)
            self._h = None

    __del__ = close

    def set_density(self, r):
        p, mem = _ptr(r)
        check(lib().anel_mg_ctx_set_density(self._h, p, mem))

    def solve(self, phif, rhsf, stream=None, allow_noconv: bool = True):
        """mg_solver(phif, rhsf, iter, relmax): phif updated in place.
        Returns (iter, relmax); the full report is in ``last_report``."""
        pp, m1 = _ptr(phif)
        pr, m2 = _ptr(rhsf)
        if m1 != m2:
            raise TypeError("phif and rhsf must live in the same memory space")
        s = C.c_void_p(int(stream)) if stream is not None else None
        rep = abi.MGReport()
        allow = (abi.OK, abi.ERR_NOCONV) if allow_noconv else (abi.OK,)
        check(lib().anel_mg_ctx_solve(self._h, pp, pr, m1, s, C.byref(rep)), allow)
        self.last_report = rep
        return rep.iter, rep.relmax

    def solve_batch(self, phis, rhss, stream=None, allow_noconv: bool = True):
        """anel_mg_ctx_solve_batch: the device arrays phis[b] updated in
        place from rhss[b], all members in one batched solve.  Returns the
        members' reports."""
        n = len(phis)
        if n != len(rhss) or n < 1:
            raise ValueError("phis and rhss must be non-empty and of equal length")
        dp = C.POINTER(C.c_double)
        pp = (dp * n)()
        pr = (dp * n)()
        for b in range(n):
            p1, m1 = _ptr(phis[b])
            p2, m2 = _ptr(rhss[b])
            if m1 != abi.MEM_DEVICE or m2 != abi.MEM_DEVICE:
                raise TypeError("batched solves take device arrays")
            pp[b] = p1
            pr[b] = p2
        s = C.c_void_p(int(stream)) if stream is not None else None
        reps = (abi.MGReport * n)()
        allow = (abi.OK, abi.ERR_NOCONV) if allow_noconv else (abi.OK,)
        check(lib().anel_mg_ctx_solve_batch(self._h, n, pp, pr, s, reps), allow)
        return list(reps)

    def set_profiling(self, on: bool):
        check(lib().anel_mg_ctx_set_profiling(self._h, 1 if on else 0))

    def levels(self) -> np.ndarray:
        out = (C.c_int32 * (12 * abi.MAX_LEVELS))()
        n = lib().anel_mg_ctx_levels(self._h, out, abi.MAX_LEVELS)
        return np.array(out[: 12 * n], dtype=np.int64).reshape(n, 12)

    def debug_pass(self, which: int, phi_dev, src_dev, stream=None):
        pp, m1 = _ptr(phi_dev)
        ps, m2 = _ptr(src_dev)
        if m1 != abi.MEM_DEVICE or m2 != abi.MEM_DEVICE:
            raise TypeError("debug passes take device arrays")
        s = C.c_void_p(int(stream)) if stream is not None else None
        check(lib().anel_mg_ctx_debug_pass(self._h, which, pp, ps, s))
