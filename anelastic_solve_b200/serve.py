"""Serving engine for ensembles of independent shear-layer members and
standalone pressure solves.

Thin Python face of the native engine of include/anel.h
(``anel_serve_*``, csrc/serve.cu): requests queue in FIFO order, worker
threads of the library run them per bucket (grid, models, multigrid setup)
-- shear-layer members as cohorts stepping together with batched pressure
solves, standalone solves in batches -- and requests are admitted against
an HBM budget with contexts pooled per bucket.  Not a reference routine:
each reference run is its own job.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import AnelError, check, lib

__all__ = ["ServeEngine"]


class ServeEngine:
    def __init__(self, hbm_budget_bytes: int, max_active: int = 8, device: int = 0):
        st = C.c_int32(0)
        self._h = lib().anel_serve_create(int(device), int(hbm_budget_bytes), int(max_active),
                                          C.byref(st))
        if not self._h:
            raise AnelError(st.value, lib().anel_last_error().decode())
        self._keep = {}  # id -> objects the native side points into

    def submit(self, grid, mg: abi.MGParams, ns: abi.NSParams, nsteps: int, seed: int = 12345,
               amp: float = 1e-3, fields_in: dict | None = None, want_fields: bool = False) -> int:
        """Queue one member; returns its id.  With want_fields the fields
        after the last step come back from poll() under ``fields``."""
        desc, keep = abi.make_grid_desc(grid)
        req = abi.Request()
        req.grid = desc
        req.mg = mg
        req.ns = ns
        req.nsteps = int(nsteps)
        req.seed = int(seed) & 0xFFFFFFFF
        req.amp = float(amp)
        hold = [keep, req]
        if fields_in is not None:
            req.init = abi.INIT_FIELDS
            fin = abi.Fields()
            for k, a in fields_in.items():
                a = np.asfortranarray(a, dtype=np.float64)
                hold.append(a)
                setattr(fin, k, abi.dptr(a))
            hold.append(fin)
            req.fields_in = C.pointer(fin)
        else:
            req.init = abi.INIT_SHEAR
        out = None
        if want_fields:
            out = {k: np.zeros(grid.ghosted, order="F") for k in ("u", "v", "w", "p", "rho")}
            fo = abi.Fields()
            for k, a in out.items():
                setattr(fo, k, abi.dptr(a))
            hold.append(fo)
            req.fields_out = C.pointer(fo)
        rid = C.c_int64(0)
        check(lib().anel_serve_submit(self._h, C.byref(req), C.byref(rid)))
        self._keep[rid.value] = (hold, out)
        return rid.value

    def submit_poisson(self, grid, mg: abi.MGParams, rhs, phi0=None, want_solution: bool = True) -> int:
        """Queue one standalone pressure solve (ANEL_INIT_POISSON): the
        ghosted FP64 right-hand side rhs, the initial guess phi0 (None:
        zero).  Requests of one grid and multigrid setup are solved
        together in batches.  With want_solution the solution comes back
        from poll() under ``fields["p"]``; ``mg_iter`` and ``resid`` carry
        the solve's report."""
        desc, keep = abi.make_grid_desc(grid)
        req = abi.Request()
        req.grid = desc
        req.mg = mg
        req.ns = abi.make_ns_params()
        req.init = abi.INIT_POISSON
        hold = [keep, req]
        fin = abi.Fields()
        f = np.asfortranarray(rhs, dtype=np.float64)
        hold.append(f)
        fin.psrc = abi.dptr(f)
        if phi0 is not None:
            p0 = np.asfortranarray(phi0, dtype=np.float64)
            hold.append(p0)
            fin.p = abi.dptr(p0)
        hold.append(fin)
        req.fields_in = C.pointer(fin)
        out = None
        if want_solution:
            out = {"p": np.zeros(grid.ghosted, order="F")}
            fo = abi.Fields()
            fo.p = abi.dptr(out["p"])
            hold.append(fo)
            req.fields_out = C.pointer(fo)
        rid = C.c_int64(0)
        check(lib().anel_serve_submit(self._h, C.byref(req), C.byref(rid)))
        self._keep[rid.value] = (hold, out)
        return rid.value

    def poll(self, wait_ms: int = 0, cap: int = 256) -> list[dict]:
        buf = (abi.Result * cap)()
        n = C.c_int32(0)
        check(lib().anel_serve_poll(self._h, buf, cap, C.byref(n), int(wait_ms)))
        res = []
        for q in range(n.value):
            r = buf[q]
            d = {f: getattr(r, f) for f, _ in abi.Result._fields_}
            _, out = self._keep.pop(r.id, (None, None))
            d["fields"] = out
            res.append(d)
        return res

    def drain(self):
        check(lib().anel_serve_drain(self._h))

    def stats(self) -> dict:
        st = abi.ServeStats()
        check(lib().anel_serve_stats_get(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in abi.ServeStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().anel_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
