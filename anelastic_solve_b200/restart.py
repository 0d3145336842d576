"""Restart files in the reference's layout (ANELASTIC_SL/dns/Restart.F90).

``write``/``read`` move host arrays through the library's codec (no GPU);
``NSSolver.write_restart``/``read_restart`` move a stepper context's
device fields.  ``filename`` builds the names the reference gives them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from ._lib import check, lib

__all__ = ["filename", "write", "read", "header"]


def filename(basename: str, nstep: int, coords=None) -> str:
    """write_flow_small: basename//nstep; write_flow_big (coords given):
    basename//c1_c2_c3.nstep (concati writes an integer without padding,
    utils/string.F90:37-77)."""
    if coords is None:
        return f"{basename}{int(nstep)}"
    c1, c2, c3 = (int(c) for c in coords)
    return f"{basename}{c1}_{c2}_{c3}.{int(nstep)}"


def header(nstep=1, time=0.0, delt=0.0, g=0.0, rho_0=0.0, scal1_0=0.0, Re=1.0, Pr=1.0, Sc=1.0):
    h = abi.RestartHeader()
    h.nstep = int(nstep)
    for k, v in (("time", time), ("delt", delt), ("g", g), ("rho_0", rho_0), ("scal1_0", scal1_0),
                 ("Re", Re), ("Pr", Pr), ("Sc", Sc)):
        setattr(h, k, float(v))
    return h


def _dims(fields):
    X, Y, Z = fields["u"].shape
    return X - 2, Y - 2, Z - 2


def write(path, fields: dict, hdr: abi.RestartHeader, layout: int = abi.RESTART_SMALL):
    """Write the six ghosted fields (Fortran-ordered float64 arrays)."""
    nx, ny, nz = _dims(fields)
    arrs = [np.asfortranarray(fields[k], dtype=np.float64) for k in abi.RESTART_FIELDS]
    ptrs = (C.POINTER(C.c_double) * 6)(*[abi.dptr(a) for a in arrs])
    check(lib().anel_restart_write(os.fsencode(path), int(layout), C.byref(hdr), nx, ny, nz, ptrs))


def read(path, shape, layout: int = abi.RESTART_SMALL):
    """Read a file for interior sizes shape = (nx, ny, nz): (header, fields)."""
    nx, ny, nz = (int(v) for v in shape)
    arrs = [np.zeros((nx + 2, ny + 2, nz + 2), order="F") for _ in abi.RESTART_FIELDS]
    ptrs = (C.POINTER(C.c_double) * 6)(*[abi.dptr(a) for a in arrs])
    h = abi.RestartHeader()
    check(lib().anel_restart_read(os.fsencode(path), int(layout), C.byref(h), nx, ny, nz, ptrs))
    return h, dict(zip(abi.RESTART_FIELDS, arrs))
