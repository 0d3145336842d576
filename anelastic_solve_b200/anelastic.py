"""Anelastic background profiles of the reference (set_densityBG,
ANELASTIC_SL/dns/IC.F90:1062-1096), which the reference's initialisation
always calls (dns/initialize.F90:59).

At every cell, with zz = zc(k) - X3center:
    tz   = 300.0 - 0.0065 zz
    qv0  = 0.0115 - 0.000002 zz
    pz   = 101325.0 exp(5.5547 log(46153.8 - zz) - 2.28088 log(317030.0 - zz) - 30.7647)
    densityBG = tz / (pz/101325.0)**(287.1/1004.0)
    r    = pz (1.0 + qv0) / (Rd tz (1.0 + qv0/evv)),  Rd = 287.1, Rv = 461.5, evv = Rd/Rv
The source writes its constants as default (single precision) REAL
literals: each is rounded to float32 and widened where it meets a double,
and 287.1/1004.0 is a single-precision quotient.  Rd and Rv are double
variables assigned from such literals.  log/exp/pow are the C library's,
as in the compiled reference.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["background_profiles", "set_density_bg"]


def _f(x: float) -> float:
    """A default REAL literal: rounded to float32, widened to double."""
    return float(np.float32(x))


RV = _f(461.5)
RD = _f(287.1)
EVV = RD / RV
KAPPA = float(np.float32(287.1) / np.float32(1004.0))  # single-precision quotient


def background_profiles(zc, x3center: float = 0.0) -> dict:
    """Profiles tz, qv0, pz, densityBG, r at the cell centres zc (the
    ghosted z axis, k = 1..nz+2)."""
    out = {k: np.empty(len(zc)) for k in ("tz", "qv0", "pz", "densityBG", "r")}
    for k, z in enumerate(zc):
        zz = float(z) - float(x3center)
        tz = 300.0 - _f(0.0065) * zz
        qv0 = _f(0.0115) - _f(0.000002) * zz
        pz = 101325.0 * math.exp(_f(5.5547) * math.log(_f(46153.8) - zz)
                                 - _f(2.28088) * math.log(317030.0 - zz) - _f(30.7647))
        out["tz"][k] = tz
        out["qv0"][k] = qv0
        out["pz"][k] = pz
        out["densityBG"][k] = tz / math.pow(pz / 101325.0, KAPPA)
        out["r"][k] = pz * (1.0 + qv0) / (RD * tz * (1.0 + qv0 / EVV))
    return out


def set_density_bg(fields: dict, grid, x3center: float = 0.0) -> dict:
    """Fill fields["r"] and fields["densityBG"] (ghosted, Fortran order) with
    the horizontally uniform profiles, as set_densityBG does on the whole
    array (ghosts included).  Returns the z profiles."""
    prof = background_profiles(grid.z.xc, x3center)
    for name in ("r", "densityBG"):
        fields[name][...] = prof[name][None, None, :]
    return prof
