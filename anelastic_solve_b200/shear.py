"""Seeded initial state of the temporally evolving stratified shear layer.

Mean flow U = tanh(z) (u at (xe, yc, zc)), rho = -tanh(z) at cell centres,
v = w = 0, plus uniform noise amp*(2U[0,1)-1) on u, v, w where |zc| < 2.
The uniform numbers come from the Park-Miller "minimal standard"
generator (x <- 16807 x mod 2^31-1, U = x/(2^31-1); Park & Miller, CACM
31(10), 1988), the method of ANELASTIC_SL/dns/isoSpec.F90:1484-1531,
drawn in Fortran order (i fastest) for u, then v, then w.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

_M = 2147483647
_A = 16807


def park_miller(seed: int, n: int) -> np.ndarray:
    """n uniform numbers in (0,1) from the minimal standard generator,
    computed in blocks: x_{b+t} = x_b * a^t mod m."""
    out = np.empty(n, dtype=np.float64)
    x = int(seed) % _M or 1
    blk = 1 << 16
    pw = np.empty(blk, dtype=np.int64)
    p = 1
    for t in range(blk):
        p = (p * _A) % _M
        pw[t] = p  # a^(t+1)
    q = 0
    while q < n:
        m = min(blk, n - q)
        vals = _mulmod(x, pw[:m])
        out[q:q + m] = vals / _M
        x = int(vals[-1])
        q += m
    return out


def _mulmod(x: int, powers: np.ndarray) -> np.ndarray:
    """(x * p) mod (2^31-1) for an int64 array p, without overflow."""
    x_hi, x_lo = x >> 16, x & 0xFFFF
    hi = ((powers * x_hi) % _M) * 65536 % _M
    lo = (powers * x_lo) % _M
    return (hi + lo) % _M


def shear_layer_fields(grid, amp: float = 1e-3, seed: int = 12345, zmax: float = 2.0):
    """Dict of Fortran-ordered ghosted FP64 fields (ghosts unset: the caller
    ghosts/projects).  r = densityBG = 1 (Boussinesq limit)."""
    sh = grid.ghosted
    zc = grid.z.xc
    f = {n: np.zeros(sh, order="F") for n in abi.FIELD_NAMES}
    # tanh per level by the C library (not numpy's vectorised tanh), so the
    # device generator of the serving engine reproduces this state exactly
    th = np.array([math.tanh(z) for z in zc])
    f["u"][:] = th[None, None, :]
    f["rho"][:] = -th[None, None, :]
    f["r"][:] = 1.0
    f["densityBG"][:] = 1.0
    mask = (np.abs(zc) < zmax)[None, None, :]
    N = int(np.prod(sh))
    rnd = park_miller(seed, 3 * N)
    for q, name in enumerate(("u", "v", "w")):
        pert = (amp * (2.0 * rnd[q * N:(q + 1) * N] - 1.0)).reshape(sh, order="F")
        f[name] += np.where(mask, pert, 0.0)
    return f
