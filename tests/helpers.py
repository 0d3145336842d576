"""Shared builders for the tests: grids, seeded fields, parameters."""
from __future__ import annotations

import numpy as np

from anelastic_solve_b200 import abi
from anelastic_solve_b200 import grid as G

# face order of tbc/vbc: X2max X3min X2min X3max X1min X1max
PERIODIC_XY_NEUMANN_Z = (0, 1, 0, 1, 0, 0)


def field(g: G.Grid, rng=None, scale=1.0) -> np.ndarray:
    """Seeded Fortran-ordered ghosted float64 field."""
    rng = rng if rng is not None else np.random.default_rng(0)
    return np.asfortranarray(scale * rng.standard_normal(g.ghosted))


def zeros(g: G.Grid) -> np.ndarray:
    return np.zeros(g.ghosted, order="F")


def remove_mean(a: np.ndarray) -> np.ndarray:
    out = a.copy(order="F")
    out[1:-1, 1:-1, 1:-1] -= out[1:-1, 1:-1, 1:-1].mean()
    return out


def small_grid(nx=16, ny=8, nz=16, stretched=False) -> G.Grid:
    return G.shear_layer_grid(nx, ny, nz, stretched=stretched)


def levels_for(g: G.Grid, coarsest=2):
    """Per-direction level counts giving a coarsest grid of `coarsest` cells
    (or the smallest power-of-two divisor otherwise)."""
    out = []
    for n in g.shape:
        L = 1
        while n % 2 == 0 and n // 2 >= coarsest:
            n //= 2
            L += 1
        out.append(L)
    return tuple(out)


def mg_params(g: G.Grid, **kw) -> abi.MGParams:
    kw.setdefault("levels", levels_for(g))
    kw.setdefault("tbc", PERIODIC_XY_NEUMANN_Z)
    return abi.make_mg_params(**kw)


def rel_l2(a, b, interior=True):
    if interior:
        a = a[1:-1, 1:-1, 1:-1]
        b = b[1:-1, 1:-1, 1:-1]
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def remove_vmean(a: np.ndarray, g: G.Grid) -> np.ndarray:
    """Subtract the volume-weighted interior mean (the compatibility
    condition of the metric operator, whose left null vector is the cell
    volume)."""
    vol = (g.x.dxc[1:-1, None, None] * g.y.dxc[None, 1:-1, None] * g.z.dxc[None, None, 1:-1])
    out = a.copy(order="F")
    inner = out[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    return out


def compatible(a: np.ndarray, g: G.Grid, mode: int) -> np.ndarray:
    return remove_vmean(a, g) if mode == abi.MODE_METRIC else remove_mean(a)
