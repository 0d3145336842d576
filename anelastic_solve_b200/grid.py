"""Staggered-grid metric arrays and the reference's grid-file format.

A direction with ``n`` interior cells is described by six arrays of length
``n + 2`` (Fortran indices 1..n+2, ghost cells at both ends), exactly the
arrays ``load_grid`` reads from ``x?_grid.in``
(ANELASTIC_SL/utils/loadGrid.F90:38-90):

* ``xe``  -- cell upper edge (face) coordinate: cell ``k`` spans ``xe(k-1)..xe(k)``
* ``xc``  -- cell centre
* ``dxe`` -- ``xc(k+1) - xc(k)`` (centre-to-centre spacing)
* ``dxc`` -- ``xe(k) - xe(k-1)`` (cell width)
* ``rdxe``, ``rdxc`` -- their reciprocals

The ghost cells mirror the width of their interior neighbour and the
end fix-ups of loadGrid.F90:79-90 are applied, so a grid built here and one
read back from a file written here are identical.
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path

import numpy as np

__all__ = ["Axis", "Grid", "uniform_axis", "tanh_axis", "write_grid_file", "read_grid_file",
           "shear_layer_grid"]


@dataclasses.dataclass
class Axis:
    n: int
    L: float
    xe: np.ndarray
    xc: np.ndarray
    dxe: np.ndarray
    dxc: np.ndarray
    rdxe: np.ndarray
    rdxc: np.ndarray
    x0: float = 0.0
    gridtype: str = "uniform"

    def arrays(self):
        return (self.xe, self.xc, self.dxe, self.dxc, self.rdxe, self.rdxc)


@dataclasses.dataclass
class Grid:
    x: Axis
    y: Axis
    z: Axis

    @property
    def shape(self):
        """(nx, ny, nz) interior cells."""
        return (self.x.n, self.y.n, self.z.n)

    @property
    def ghosted(self):
        """(nx+2, ny+2, nz+2); a field is stored Fortran-ordered with this shape."""
        return (self.x.n + 2, self.y.n + 2, self.z.n + 2)


def _axis_from_edges(edges: np.ndarray, gridtype: str) -> Axis:
    """``edges`` are the n+1 face coordinates xe(1..n+1) (bottom wall first)."""
    edges = np.asarray(edges, dtype=np.float64)
    n = edges.size - 1
    xe = np.empty(n + 2)
    xe[: n + 1] = edges
    dxc = np.empty(n + 2)
    dxc[1 : n + 1] = edges[1:] - edges[:-1]
    dxc[0] = dxc[1]
    dxc[n + 1] = dxc[n]
    xe[n + 1] = xe[n] + dxc[n + 1]
    xc = np.empty(n + 2)
    xc[1 : n + 1] = 0.5 * (edges[1:] + edges[:-1])
    xc[0] = xe[0] - 0.5 * dxc[0]
    xc[n + 1] = xe[n] + 0.5 * dxc[n + 1]
    dxe = np.empty(n + 2)
    dxe[: n + 1] = xc[1:] - xc[:-1]
    dxe[n + 1] = dxe[n]
    rdxe = 1.0 / dxe
    rdxc = 1.0 / dxc
    # loadGrid.F90:79-90 end fix-ups (idempotent for grids built here)
    dxc[n + 1] = dxc[n]
    rdxc[n + 1] = rdxc[n]
    dxe[n + 1] = dxe[n]
    rdxe[n + 1] = rdxe[n]
    dxc[0] = dxc[1]
    rdxc[0] = rdxc[1]
    dxe[0] = dxe[1]
    rdxe[0] = rdxe[1]
    xe[n + 1] = xe[n] + dxc[n + 1]
    xc[n + 1] = xc[n] + dxe[n]
    xe[0] = xe[1] - dxc[1]
    xc[0] = xc[1] - dxe[0]
    L = float(edges[-1] - edges[0])
    return Axis(n=n, L=L, xe=xe, xc=xc, dxe=dxe, dxc=dxc, rdxe=rdxe, rdxc=rdxc,
                x0=float(xc[0]), gridtype=gridtype)


def uniform_axis(n: int, L: float, start: float = 0.0) -> Axis:
    """Uniform spacing h = L/n starting at ``start``.  dxc, dxe and their
    reciprocals hold the single value h (1/h) at every index, as the
    reference's uniform grid files do (ANELASTIC_SL/run_dir/x?_grid.in), so
    the metric coefficients are bitwise identical along the axis."""
    h = L / n
    k = np.arange(n + 2, dtype=np.float64)
    xe = start + h * k          # xe(1) = start, xe(n+1) = start + L
    xc = start + h * (k - 0.5)
    d = np.full(n + 2, h)
    r = np.full(n + 2, 1.0 / h)
    return Axis(n=n, L=float(L), xe=xe, xc=xc, dxe=d.copy(), dxc=d.copy(), rdxe=r.copy(),
                rdxc=r.copy(), x0=float(xc[0]), gridtype="uniform")


def tanh_axis(n: int, half: float = 10.0, factor: float = 2.0) -> Axis:
    """tanh-stretched axis on [-half, half] (cells narrowest at the walls):
    ze_k = half * tanh(factor*s_k)/tanh(factor), s_k = -1 + 2(k-1)/n, k = 1..n+1."""
    s = -1.0 + 2.0 * np.arange(n + 1, dtype=np.float64) / n
    edges = half * np.tanh(factor * s) / math.tanh(factor)
    return _axis_from_edges(edges, "tanh")


def shear_layer_grid(nx: int, ny: int, nz: int, stretched: bool = True) -> Grid:
    """Shear-layer domain 4*pi x 2*pi x 20, periodic x,y; z tanh-stretched
    (factor 2 about z = 0) or uniform on [-10, 10]."""
    gx = uniform_axis(nx, 4.0 * math.pi)
    gy = uniform_axis(ny, 2.0 * math.pi)
    gz = tanh_axis(nz, 10.0, 2.0) if stretched else uniform_axis(nz, 20.0, -10.0)
    return Grid(gx, gy, gz)


def _fmt(v: float) -> str:
    return f"{v: .16E}".replace("E", "D")


def write_grid_file(path, axis: Axis, label: str = "X1") -> None:
    """Write the reference's x?_grid.in layout: 2 comment lines, nxp2, L,
    x0, Gridtype, then ``i xe xc dxe dxc rdxe rdxc`` per index."""
    lines = [f"#{label}-GRID",
             "#   i  xe  xc  dxe  dxc  rdxe  rdxc",
             f"{axis.n + 2:6d}", _fmt(axis.L), _fmt(axis.x0), f" {axis.gridtype}"]
    for i in range(axis.n + 2):
        lines.append(f"{i + 1:5d} " + " ".join(_fmt(a[i]) for a in axis.arrays()))
    Path(path).write_text("\n".join(lines) + "\n")


def read_grid_file(path) -> Axis:
    """Read an x?_grid.in file (loadGrid.F90:44-58) and apply the end fix-ups."""
    raw = Path(path).read_text().splitlines()
    nxp2 = int(raw[2].split()[0])
    L = float(raw[3].split()[0].replace("D", "E").replace("d", "e"))
    x0 = float(raw[4].split()[0].replace("D", "E").replace("d", "e"))
    gtype = raw[5].strip()
    cols = np.zeros((6, nxp2))
    for q in range(nxp2):
        parts = raw[6 + q].replace("D", "E").replace("d", "e").split()
        cols[:, q] = [float(t) for t in parts[1:7]]
    xe, xc, dxe, dxc, rdxe, rdxc = (c.copy() for c in cols)
    n = nxp2 - 2
    dxc[n + 1] = dxc[n]
    rdxc[n + 1] = rdxc[n]
    dxe[n + 1] = dxe[n]
    rdxe[n + 1] = rdxe[n]
    dxc[0] = dxc[1]
    rdxc[0] = rdxc[1]
    dxe[0] = dxe[1]
    rdxe[0] = rdxe[1]
    xe[n + 1] = xe[n] + dxc[n + 1]
    xc[n + 1] = xc[n] + dxe[n]
    xe[0] = xe[1] - dxc[1]
    xc[0] = xc[1] - dxe[0]
    return Axis(n=n, L=L, xe=xe, xc=xc, dxe=dxe, dxc=dxc, rdxe=rdxe, rdxc=rdxc, x0=x0,
                gridtype=gtype)
