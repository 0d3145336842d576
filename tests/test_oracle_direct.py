"""Direct solves pin the oracle's multigrid (CPU only).

The reference ships no solver outputs.  Besides ptest's analytic cases, the
oracle's fine-grid operators are therefore restated here in vectorised
numpy, straight from the reference's formulas.  The oracle's converged
multigrid solutions are then checked against a dense direct solve of the
restated system:

- metric mode: the operator is the projection's Psource(Pgrad(p))
  (Pgrad ANELASTIC_SL/dns/NSsolver.F90:2023-2085, Psource :2167-2223,
  dt = 1) with an anelastic density r(z) (set_densityBG,
  dns/IC.F90:1062-1096) on a tanh-stretched z axis; the walls carry no
  flux (w = 0 there);
- literal mode: mgdpfpde's coefficients (mgMK/mg_pfpde.F90:34-56) on a
  uniform grid, with mg_bdry's ghost rules for periodic and homogeneous
  Neumann faces (mgMK/mg_bdry.F90:72-190).

In each mode two things are checked.  The oracle's operator applied to a
random field agrees with the restatement to rounding.  The oracle's
multigrid solution, solved to a relative residual of 1e-13, agrees with the
direct solution modulo the operator's null space.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleMG

from .helpers import PERIODIC_XY_NEUMANN_Z, levels_for, remove_mean, remove_vmean


def _wrap_xy(a):
    """Periodic ghosts in x, then y (the face ghosts the 7-point stencil
    reads)."""
    a[0, :, :] = a[-2, :, :]
    a[-1, :, :] = a[1, :, :]
    a[:, 0, :] = a[:, -2, :]
    a[:, -1, :] = a[:, 1, :]


def _bcast(v, d):
    sl = [None, None, None]
    sl[d] = slice(None)
    return v[tuple(sl)]


def psource_pgrad(p, g, r):
    """div(r grad(p/r)) of the projection on the interior: Pgrad's face
    gradients, then Psource's divergence of r times them, dt = 1."""
    q = p / r
    # x, y faces: r cancels (r depends on z only)
    gx = (q[1:, 1:-1, 1:-1] - q[:-1, 1:-1, 1:-1]) * _bcast(g.x.rdxe[:-1], 0)
    gy = (q[1:-1, 1:, 1:-1] - q[1:-1, :-1, 1:-1]) * _bcast(g.y.rdxe[:-1], 1)
    gz = (q[1:-1, 1:-1, 1:] - q[1:-1, 1:-1, :-1]) * _bcast(g.z.rdxe[:-1], 2)
    rc = r[1:-1, 1:-1, :]
    rbar = 0.5 * (rc[:, :, 1:] + rc[:, :, :-1])      # r at the z faces 1..nz+1
    fz = rbar * gz                                   # r-weighted z fluxes
    fz[:, :, 0] = 0.0                                # walls: w = 0
    fz[:, :, -1] = 0.0
    rint = r[1:-1, 1:-1, 1:-1]
    out = (rint * (gx[1:, :, :] - gx[:-1, :, :])) * _bcast(g.x.rdxc[1:-1], 0)
    out = out + (rint * (gy[:, 1:, :] - gy[:, :-1, :])) * _bcast(g.y.rdxc[1:-1], 1)
    out = out + (fz[:, :, 1:] - fz[:, :, :-1]) * _bcast(g.z.rdxc[1:-1], 2)
    return out


def literal_apply(p, g):
    """mgdpfpde's operator with r = 1 on the interior: 1/dl^2 per direction,
    dl = L / float(n); ghosts from mg_bdry (periodic x, y; homogeneous
    Neumann z: the ghost repeats the first interior cell)."""
    a = p.copy(order="F")
    _wrap_xy(a)
    a[:, :, 0] = a[:, :, 1]
    a[:, :, -1] = a[:, :, -2]
    t = [1.0 / (ax.L / float(np.float32(ax.n))) ** 2 for ax in (g.x, g.y, g.z)]
    c = a[1:-1, 1:-1, 1:-1]
    return (t[0] * (a[:-2, 1:-1, 1:-1] + a[2:, 1:-1, 1:-1]) + t[1] * (a[1:-1, :-2, 1:-1] + a[1:-1, 2:, 1:-1])
            + t[2] * (a[1:-1, 1:-1, :-2] + a[1:-1, 1:-1, 2:]) - 2.0 * (t[0] + t[1] + t[2]) * c)


def dense_operator(apply, g):
    """The interior operator as a dense matrix, column by column (i fastest)."""
    nx, ny, nz = g.shape
    n = nx * ny * nz
    A = np.empty((n, n))
    e = np.zeros(g.ghosted, order="F")
    for col in range(n):
        i, j, k = col % nx, (col // nx) % ny, col // (nx * ny)
        e[1 + i, 1 + j, 1 + k] = 1.0
        A[:, col] = apply(e).reshape(-1, order="F")
        e[1 + i, 1 + j, 1 + k] = 0.0
    return A


def _interior(a):
    return a[1:-1, 1:-1, 1:-1].reshape(-1, order="F")


def _drop(v, null):
    """v minus its component along the null vector."""
    return v - (v @ null) / (null @ null) * null


def _case(mode):
    if mode == abi.MODE_METRIC:
        g = G.shear_layer_grid(16, 8, 16, stretched=True)
        f = {"r": np.zeros(g.ghosted, order="F"), "densityBG": np.zeros(g.ghosted, order="F")}
        anelastic.set_density_bg(f, g, x3center=-2000.0)  # a 20 m column 2 km up
        r = f["r"]
        assert r.std() > 0

        def apply(p):
            a = p.copy(order="F")
            _wrap_xy(a)
            return psource_pgrad(a, g, r)

        return g, r, apply
    g = G.shear_layer_grid(16, 8, 16, stretched=False)
    return g, np.ones(g.ghosted, order="F"), lambda p: literal_apply(p, g)


@pytest.mark.parametrize("mode", [abi.MODE_METRIC, abi.MODE_LITERAL])
def test_oracle_operator_equals_restatement(mode):
    g, r, apply = _case(mode)
    p = abi.make_mg_params(levels_for(g), tbc=PERIODIC_XY_NEUMANN_Z, mode=mode)
    o = OracleMG(g, p)
    o.set_density(r)
    rng = np.random.default_rng(5)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    o.debug_pass(1, phi, np.zeros(g.ghosted, order="F"))  # mg_bdry ghosts
    got = o.apply(phi)[1:-1, 1:-1, 1:-1]
    ref = apply(phi)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("mode", [abi.MODE_METRIC, abi.MODE_LITERAL])
def test_multigrid_solution_equals_direct_solve(mode):
    g, r, apply = _case(mode)
    A = dense_operator(apply, g)
    # null vector: p = r (metric: grad(p/r) = 0), constants (literal, r = 1)
    null = _interior(r)
    np.testing.assert_allclose(A @ null, 0.0, atol=1e-10 * np.abs(A).max())
    rng = np.random.default_rng(11)
    src = np.asfortranarray(rng.standard_normal(g.ghosted))
    # compatibility: the left null vector is the cell volume (metric) or 1
    src = remove_vmean(src, g) if mode == abi.MODE_METRIC else remove_mean(src)
    x_direct = np.linalg.lstsq(A, _interior(src), rcond=None)[0]
    assert np.linalg.norm(A @ x_direct - _interior(src)) < 1e-10 * np.linalg.norm(_interior(src))

    p = abi.make_mg_params(levels_for(g), maxcy=300, tolmax=1e-13, tbc=PERIODIC_XY_NEUMANN_Z, mode=mode,
                           smoother=abi.SMOOTHER_ZLINE, stop=abi.STOP_RESID)
    o = OracleMG(g, p)
    o.set_density(r)
    phi = np.zeros(g.ghosted, order="F")
    it, res = o.solve(phi, src.copy(order="F"))
    assert it <= 300 and res <= 1e-13
    a, b = _drop(_interior(phi), null), _drop(x_direct, null)
    assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)
