"""The oracle's Crank-Nicolson z solve, restated from the reference (CPU
only).

var_advance_CN_PL (ANELASTIC_SL/dns/NSsolver.F90:3054-3465, DNS terms, as
rk_ss calls it with f1 = f3 = 1, f2 = a3; NSsolver.F90:510-517) is written
here with numpy: the tridiagonal rows with their swapped face pairing, the
explicit half of the z diffusion in the right-hand side, the wall rows of
the boundary codes TB (free-slip walls: u, v Neumann; w Dirichlet, with the
edge-node row when ew = 1; rho and scal1 Neumann on two rows each side),
and the reference's Thomas routine (mgMK/mg_relax.F90:541-595) over
k = 1..nz+2, vectorised across columns, with and without the LES eddy
terms (random nuT, kappaT, nappaT); then the parts of the field's ghost
pass that touch the interior (w's edge node, the scalars' two-point
Neumann rows).  Every expression keeps the
Fortran operand order, so the interior of the solved field must equal the
oracle's bit for bit, for every variable, on random fields with r(z) on a
stretched grid.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for

RE, PR, SC = 1000.0, 0.7, 2.0
A3, RKDT = 0.75, 0.013


def thomas(a, b, c, G_):
    """mg_relax.F90:541-595 along the last axis (a, b overwritten, c kept)."""
    a, b, G_ = a.copy(), b.copy(), G_.copy()
    n = a.shape[-1]
    for j in range(n - 1):
        a[..., j + 1] = -a[..., j + 1] / b[..., j]
        b[..., j + 1] = b[..., j + 1] + a[..., j + 1] * c[..., j]
        G_[..., j + 1] = G_[..., j + 1] + a[..., j + 1] * G_[..., j]
    G_[..., n - 1] = G_[..., n - 1] / b[..., n - 1]
    for j in range(n - 2, -1, -1):
        G_[..., j] = (G_[..., j] - c[..., j] * G_[..., j + 1]) / b[..., j]
    return G_


def _eddy_pair(var, E, g, R, k):
    """The LES face coefficients (tmp1, tmp2) of var_advance_CN_PL
    (NSsolver.F90:3130-3160) on the interior columns, or None without LES.
    u and v pair the upper-face density average with the lower-face eddy
    average, as the reference writes them."""
    if E is None:
        return None
    nx, ny, _ = g.shape

    def col(a, di=0, dj=0):
        return a[1 + di:nx + 1 + di, 1 + dj:ny + 1 + dj, :]

    rk, rkp, rkm = R[:, :, k], R[:, :, k + 1], R[:, :, k - 1]
    if var == 3:
        nu = col(E["nuT"])
        return (-nu[:, :, k] * rk / (0.5 * (rkp + rk)), -nu[:, :, k + 1] * rkp / (0.5 * (rkp + rk)))
    raver1 = 0.5 * (rkp + rk)
    raver2 = 0.5 * (rk + rkm)
    if var in (1, 2):
        a, b = col(E["nuT"]), col(E["nuT"], 1, 0) if var == 1 else col(E["nuT"], 0, 1)
        t1 = -0.25 * (a[:, :, k] + b[:, :, k] + a[:, :, k - 1] + b[:, :, k - 1]) * raver1 / rk
        t2 = -0.25 * (a[:, :, k] + b[:, :, k] + a[:, :, k + 1] + b[:, :, k + 1]) * raver2 / rk
        return t1, t2
    kT = col(E["kappaT"] if var == 5 else E["nappaT"])
    t1 = -0.5 * (kT[:, :, k] + kT[:, :, k - 1])
    t2 = -0.5 * (kT[:, :, k] + kT[:, :, k + 1])
    if var == 5:
        t1 = t1 * raver1 / rk
        t2 = t2 * raver2 / rk
    return t1, t2


def cn_restated(g, nsp, r, q, u, var, a3=A3, rkdt=RKDT, eddy=None):
    """The solved interior of var_advance_CN_PL(q, u, 1, a3, 1, rkdt, var);
    eddy = {nuT, kappaT, nappaT} (ghosted) adds the LES terms."""
    nx, ny, nz = g.shape
    z = g.z
    rRe = 1.0 / RE
    # interior columns, k = 1..nz+2 along the last axis (array index k-1)
    sl = (slice(1, nx + 1), slice(1, ny + 1))
    R, U, Q = r[sl], u[sl], q[sl]
    shape = (nx, ny, nz + 2)
    sub, diag, sup, rhs = (np.zeros(shape) for _ in range(4))
    k = np.arange(1, nz + 1)          # array index of Fortran k = 2..nz+1
    rdze, rdzc = z.rdxe, z.rdxc
    rk, rkp, rkm = R[:, :, k], R[:, :, k + 1], R[:, :, k - 1]
    rhs[:, :, k] = 1.0 * U[:, :, k] + a3 * Q[:, :, k] * 1.0
    if var != 3:
        raver1 = 0.5 * (rkp + rk)
        raver2 = 0.5 * (rk + rkm)
        if var in (1, 2):
            t1 = (rRe + 0.0) * raver1 / rk
            t2 = (rRe + 0.0) * raver2 / rk
        elif var == 5:
            t1 = (rRe * (1.0 / PR) + 0.0) * raver1 / rk
            t2 = (rRe * (1.0 / PR) + 0.0) * raver2 / rk
        else:
            t1 = np.broadcast_to(rRe * (1.0 / SC) + 0.0, rk.shape)
            t2 = t1
        sub[:, :, k] = -0.5 * rkdt * t1 * rdze[k - 1] * rdzc[k]
        sup[:, :, k] = -0.5 * rkdt * t2 * rdze[k] * rdzc[k]
        diag[:, :, k] = 1.0 + 0.5 * rkdt * (t1 * rdze[k - 1] + t2 * rdze[k]) * rdzc[k]
        rhs[:, :, k] = rhs[:, :, k] + rkdt * 0.5 * (
            t2 * (U[:, :, k + 1] - U[:, :, k]) * rdze[k] - t1 * (U[:, :, k] - U[:, :, k - 1]) * rdze[k - 1]
        ) * rdzc[k]
        e = _eddy_pair(var, eddy, g, R, k)
        if e is not None:
            e1, e2 = e
            sub[:, :, k] = sub[:, :, k] - 1 * 0.5 * rkdt * e1 * rdze[k - 1] * rdzc[k]
            sup[:, :, k] = sup[:, :, k] - 1 * 0.5 * rkdt * e2 * rdze[k] * rdzc[k]
            diag[:, :, k] = diag[:, :, k] + 1 * 0.5 * rkdt * (e1 * rdze[k - 1] + e2 * rdze[k]) * rdzc[k]
            rhs[:, :, k] = rhs[:, :, k] + 1 * rkdt * 0.5 * (
                e2 * (U[:, :, k + 1] - U[:, :, k]) * rdze[k] - e1 * (U[:, :, k] - U[:, :, k - 1]) * rdze[k - 1]
            ) * rdzc[k]
    else:
        t1 = (rRe + 0.0) * rk / (0.5 * (rkp + rk))
        t2 = (rRe + 0.0) * rkp / (0.5 * (rkp + rk))
        sub[:, :, k] = -0.5 * rkdt * t1 * rdze[k] * rdzc[k]
        sup[:, :, k] = -0.5 * rkdt * t2 * rdze[k] * rdzc[k + 1]
        diag[:, :, k] = 1.0 + 0.5 * rkdt * (t1 * rdzc[k] + t2 * rdzc[k + 1]) * rdze[k]
        rhs[:, :, k] = rhs[:, :, k] + rkdt * 0.5 * (
            t2 * (U[:, :, k + 1] - U[:, :, k]) * rdzc[k + 1] - t1 * (U[:, :, k] - U[:, :, k - 1]) * rdzc[k]
        ) * rdze[k]
        e = _eddy_pair(var, eddy, g, R, k)
        if e is not None:
            e1, e2 = e
            sub[:, :, k] = sub[:, :, k] - 1 * 1.0 * rkdt * e1 * rdze[k] * rdzc[k]
            sup[:, :, k] = sup[:, :, k] - 1 * 1.0 * rkdt * e2 * rdze[k] * rdzc[k + 1]
            diag[:, :, k] = diag[:, :, k] + 1 * 1.0 * rkdt * (e1 * rdzc[k] + e2 * rdzc[k + 1]) * rdze[k]
            rhs[:, :, k] = rhs[:, :, k] + 1 * rkdt * 1.0 * (
                e2 * (U[:, :, k + 1] - U[:, :, k]) * rdzc[k + 1] - e1 * (U[:, :, k] - U[:, :, k - 1]) * rdzc[k]
            ) * rdze[k]

    def row(kk, a, b, c, d):
        sub[:, :, kk], diag[:, :, kk], sup[:, :, kk], rhs[:, :, kk] = a, b, c, d

    tbmin, tbmax = nsp.tb[2][0][var - 1], nsp.tb[2][1][var - 1]
    vbmin, vbmax = nsp.vb[2][0][var - 1], nsp.vb[2][1][var - 1]
    sz0, ez1 = 0, nz + 1                     # array index of sz-1 and ez+1
    if tbmin == 1:
        row(sz0, 0.0, 1.0, 0.0, vbmin)
    elif tbmin == 2:
        if var == 3:
            row(sz0, 0.0, -1.0, 1.0, z.dxc[sz0] * vbmin)
        elif var in (5, 8):
            row(sz0, 0.0, -1.0, 1.0, z.dxe[sz0] * vbmin)
            row(sz0 + 1, 0.0, -1.0, 1.0, z.dxe[sz0 + 1] * vbmin)
        else:
            row(sz0, 0.0, -1.0, 1.0, z.dxe[sz0] * vbmin)
    elif tbmin == 6:
        row(sz0, 0.0, 1.0, 1.0, 2.0 * vbmin)
    if tbmax == 1:
        row(ez1, 0.0, 1.0, 0.0, vbmax)
    elif tbmax == 2:
        if var == 3:
            row(ez1, -1.0, 1.0, 0.0, z.dxc[ez1] * vbmax)
        elif var in (5, 8):
            row(ez1, -1.0, 1.0, 0.0, z.dxe[ez1] * vbmax)
            row(ez1 - 1, -1.0, 1.0, 0.0, z.dxe[ez1 - 1] * vbmax)
        else:
            row(ez1, -1.0, 1.0, 0.0, z.dxe[ez1] * vbmax)
    elif tbmax == 6:
        row(ez1, 1.0, 1.0, 0.0, 2.0 * vbmax)
    elif tbmax == 7:
        row(ez1, 0.0, 1.0, 0.0, 0.0)
        row(ez1 - 1, 0.0, 1.0, 0.0, 0.0)
    x = thomas(sub, diag, sup, rhs)[:, :, 1:nz + 1]
    if var in (5, 8) and tbmin == 2 and tbmax == 2 and vbmin == 0.0 and vbmax == 0.0:
        # the field's ghost pass after the solve: two-point Neumann of the
        # scalars resets the first and last interior rows from their
        # neighbours (bound_update, dns/BC.F90:532,537; wall value 0)
        x[:, :, 0] = x[:, :, 1]
        x[:, :, -1] = x[:, :, -2]
    return x


@pytest.fixture(scope="module", params=[False, True], ids=["dns", "les"])
def case(request):
    les = request.param
    g = G.shear_layer_grid(12, 8, 20, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=RE, Pr=PR, Sc=SC, ew=1, scal1_on=1, les=les)
    f = shear.shear_layer_fields(g)
    eddy = None
    if les:  # eddy coefficients of either sign, ghosts included
        rng = np.random.default_rng(99)
        for k in ("nuT", "kappaT", "nappaT"):
            f[k] = np.asfortranarray(0.01 * rng.standard_normal(g.ghosted))
        eddy = {k: f[k] for k in ("nuT", "kappaT", "nappaT")}
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    o = OracleNS(g, mgp, nsp, f)
    return g, nsp, f, o, eddy


@pytest.mark.parametrize("var", [1, 2, 3, 5, 8])
def test_crank_nicolson_equals_restatement(case, var):
    g, nsp, f, o, eddy = case
    rng = np.random.default_rng(var)
    u = np.asfortranarray(rng.standard_normal(g.ghosted))
    q = np.asfortranarray(rng.standard_normal(g.ghosted))
    got = o.crank_nicolson(q, u, A3, RKDT, var)[1:-1, 1:-1, 1:-1]
    ref = cn_restated(g, nsp, f["r"], q, u, var, eddy=eddy)
    assert np.abs(ref).max() > 0
    if var == 3:
        # ew = 1: the ghost pass that follows the solve makes w at the top
        # wall node (k = nz+1) the wall value
        assert not np.any(got[:, :, -1])
        got, ref = got[:, :, :-1], ref[:, :, :-1]
    np.testing.assert_array_equal(got, ref)
