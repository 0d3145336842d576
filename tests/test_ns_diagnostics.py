"""Plane statistics of the reference driver's per-step dk/dt block
(NSsolver.F90:288-395): center_velocity (StatTools.F90:87-289, with
interpoly/divdiffs :563-653), avgX1X2 (Average.F90:279-368), the mean
profiles, the second moments of the fluctuations and their time
derivatives.

Per-cell values (centred velocities, fluctuations, squares) follow the
reference expressions exactly.  The numpy restatement sums the planes in
the oracle's sequential order and matches it bit for bit.  The GPU's plane
sums are a fixed-order parallel sum, so its profiles are compared
within 1e-12 of the profile's largest magnitude, and the derivative
profiles, which divide a difference of two such sums by the step, within
1e-12 * max|profile| / dt.  LITERAL mode keeps the reference's stretched-
axis interpolation as written (values used as abscissae), which is Inf or
NaN where two values of the window coincide: NaN positions must agree.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for

# ghost() type codes of the oracle (u, v, w, rho, cfluc, scal1)
VT_U, VT_V, VT_W, VT_RHO, VT_CFLUC, VT_SCAL1 = 0, 1, 2, 4, 5, 12
BASE = {"dU1dt": "U1", "dU2dt": "U2", "dTdt": "T", "dSdt": "S", "dMKEdt": "MKE", "dkdt": "TKE",
        "dt2dt": "t2", "ds2dt": "s2"}


def compare(got, ref, dt, what=""):
    for name in abi.DIAG_NAMES:
        base = ref[BASE.get(name, name)]
        fin = base[np.isfinite(base)]
        scale = np.abs(fin).max() if fin.size else 1.0
        atol = 1e-12 * (scale / dt if name in BASE else scale) + 1e-300
        np.testing.assert_allclose(got[name], ref[name], rtol=1e-12, atol=atol, equal_nan=True,
                                   err_msg=f"{what} {name}")


# --------------------------------------------------- numpy restatement
def _newton5(x, y, loc):
    d = [list(y)]
    for j in range(1, 5):
        prev = d[-1]
        d.append([None] * j + [(prev[k] - prev[k - 1]) / (x[k] - x[k - j]) for k in range(j, 5)])
    a = [d[k][k] for k in range(5)]
    s = a[4]
    for k in range(3, -1, -1):
        s = s * (loc - x[k]) + a[k]
    return s


def _center(o, g, a, d, stretched, corrected):
    out = np.zeros_like(a, order="F")
    n = (g.x.n, g.y.n, g.z.n)[d]
    ax = (g.x, g.y, g.z)[d]
    inner = [slice(1, -1)] * 3

    def take(idx):  # interior of the other two axes at Fortran index idx along d
        s = list(inner)
        s[d] = idx - 1
        return a[tuple(s)]

    with np.errstate(divide="ignore", invalid="ignore"):
        for q in range(2, n + 2):
            s = list(inner)
            s[d] = q - 1
            if not stretched:
                out[tuple(s)] = 0.5 * (take(q) + take(q - 1))
            else:
                lo = 1 if q == 2 else (n - 2 if q == n + 1 else q - 2)
                dep = [take(lo + m) for m in range(5)]
                ind = [ax.xe[lo + m - 1] for m in range(5)]
                loc = ax.xc[q - 1]
                out[tuple(s)] = _newton5(ind, dep, loc) if corrected else _newton5(dep, ind, loc)
    o.ghost(out, (VT_U, VT_V, VT_W)[d])
    return out


def _avg(o, g, var, vt):
    """avgX1X2: sum var*dxc*dyc / Area per plane, summed sequentially in the
    reference's loop order (i fastest)."""
    o.ghost(var, vt)
    dx, dy = g.x.dxc[1:-1, None], g.y.dxc[None, 1:-1]
    area = sum(g.x.dxc[i] * g.y.dxc[j] for j in range(1, g.y.n + 1) for i in range(1, g.x.n + 1))
    out = np.empty(var.shape[2])
    for k in range(var.shape[2]):
        terms = ((var[1:-1, 1:-1, k] * dx) * dy).reshape(-1, order="F")
        out[k] = np.add.accumulate(np.concatenate(([0.0], terms)))[-1] / area
    return out


def _fluct_sq(o, a, mean):
    t = a.copy(order="F")
    t[1:-1, 1:-1, 1:-1] -= mean[None, None, 1:-1]
    o.ghost(t, VT_CFLUC)
    return np.asfortranarray(t * t)


def numpy_block(o, g, f, mode, stretched, old, dtt):
    corr = mode == abi.DIAG_CORRECTED
    uc = _center(o, g, f["u"], 0, stretched[0], corr)
    vc = _center(o, g, f["v"], 1, stretched[1], corr)
    wc = _center(o, g, f["w"], 2, stretched[2], corr)
    with np.errstate(invalid="ignore", over="ignore"):
        m1, m2 = _avg(o, g, uc, VT_U), _avg(o, g, vc, VT_V)
        m3, m4 = _avg(o, g, f["rho"], VT_RHO), _avg(o, g, f["scal1"], VT_SCAL1)
        sq = []
        for c, vt in ((uc, VT_U), (vc, VT_V), (wc, VT_W)):
            sq.append(_avg(o, g, _fluct_sq(o, c, _avg(o, g, c, vt)), vt))
        tt = _avg(o, g, _fluct_sq(o, f["rho"], _avg(o, g, f["rho"], VT_RHO)), VT_RHO)
        ss = _avg(o, g, _fluct_sq(o, f["scal1"], _avg(o, g, f["scal1"], VT_SCAL1)), VT_SCAL1)
        now = {"U1": m1, "U2": m2, "T": m3, "S": m4, "MKE": m1 + m2,
               "TKE": 1.0 / 2.0 * (sq[0] + sq[1] + sq[2]), "t2": tt, "s2": ss}
        out = dict(now)
        for d, b in BASE.items():
            out[d] = (now[b] - old[b]) / dtt
    return out


def _case(n=(16, 8, 16), ew=1):
    g_ = G.shear_layer_grid(*n, stretched=True)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=ew, scal1_on=1)
    f = shear.shear_layer_fields(g_, amp=1e-3)
    f["scal1"][...] = np.asfortranarray(np.random.default_rng(3).standard_normal(f["scal1"].shape))
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    return g_, mgp, nsp, f, o


@pytest.mark.parametrize("mode", [abi.DIAG_LITERAL, abi.DIAG_CORRECTED])
def test_oracle_block_matches_numpy_restatement(mode):
    """Two independent restatements of the block agree bit for bit (CPU):
    the plane sums run in the same sequential order; the derivatives divide
    by time - told, told being the time before the step (0 here)."""
    g_, mgp, nsp, f, o = _case()
    rep = o.step()
    zeros = {b: np.zeros(g_.z.n + 2) for b in BASE.values()}
    work = {k: f[k].copy(order="F") for k in ("u", "v", "w", "rho", "scal1")}
    ref = numpy_block(o, g_, work, mode, (0, 0, 1), zeros, rep.time - 0.0)
    got = o.diagnostics(mode, (0, 0, 1))
    for name in abi.DIAG_NAMES:
        np.testing.assert_array_equal(got[name], ref[name], err_msg=name)
    if mode == abi.DIAG_CORRECTED:
        for name in abi.DIAG_NAMES:
            assert np.isfinite(got[name]).all(), name


def test_literal_interpolation_is_the_inverse_interpolant():
    """interpoly(dep, ind, loc, 4) as written passes the values to divdiffs as
    abscissae: on points of a straight line w = 2 z + 1 its result at loc is
    the z where the line takes the value loc."""
    z = np.array([0.0, 0.3, 0.7, 1.2, 1.8])
    w = 2.0 * z + 1.0
    assert _newton5(w, z, 2.4) == pytest.approx((2.4 - 1.0) / 2.0, rel=1e-14)
    assert _newton5(z, w, 0.5) == pytest.approx(2.0 * 0.5 + 1.0, rel=1e-14)


# ------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("ew", [1, 0])
@pytest.mark.parametrize("mode", [abi.DIAG_LITERAL, abi.DIAG_CORRECTED])
def test_gpu_diagnostics_match_oracle(mode, ew):
    from anelastic_solve_b200.ns import NSSolver

    g_, mgp, nsp, f, o = _case(n=(32, 16, 32), ew=ew)
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    s.set_diagnostics(True, mode, (0, 0, 1))
    for n in range(2):
        ro = o.step()
        rg = s.step(1)
        assert ro.time == rg.time
        compare(s.diagnostics(), o.diagnostics(mode, (0, 0, 1)), ro.dt, f"step {n} mode {mode}")
        assert rg.diag_ms > 0.0


@pytest.mark.gpu
def test_gpu_diagnostics_explicit_call_and_reset():
    """compute_diagnostics on the fields after a step equals the block that
    step() runs; profiles start from zero."""
    from anelastic_solve_b200.ns import NSSolver

    g_, mgp, nsp, f, o = _case(n=(32, 16, 32))
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    assert all(not v.any() for v in s.diagnostics().values())
    s.set_diagnostics(False, abi.DIAG_CORRECTED, (0, 0, 1))
    ro = o.step()
    s.step(1)
    s.compute_diagnostics()
    compare(s.diagnostics(), o.diagnostics(abi.DIAG_CORRECTED, (0, 0, 1)), ro.dt, "explicit")
