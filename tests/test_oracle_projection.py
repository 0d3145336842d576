"""The oracle's projection, checked by restatements of the reference's own
diagnostics (CPU only).

- divergence (ANELASTIC_SL/dns/Routines.F90:54-183): per cell
  (u_i - u_(i-1)) rdxc + (v_j - v_(j-1)) rdyc + (w_k - w_(k-1)) rdzc, the
  volume-weighted mean of |div| and the largest |div|;
- Psource (dns/NSsolver.F90:2167-2223): the r-weighted divergence that the
  projection removes; with an anelastic r(z) it is the quantity the
  pressure equation zeroes, while the plain divergence is not zero.

After the oracle's initial projection, solved to a relative residual of
1e-12, the restated divergence equals the oracle's report.  It is within
the bound max|div u| <= 1e-10 max|u| / dz_min for r = 1, and the restated
Psource is below 1e-9 of its value before the projection for r(z).  The
first step's time step is calcdt's (dns/Routines.F90:186-258, capped by
dtmax as in dns/NSsolver.F90:72-73), restated in its own sum order.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for


def _bc(v, d):
    sl = [None, None, None]
    sl[d] = slice(None)
    return v[tuple(sl)]


def divergence(f, g):
    u, v, w = f["u"], f["v"], f["w"]
    return ((u[1:-1, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) * _bc(g.x.rdxc[1:-1], 0)
            + (v[1:-1, 1:-1, 1:-1] - v[1:-1, :-2, 1:-1]) * _bc(g.y.rdxc[1:-1], 1)
            + (w[1:-1, 1:-1, 1:-1] - w[1:-1, 1:-1, :-2]) * _bc(g.z.rdxc[1:-1], 2))


def psource(f, g):
    """r-weighted divergence (dt = 1): r u and r v at the cell's own level,
    the face averages of r for w."""
    u, v, w, r = f["u"], f["v"], f["w"], f["r"]
    rc = r[1:-1, 1:-1, 1:-1]
    rp = 0.5 * (r[1:-1, 1:-1, 1:-1] + r[1:-1, 1:-1, 2:])
    rm = 0.5 * (r[1:-1, 1:-1, 1:-1] + r[1:-1, 1:-1, :-2])
    return ((rc * u[1:-1, 1:-1, 1:-1] - rc * u[:-2, 1:-1, 1:-1]) * _bc(g.x.rdxc[1:-1], 0)
            + (rc * v[1:-1, 1:-1, 1:-1] - rc * v[1:-1, :-2, 1:-1]) * _bc(g.y.rdxc[1:-1], 1)
            + (rp * w[1:-1, 1:-1, 1:-1] - rm * w[1:-1, 1:-1, :-2]) * _bc(g.z.rdxc[1:-1], 2))


def _projected(anel, cfl=None):
    g = G.shear_layer_grid(32, 16, 32, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), maxcy=300, tolmax=1e-12, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, stop=abi.STOP_RESID)
    kw = {"cfl": cfl, "dtmax": 1e9} if cfl else {"dtmax": 0.01}
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, ew=1, scal1_on=1, **kw)
    f = shear.shear_layer_fields(g, amp=1e-2)
    if anel:
        anelastic.set_density_bg(f, g, x3center=-1000.0)
        assert f["r"].std() > 0
    o = OracleNS(g, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    before = psource(f, g)
    o.project()
    return g, f, o, before


def test_divergence_restated_and_bounded():
    g, f, o, _ = _projected(False)
    d = divergence(f, g)
    vol = _bc(g.x.dxc[1:-1], 0) * _bc(g.y.dxc[1:-1], 1) * _bc(g.z.dxc[1:-1], 2)
    vol = np.broadcast_to(vol, d.shape)
    avg, mx = o.divergence()
    assert mx == np.abs(d).max()
    assert avg == pytest.approx((np.abs(d) * vol).sum() / vol.sum(), rel=1e-12)
    umax = max(np.abs(f[k][1:-1, 1:-1, 1:-1]).max() for k in ("u", "v", "w"))
    assert 0.0 < mx <= 1e-10 * umax / g.z.dxc[1:-1].min()


def test_anelastic_projection_zeroes_psource():
    g, f, o, before = _projected(True)
    after = psource(f, g)
    assert np.abs(after).max() <= 1e-9 * np.abs(before).max()
    # the plain divergence is not what the anelastic projection zeroes
    assert np.abs(divergence(f, g)).max() > 1e3 * np.abs(after).max()


def test_calcdt_restated():
    g, f, o, _ = _projected(False, cfl=0.5)
    u, v, w = f["u"], f["v"], f["w"]
    adv = _bc(g.x.rdxc[1:-1], 0) * np.abs(0.5 * (u[1:-1, 1:-1, 1:-1] + u[:-2, 1:-1, 1:-1]))
    adv = adv + _bc(g.z.rdxc[1:-1], 2) * np.abs(0.5 * (w[1:-1, 1:-1, 1:-1] + w[1:-1, 1:-1, :-2]))
    adv = adv + _bc(g.y.rdxc[1:-1], 1) * np.abs(0.5 * (v[1:-1, 1:-1, 1:-1] + v[1:-1, :-2, 1:-1]))
    dt = min(0.5 / adv.max(), 1e9)
    assert o.step().dt == dt
