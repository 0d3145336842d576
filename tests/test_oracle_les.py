"""The oracle's Smagorinsky update, restated from the reference (CPU only).

straincal's strain magnitude |S| (ANELASTIC_SL/les/straincal.F90:48-73)
and filter width delg (:126-134, '3root' and '2root'), the model
coefficients of SSM, SSMrho and SSMscal1 (les/SSM.F90, with the wall
damping as written: REAL(4) 0.41, Zo = 0.3d0 for the velocity and the
scal1 model, Zo = 0.3 REAL(4) for rho; or without damping), and SGSdiff's
nuT, kappaT, nappaT (straincal.F90:339-414) are written here with numpy in
the Fortran operand order; x**2.d0 is x*x and x**(1.d0/3.d0) is pow.  On
random velocities on a stretched grid the oracle's eddy coefficients must
equal them bit for bit.
"""
import math

import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for
from .test_oracle_rhs import _Shift

SSM_CONST, PR_SGS = 0.0289, 0.7
_pow = np.frompyfunc(math.pow, 2, 1)


def strain_magnitude(f, h):
    S, M = h.S, h.M
    l1, l2, l3 = f["u"], f["v"], f["w"]
    TS11 = (S(l1, 1) - S(l1)) * M(0, "rdxc")
    TS22 = (S(l2, 0, 1) - S(l2)) * M(1, "rdxc")
    TS33 = (S(l3, 0, 0, 1) - S(l3)) * M(2, "rdxc")
    t1 = 0.25 * (S(l1) + S(l1, 1) + S(l1, 0, 1) + S(l1, 1, 1))
    t2 = 0.25 * (S(l1) + S(l1, 1) + S(l1, 0, -1) + S(l1, 1, -1))
    t3 = 0.25 * (S(l2) + S(l2, 0, 1) + S(l2, 1) + S(l2, 1, 1))
    t4 = 0.25 * (S(l2) + S(l2, 0, 1) + S(l2, -1) + S(l2, -1, 1))
    TS12 = 0.5 * ((t1 - t2) * M(1, "rdxc") + (t3 - t4) * M(0, "rdxc"))
    t1 = 0.25 * (S(l1) + S(l1, 1) + S(l1, 0, 0, 1) + S(l1, 1, 0, 1))
    t2 = 0.25 * (S(l1) + S(l1, 1) + S(l1, 0, 0, -1) + S(l1, 1, 0, -1))
    t3 = 0.25 * (S(l3) + S(l3, 0, 0, 1) + S(l3, 1) + S(l3, 1, 0, 1))
    t4 = 0.25 * (S(l3) + S(l3, 0, 0, 1) + S(l3, -1) + S(l3, -1, 0, 1))
    TS13 = 0.5 * ((t1 - t2) * M(2, "rdxc") + (t3 - t4) * M(0, "rdxc"))
    t1 = 0.25 * (S(l2) + S(l2, 0, 1) + S(l2, 0, 0, 1) + S(l2, 0, 1, 1))
    t2 = 0.25 * (S(l2) + S(l2, 0, 1) + S(l2, 0, 0, -1) + S(l2, 0, 1, -1))
    t3 = 0.25 * (S(l3) + S(l3, 0, 0, 1) + S(l3, 0, 1) + S(l3, 0, 1, 1))
    t4 = 0.25 * (S(l3) + S(l3, 0, 0, 1) + S(l3, 0, -1) + S(l3, 0, -1, 1))
    TS23 = 0.5 * ((t1 - t2) * M(2, "rdxc") + (t3 - t4) * M(1, "rdxc"))
    return math.sqrt(2.0) * np.sqrt(TS11 * TS11 + TS22 * TS22 + TS33 * TS33 + 2.0 * (TS12 * TS12)
                                    + 2.0 * (TS13 * TS13) + 2.0 * (TS23 * TS23))


def filter_width(h, delta):
    M = h.M
    if delta == abi.DELTA_3ROOT:
        x = M(0, "dxc") * M(1, "dxc") * M(2, "dxc")
        return _pow(x, 1.0 / 3.0).astype(np.float64)
    x = M(0, "dxc") * M(0, "dxc") + M(1, "dxc") * M(1, "dxc") + M(2, "dxc") * M(2, "dxc")
    return _pow(x, 1.0 / 2.0).astype(np.float64)


def damping(h, dg, zo):
    """((0.41 (zc + Zo))^2 / ((0.41 (zc + Zo))^2 + SSM_const delg^2))"""
    a = float(np.float32(0.41)) * (h.M(2, "xc") + zo)
    return (a * a) / ((a * a) + SSM_CONST * (dg * dg))


@pytest.mark.parametrize("delta", [abi.DELTA_3ROOT, abi.DELTA_2ROOT], ids=["3root", "2root"])
@pytest.mark.parametrize("damp", [abi.DAMP_LITERAL, abi.DAMP_NONE], ids=["damped", "undamped"])
def test_eddy_coefficients_equal_restatement(delta, damp):
    g = G.shear_layer_grid(16, 8, 24, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=50000.0, g=-0.1, ew=1, scal1_on=1, les=True, ssm_const=SSM_CONST,
                             pr_sgs=PR_SGS, les_delta=delta, les_damp=damp)
    rng = np.random.default_rng(21)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w"):
        f[k][...] = rng.standard_normal(g.ghosted)
    for k in ("nuT", "kappaT", "nappaT"):
        f[k] = np.zeros(g.ghosted, order="F")
    o = OracleNS(g, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2)):
        o.ghost(f[name], vt)
    h = _Shift(g)
    modS = strain_magnitude(f, h)
    dg = np.broadcast_to(filter_width(h, delta), modS.shape)
    if damp == abi.DAMP_LITERAL:
        Csgs = SSM_CONST * damping(h, dg, 0.3)
        CT = Csgs / PR_SGS * damping(h, dg, float(np.float32(0.3)))
        CS = Csgs / PR_SGS * damping(h, dg, 0.3)
    else:
        Csgs = np.broadcast_to(SSM_CONST * 1.0, modS.shape)
        CT = Csgs / PR_SGS * 1.0
        CS = CT
    o.les_update()
    for name, C in (("nuT", Csgs), ("kappaT", CT), ("nappaT", CS)):
        ref = -(C + 0.0) * (dg * dg) * modS + 0.0
        assert np.abs(ref).max() > 0
        np.testing.assert_array_equal(f[name][1:-1, 1:-1, 1:-1], ref, err_msg=name)
