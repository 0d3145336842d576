"""The oracle's explicit right-hand sides, restated from the reference
(CPU only).

u1_rhs, u2_rhs, u3_rhs, rho_rhs and scal1_rhs
(ANELASTIC_SL/dns/NSsolver.F90:585-2020, the terms of the Crank-Nicolson
configuration: x/y diffusion, flux-form advection with the anelastic r(z)
weights, buoyancy against densityBG, and the LES eddy terms with random
nuT, kappaT, nappaT, including u2's face pairing and scal1's sign slip) are
written here as whole-array numpy expressions.  Each expression keeps the Fortran
statement's operand order, so the interior values must equal the oracle's
bit for bit.  The fields are random on a stretched grid with a non-uniform
r(z) and densityBG(z), so every term and weight contributes.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for

RE, PR, SC, GRAV = 1000.0, 0.7, 2.0, -0.12


class _Shift:
    """S(a, di, dj, dk): the interior block of a shifted by (di, dj, dk);
    M(axis, name, off): a metric array at Fortran index i + off, broadcast
    along its direction."""

    def __init__(self, g):
        self.g = g
        self.n = g.shape

    def S(self, a, di=0, dj=0, dk=0):
        nx, ny, nz = self.n
        return a[1 + di:1 + nx + di, 1 + dj:1 + ny + dj, 1 + dk:1 + nz + dk]

    def M(self, d, name, off=0):
        ax = (self.g.x, self.g.y, self.g.z)[d]
        v = getattr(ax, name)[1 + off:1 + ax.n + off]
        sl = [None, None, None]
        sl[d] = slice(None)
        return v[tuple(sl)]


def u1_rhs(f, h, rRe, les=False):
    S, M = h.S, h.M
    u, v, w, r = f["u"], f["v"], f["w"], f["r"]
    Ut = 0.0 + (rRe * ((S(u, 1) - S(u)) * M(0, "rdxc", 1) - (S(u) - S(u, -1)) * M(0, "rdxc")) * M(0, "rdxe")
                + rRe * ((S(u, 0, 1) - S(u)) * M(1, "rdxe") - (S(u) - S(u, 0, -1)) * M(1, "rdxe", -1))
                * M(1, "rdxc"))
    ua2 = 0.5 * (S(u, 1) + S(u))
    ua1 = 0.5 * (S(u) + S(u, -1))
    Ut = Ut + (ua1 * ua1 - ua2 * ua2) * M(0, "rdxe")
    ua2 = 0.5 * (S(u, 0, 0, 1) + S(u))
    ua1 = 0.5 * (S(u) + S(u, 0, 0, -1))
    ra2 = 0.5 * (S(r, 0, 0, 1) + S(r))
    ra1 = 0.5 * (S(r) + S(r, 0, 0, -1))
    wa2 = 0.5 * (S(w, 1) + S(w))
    wa1 = 0.5 * (S(w, 1, 0, -1) + S(w, 0, 0, -1))
    Ut = Ut + (ra1 * ua1 * wa1 - ra2 * ua2 * wa2) * M(2, "rdxc") / S(r)
    ua2 = 0.5 * (S(u, 0, 1) + S(u))
    ua1 = 0.5 * (S(u) + S(u, 0, -1))
    va2 = 0.5 * (S(v, 1) + S(v))
    va1 = 0.5 * (S(v, 1, -1) + S(v, 0, -1))
    Ut = Ut + (ua1 * va1 - ua2 * va2) * M(1, "rdxc")
    if not les:
        return Ut
    nu = f["nuT"]  # NSsolver.F90:761-780
    Ut = Ut - 1 * 2.0 * (S(nu, 1) * (S(u, 1) - S(u)) * M(0, "rdxc", 1)
                         - S(nu) * (S(u) - S(u, -1)) * M(0, "rdxc")) * M(0, "rdxe")
    n1 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, -1) + S(nu, 1, -1))
    n2 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, 1) + S(nu, 1, 1))
    Ut = Ut - 1 * 1.0 * (n2 * (S(u, 0, 1) - S(u)) * M(1, "rdxe") - n1 * (S(u) - S(u, 0, -1)) * M(1, "rdxe", -1)) \
        * M(1, "rdxc")
    Ut = Ut - 1 * 1.0 * (n2 * (S(v, 1, 1) - S(v, 0, 1)) * M(0, "rdxe") - n1 * (S(v, 1) - S(v)) * M(0, "rdxe")) \
        * M(1, "rdxc")
    n1 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, 0, -1) + S(nu, 1, 0, -1))
    n2 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, 0, 1) + S(nu, 1, 0, 1))
    ra2 = 0.5 * (S(r, 0, 0, 1) + S(r))
    ra1 = 0.5 * (S(r) + S(r, 0, 0, -1))
    return Ut - 1 * 1.0 * (ra2 * n2 * (S(w, 1) - S(w)) * M(0, "rdxe")
                           - ra1 * n1 * (S(w, 1, 0, -1) - S(w, 0, 0, -1)) * M(0, "rdxe")) * M(2, "rdxc") / S(r)


def u2_rhs(f, h, rRe, les=False):
    S, M = h.S, h.M
    u, v, w, r = f["u"], f["v"], f["w"], f["r"]
    Vt = 0.0 + (rRe * ((S(v, 1) - S(v)) * M(0, "rdxe") - (S(v) - S(v, -1)) * M(0, "rdxe", -1)) * M(0, "rdxc")
                + rRe * ((S(v, 0, 1) - S(v)) * M(1, "rdxc", 1) - (S(v) - S(v, 0, -1)) * M(1, "rdxc"))
                * M(1, "rdxe"))
    va1 = 0.5 * (S(v, 0, 1) + S(v))
    va2 = 0.5 * (S(v) + S(v, 0, -1))
    Vt = Vt - (va1 * va1 - va2 * va2) * M(1, "rdxe")
    va1 = 0.5 * (S(v, 1) + S(v))
    va2 = 0.5 * (S(v) + S(v, -1))
    ua1 = 0.5 * (S(u, 0, 1) + S(u))
    ua2 = 0.5 * (S(u, -1, 1) + S(u, -1))
    Vt = Vt - (ua1 * va1 - ua2 * va2) * M(0, "rdxc")
    va1 = 0.5 * (S(v, 0, 0, 1) + S(v))
    va2 = 0.5 * (S(v) + S(v, 0, 0, -1))
    ra1 = 0.5 * (S(r, 0, 0, 1) + S(r))
    ra2 = 0.5 * (S(r) + S(r, 0, 0, -1))
    wa1 = 0.5 * (S(w, 0, 1) + S(w))
    wa2 = 0.5 * (S(w, 0, 1, -1) + S(w, 0, 0, -1))
    Vt = Vt - (ra1 * wa1 * va1 - ra2 * wa2 * va2) * M(2, "rdxc") / S(r)
    if not les:
        return Vt
    nu = f["nuT"]  # NSsolver.F90:1038-1060 (raver2, the lower face, with nuTaver2)
    n1 = 0.25 * (S(nu) + S(nu, -1) + S(nu, 0, 1) + S(nu, -1, 1))
    n2 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, 1) + S(nu, 1, 1))
    Vt = Vt - 1 * 1.0 * (n2 * (S(v, 1) - S(v)) * M(0, "rdxe") - n1 * (S(v) - S(v, -1)) * M(0, "rdxe", -1)) \
        * M(0, "rdxc")
    Vt = Vt - 1 * 1.0 * (n2 * (S(u, 1, 1) - S(u, 1)) * M(1, "rdxe") - n1 * (S(u, 0, 1) - S(u)) * M(1, "rdxe")) \
        * M(0, "rdxc")
    Vt = Vt - 1 * 2.0 * (S(nu, 0, 1) * (S(v, 0, 1) - S(v)) * M(1, "rdxc", 1)
                         - S(nu) * (S(v) - S(v, 0, -1)) * M(1, "rdxc")) * M(1, "rdxe")
    n1 = 0.25 * (S(nu) + S(nu, 0, 1) + S(nu, 0, 0, -1) + S(nu, 0, 1, -1))
    n2 = 0.25 * (S(nu) + S(nu, 0, 1) + S(nu, 0, 0, 1) + S(nu, 0, 1, 1))
    ra1 = 0.5 * (S(r, 0, 0, 1) + S(r))
    ra2 = 0.5 * (S(r) + S(r, 0, 0, -1))
    return Vt - 1 * 1.0 * (ra2 * n2 * (S(w, 0, 1) - S(w)) * M(1, "rdxe")
                           - ra1 * n1 * (S(w, 0, 1, -1) - S(w, 0, 0, -1)) * M(1, "rdxe")) * M(2, "rdxc") / S(r)


def u3_rhs(f, h, rRe, g, ew, les=False):
    S, M = h.S, h.M
    u, v, w, r, rho, bg = f["u"], f["v"], f["w"], f["r"], f["rho"], f["densityBG"]
    Wt = 0.0 + 0.5 * g * ((S(rho, 0, 0, 1) - S(bg, 0, 0, 1)) + (S(rho) - S(bg))) / (
        0.5 * (S(bg, 0, 0, 1) + S(bg)))
    # Wtemp + x-term + y-term, added left to right onto the buoyancy
    Wt = (Wt + rRe * ((S(w, 1) - S(w)) * M(0, "rdxe") - (S(w) - S(w, -1)) * M(0, "rdxe", -1)) * M(0, "rdxc")
          + rRe * ((S(w, 0, 1) - S(w)) * M(1, "rdxe") - (S(w) - S(w, 0, -1)) * M(1, "rdxe", -1)) * M(1, "rdxc"))
    wa1 = 0.5 * (S(w, 0, 0, 1) + S(w))
    wa2 = 0.5 * (S(w) + S(w, 0, 0, -1))
    Wt = Wt - (S(r) * wa1 * wa1 - S(r, 0, 0, 1) * wa2 * wa2) * M(2, "rdxe") / (0.5 * (S(r) + S(r, 0, 0, 1)))
    wa1 = 0.5 * (S(w, 1) + S(w))
    wa2 = 0.5 * (S(w) + S(w, -1))
    ua1 = 0.5 * (S(u, 0, 0, 1) + S(u))
    ua2 = 0.5 * (S(u, -1, 0, 1) + S(u, -1))
    Wt = Wt - (ua1 * wa1 - ua2 * wa2) * M(0, "rdxc")
    wa1 = 0.5 * (S(w, 0, 1) + S(w))
    wa2 = 0.5 * (S(w) + S(w, 0, -1))
    va1 = 0.5 * (S(v, 0, 0, 1) + S(v))
    va2 = 0.5 * (S(v, 0, -1, 1) + S(v, 0, -1))
    Wt = Wt - (va1 * wa1 - va2 * wa2) * M(1, "rdxc")
    if les:
        nu = f["nuT"]  # NSsolver.F90:1339-1356
        n1 = 0.25 * (S(nu) + S(nu, -1) + S(nu, 0, 0, 1) + S(nu, -1, 0, 1))
        n2 = 0.25 * (S(nu) + S(nu, 1) + S(nu, 0, 0, 1) + S(nu, 1, 0, 1))
        Wt = Wt - 1 * 1.0 * (n2 * (S(w, 1) - S(w)) * M(0, "rdxe") - n1 * (S(w) - S(w, -1)) * M(0, "rdxe", -1)) \
            * M(0, "rdxc")
        Wt = Wt - 1 * 1.0 * (n2 * (S(u, 1, 0, 1) - S(u, 1)) * M(2, "rdxe") - n1 * (S(u, 0, 0, 1) - S(u))
                             * M(2, "rdxe")) * M(0, "rdxc")
        n1 = 0.25 * (S(nu) + S(nu, 0, -1) + S(nu, 0, 0, 1) + S(nu, 0, -1, 1))
        n2 = 0.25 * (S(nu) + S(nu, 0, 1) + S(nu, 0, 0, 1) + S(nu, 0, 1, 1))
        Wt = Wt - 1 * 1.0 * (n2 * (S(w, 0, 1) - S(w)) * M(1, "rdxe") - n1 * (S(w) - S(w, 0, -1)) * M(1, "rdxe", -1)) \
            * M(1, "rdxc")
        Wt = Wt - 1 * 1.0 * (n2 * (S(v, 0, 1, 1) - S(v, 0, 1)) * M(2, "rdxe") - n1 * (S(v, 0, 0, 1) - S(v))
                             * M(2, "rdxe")) * M(1, "rdxc")
    if ew:  # the loops run to k = ez - EW
        Wt[:, :, -1] = 0.0
    return Wt


def scalar_rhs(f, h, name, D, r_weighted, les=False):
    S, M = h.S, h.M
    u, v, w, r, c = f["u"], f["v"], f["w"], f["r"], f[name]
    St = 0.0 + (D * ((S(c, 1) - S(c)) * M(0, "rdxe") - (S(c) - S(c, -1)) * M(0, "rdxe", -1)) * M(0, "rdxc")
                + D * ((S(c, 0, 1) - S(c)) * M(1, "rdxe") - (S(c) - S(c, 0, -1)) * M(1, "rdxe", -1))
                * M(1, "rdxc"))
    c2 = 0.5 * (S(c, 1) + S(c))
    c1 = 0.5 * (S(c) + S(c, -1))
    St = St + (S(u, -1) * c1 - S(u) * c2) * M(0, "rdxc")
    c2 = 0.5 * (S(c, 0, 1) + S(c))
    c1 = 0.5 * (S(c) + S(c, 0, -1))
    St = St + (S(v, 0, -1) * c1 - S(v) * c2) * M(1, "rdxc")
    c2 = 0.5 * (S(c, 0, 0, 1) + S(c))
    c1 = 0.5 * (S(c) + S(c, 0, 0, -1))
    if r_weighted:
        ra2 = 0.5 * (S(r, 0, 0, 1) + S(r))
        ra1 = 0.5 * (S(r) + S(r, 0, 0, -1))
        St = St + (ra1 * S(w, 0, 0, -1) * c1 - ra2 * S(w) * c2) * M(2, "rdxc") / S(r)
    else:
        St = St + (S(w, 0, 0, -1) * c1 - S(w) * c2) * M(2, "rdxc")
    if not les:
        return St
    # rho_rhs / scal1_rhs eddy terms (NSsolver.F90:1778-1793, 1962-1977);
    # scal1 keeps the reference's nappaT(i) - nappaT(i-1) in the lower average
    kT = f["kappaT" if r_weighted else "nappaT"]
    k2 = 0.5 * (S(kT, 1) + S(kT))
    k1 = 0.5 * (S(kT) + S(kT, -1)) if r_weighted else 0.5 * (S(kT) - S(kT, -1))
    St = St - 1 * 1.0 * (k2 * (S(c, 1) - S(c)) * M(0, "rdxe") - k1 * (S(c) - S(c, -1)) * M(0, "rdxe", -1)) \
        * M(0, "rdxc")
    k2 = 0.5 * (S(kT, 0, 1) + S(kT))
    k1 = 0.5 * (S(kT) + S(kT, 0, -1)) if r_weighted else 0.5 * (S(kT) - S(kT, 0, -1))
    return St - 1 * 1.0 * (k2 * (S(c, 0, 1) - S(c)) * M(1, "rdxe") - k1 * (S(c) - S(c, 0, -1)) * M(1, "rdxe", -1)) \
        * M(1, "rdxc")


def _case(les):
    g = G.shear_layer_grid(16, 8, 24, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=RE, Pr=PR, Sc=SC, g=GRAV, ew=1, scal1_on=1, les=les)
    rng = np.random.default_rng(3)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w", "rho", "scal1"):
        f[k][...] = rng.standard_normal(g.ghosted)
    if les:  # eddy coefficients of either sign, ghosts included
        for k in ("nuT", "kappaT", "nappaT"):
            f[k] = np.asfortranarray(0.01 * rng.standard_normal(g.ghosted))
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    f["rho"] += f["densityBG"]
    o = OracleNS(g, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    return g, f, o


@pytest.fixture(scope="module", params=[False, True], ids=["dns", "les"])
def case(request):
    return (*_case(request.param), request.param)


@pytest.mark.parametrize("name", ["u", "v", "w", "rho", "scal1"])
def test_rhs_equals_restatement(case, name):
    g, f, o, les = case
    h = _Shift(g)
    rRe = 1.0 / RE
    ref = {"u": lambda: u1_rhs(f, h, rRe, les),
           "v": lambda: u2_rhs(f, h, rRe, les),
           "w": lambda: u3_rhs(f, h, rRe, GRAV, ew=1, les=les),
           "rho": lambda: scalar_rhs(f, h, "rho", rRe * (1.0 / PR), True, les),
           "scal1": lambda: scalar_rhs(f, h, "scal1", rRe * (1.0 / SC), False, les)}[name]()
    got = o.rhs(name)[1:-1, 1:-1, 1:-1]
    assert np.abs(ref).max() > 0
    np.testing.assert_array_equal(got, ref)


def test_gravity_ramp_in_buoyancy():
    """gravity (ANELASTIC_SL/dns/Routines.F90:27-52): g = 0 before GT1, the
    linear ramp g_orig (t - GT1)/(GT2 - GT1) strictly between, g_orig from
    GT2 on, and at t = GT1 < GT2 the previous value is kept (no branch
    applies).  Checked through u3_rhs's buoyancy term at several times."""
    g = G.shear_layer_grid(16, 8, 24, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=RE, Pr=PR, Sc=SC, g=GRAV, ew=1, scal1_on=1)
    g_init, g_final, t1, t2 = -0.03, -0.2, 0.5, 1.5
    nsp.g_init, nsp.g_final, nsp.gt1, nsp.gt2 = g_init, g_final, t1, t2
    rng = np.random.default_rng(9)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w", "rho", "scal1"):
        f[k][...] = rng.standard_normal(g.ghosted)
    o = OracleNS(g, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    h = _Shift(g)
    expect = [(1.0, g_final * (1.0 - t1) / (t2 - t1)), (0.2, 0.0), (t1, 0.0), (2.0, g_final),
              (t1, g_final)]
    for t, gv in expect:  # t1 keeps the value of the call before it
        o.set_clock(t, 1)
        ref = u3_rhs(f, h, 1.0 / RE, gv, ew=1)
        np.testing.assert_array_equal(o.rhs("w")[1:-1, 1:-1, 1:-1], ref, err_msg=f"t={t}")
