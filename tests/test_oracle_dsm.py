"""The oracle's dynamic Smagorinsky model, restated from the reference
(CPU only).

DSM (ANELASTIC_SL/les/DSM.F90:1-258, C_avg_dir = 12) with its test filter
(filter type 2, les/filter.F90:1-149, including the zero-weight terms and
the boundary formulas, the upper one summed from the ghost inwards), the
coefficient smoothing filterHF (:152-288), the cell-centred velocities of
center_velocity (dns/StatTools.F90:87-289), the x-y plane averages of
avgX1X2 (dns/Average.F90:279-368, summed sequentially in its j-outer,
i-inner order) and the restated boundary pass, all in numpy.  DSM's
off-diagonal strain components subtract the two cross derivatives, as the
source writes them.  DSMrho and DSMscal1 (les/DSMrho.F90:1-240, the
same routine on scal1 in DSMscal1.F90) are restated the same way.  On
random fields the oracle's nuT, kappaT and nappaT from the dynamic
coefficients must equal the restatement bit for bit, on the reference
runfile's uniform grid with filters in x, y and z, for the velocity model
also with the filter off in one direction, and on a tanh-stretched z axis
with the corrected five-point centring.
"""
import math

import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for
from .test_oracle_ghost import ghost as ghost_restated
from .test_oracle_les import filter_width, strain_magnitude
from .test_oracle_rhs import _Shift

CFLUC, VT_U, VT_V, VT_W = 5, 0, 1, 2
RATIO = math.sqrt(6.0)
WA = (0.0, 1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0, 0.0)
WAB = (1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0, 0.0, 0.0)


class _Ctx:
    def __init__(self, g, nsp, filt):
        self.g, self.nsp, self.filt = g, nsp, filt

    def ghost(self, a, vt):
        ghost_restated(a, self.g, vt, self.nsp.tb, self.nsp.vb, self.nsp.ew)


def _pencils(a, d):
    """View of a with axis d last, the other two axes restricted to their
    interior."""
    v = np.moveaxis(a, d, -1)
    return v[1:-1, 1:-1, :]


def filter2(c, var, vt):
    """filter(var, out, 2, xfil, yfil, zfil, vt): per direction, then ghost."""
    out = var.copy(order="F")
    for d in range(3):
        if c.filt[d]:
            n = c.g.shape[d]
            v = _pencils(out, d)
            P = v.copy()
            new = P.copy()
            for t in range(2, n):  # Fortran sx+1 .. ex-1
                new[..., t] = (WA[0] * P[..., t - 2] + WA[1] * P[..., t - 1] + WA[2] * P[..., t]
                               + WA[3] * P[..., t + 1] + WA[4] * P[..., t + 2])
            new[..., 1] = (WAB[0] * P[..., 0] + WAB[1] * P[..., 1] + WAB[2] * P[..., 2] + WAB[3] * P[..., 3]
                           + WAB[4] * P[..., 4])
            new[..., n] = (WAB[0] * P[..., n + 1] + WAB[1] * P[..., n] + WAB[2] * P[..., n - 1]
                           + WAB[3] * P[..., n - 2] + WAB[4] * P[..., n - 3])
            v[..., 1:n + 1] = new[..., 1:n + 1]
        c.ghost(out, vt)
    return out


def filter_hf(c, var, vt):
    """filterHF(var, out, 2, 1, 1, 1, vt): a strict local extremum of its
    pencil takes the 3-point average when that is still such an extremum."""
    out = var.copy(order="F")
    w = (1.0 / 4.0, 1.0 / 2.0, 1.0 / 4.0)
    for d in range(3):
        n = c.g.shape[d]
        v = _pencils(out, d)
        P = v.copy()
        p0, pm, pp = P[..., 1:n + 1], P[..., 0:n], P[..., 2:n + 2]
        x = w[0] * pm + w[1] * p0 + w[2] * pp
        lo = (p0 < pp) & (p0 < pm)
        hi = (p0 > pp) & (p0 > pm)
        take = (lo & (x < pp) & (x < pm)) | (~lo & hi & (x > pp) & (x > pm))
        v[..., 1:n + 1] = np.where(take, x, p0)
        c.ghost(out, vt)
    return out


def center_uniform(c, a, d):
    out = np.zeros_like(a, order="F")
    src = _pencils(a, d)
    dst = _pencils(out, d)
    n = c.g.shape[d]
    dst[..., 1:n + 1] = 0.5 * (src[..., 1:n + 1] + src[..., 0:n])
    c.ghost(out, (VT_U, VT_V, VT_W)[d])
    return out


def _newton5(x, y, loc):
    """divdiffs(x, y, a, 4) and the Newton form at loc (StatTools.F90:563-653)."""
    d = [list(y)]
    for j in range(1, 5):
        prev = d[-1]
        d.append([None] * j + [(prev[k] - prev[k - 1]) / (x[k] - x[k - j]) for k in range(j, 5)])
    a = [d[k][k] for k in range(5)]
    s = a[4]
    for k in range(3, -1, -1):
        s = s * (loc - x[k]) + a[k]
    return s


def center(c, a, d):
    """center_velocity along d: the two-point mean on a uniform axis, else
    the five-point interpolation (the values over the edges when the
    interpolation is CORRECTED; LITERAL hands the values to divdiffs as
    abscissae, as the reference does)."""
    if not c.nsp.stretched[d]:
        return center_uniform(c, a, d)
    out = np.zeros_like(a, order="F")
    src, dst = _pencils(a, d), _pencils(out, d)
    ax = (c.g.x, c.g.y, c.g.z)[d]
    n = ax.n
    corrected = c.nsp.interp == abi.DIAG_CORRECTED
    with np.errstate(divide="ignore", invalid="ignore"):
        for q in range(2, n + 2):  # Fortran index of the centred value
            lo = 1 if q == 2 else (n - 2 if q == n + 1 else q - 2)
            dep = [src[..., lo - 1 + m] for m in range(5)]
            ind = [ax.xe[lo - 1 + m] for m in range(5)]
            loc = ax.xc[q - 1]
            dst[..., q - 1] = _newton5(ind, dep, loc) if corrected else _newton5(dep, ind, loc)
    c.ghost(out, (VT_U, VT_V, VT_W)[d])
    return out


def dsm_component(f, h, ij):
    S, M = h.S, h.M
    u, v, w = f["u"], f["v"], f["w"]
    if ij == 1:
        return (S(u, 1) - S(u)) * M(0, "rdxc")
    if ij == 2:
        return (S(v, 0, 1) - S(v)) * M(1, "rdxc")
    if ij == 3:
        return (S(w, 0, 0, 1) - S(w)) * M(2, "rdxc")
    if ij == 4:
        t1 = 0.25 * (S(u) + S(u, 1) + S(u, 0, 1) + S(u, 1, 1))
        t2 = 0.25 * (S(u) + S(u, 1) + S(u, 0, -1) + S(u, 1, -1))
        t3 = 0.25 * (S(v) + S(v, 0, 1) + S(v, 1) + S(v, 1, 1))
        t4 = 0.25 * (S(v) + S(v, 0, 1) + S(v, -1) + S(v, -1, 1))
        return 0.5 * ((t1 - t2) * M(1, "rdxc") - (t3 - t4) * M(0, "rdxc"))
    if ij == 5:
        t1 = 0.25 * (S(u) + S(u, 1) + S(u, 0, 0, 1) + S(u, 1, 0, 1))
        t2 = 0.25 * (S(u) + S(u, 1) + S(u, 0, 0, -1) + S(u, 1, 0, -1))
        t3 = 0.25 * (S(w) + S(w, 0, 0, 1) + S(w, 1) + S(w, 1, 0, 1))
        t4 = 0.25 * (S(w) + S(w, 0, 0, 1) + S(w, -1) + S(w, -1, 0, 1))
        return 0.5 * ((t1 - t2) * M(2, "rdxc") - (t3 - t4) * M(0, "rdxc"))
    t1 = 0.25 * (S(v) + S(v, 0, 1) + S(v, 0, 0, 1) + S(v, 0, 1, 1))
    t2 = 0.25 * (S(v) + S(v, 0, 1) + S(v, 0, 0, -1) + S(v, 0, 1, -1))
    t3 = 0.25 * (S(w) + S(w, 0, 0, 1) + S(w, 0, 1) + S(w, 0, 1, 1))
    t4 = 0.25 * (S(w) + S(w, 0, 0, 1) + S(w, 0, -1) + S(w, 0, -1, 1))
    return 0.5 * ((t1 - t2) * M(2, "rdxc") - (t3 - t4) * M(1, "rdxc"))


def avg_x1x2(c, var):
    """avgX1X2(var, outm, 'cfluc'): sum var*dxc*dyc / Area per plane, in
    the loop order (i fastest), sequentially."""
    c.ghost(var, CFLUC)
    g = c.g
    dx, dy = g.x.dxc[1:-1, None], g.y.dxc[None, 1:-1]
    area = np.add.accumulate((dx * dy).reshape(-1, order="F"))[-1]
    out = np.empty(var.shape[2])
    for k in range(var.shape[2]):
        terms = (var[1:-1, 1:-1, k] * dx) * dy  # var*dxc*dyc, left to right
        out[k] = np.add.accumulate(terms.reshape(-1, order="F"))[-1] / area
    return out


def dsm_csgs(c, f):
    g = c.g
    h = _Shift(g)
    inner = (slice(1, -1),) * 3
    dg = np.broadcast_to(filter_width(h, abi.DELTA_3ROOT), (g.x.n, g.y.n, g.z.n))
    modS = strain_magnitude(f, h)
    filt_vel = {k: filter2(c, f[k], vt) for k, vt in (("u", VT_U), ("v", VT_V), ("w", VT_W))}
    fmodS = np.zeros(g.ghosted, order="F")
    fmodS[inner] = strain_magnitude(filt_vel, h)
    c.ghost(fmodS, CFLUC)
    cen = [center(c, f[k], d) for d, k in enumerate(("u", "v", "w"))]
    fcen = [filter2(c, a, CFLUC) for a in cen]
    pa, pb = (0, 0, 1, 2, 0, 0, 1), (0, 0, 1, 2, 1, 2, 2)
    l4 = np.zeros(g.ghosted, order="F")
    csgs = np.zeros(g.ghosted, order="F")
    for ij in range(1, 7):
        l1 = np.zeros(g.ghosted, order="F")
        l1[inner] = dsm_component(f, h, ij)
        c.ghost(l1, CFLUC)
        l2 = np.zeros(g.ghosted, order="F")
        l2[inner] = (dg * dg) * modS * l1[inner]
        c.ghost(l2, CFLUC)
        l3 = filter2(c, l2, CFLUC)
        l2 = filter2(c, l1, CFLUC)
        l1 = fmodS.copy(order="F")
        rd = RATIO * dg
        l2[inner] = (rd * rd) * l1[inner] * l2[inner]
        c.ghost(l2, CFLUC)
        l3 = l3 - l2
        c.ghost(l3, CFLUC)
        l2 = filter2(c, cen[pa[ij]] * cen[pb[ij]], CFLUC)
        fa, fb = fcen[pa[ij]], fcen[pb[ij]]
        if ij <= 3:
            l4 = l4 + l3 * l2
            l4 = l4 - l3 * fa * fb
            csgs = csgs + l3 * l3
        else:
            l4 = l4 + 2.0 * l3 * l2
            l4 = l4 - 2.0 * l3 * fa * fb
            csgs = csgs + 2.0 * l3 * l3
    num, den = l4.copy(order="F"), csgs.copy(order="F")
    c.ghost(num, CFLUC)
    c.ghost(den, CFLUC)
    pn, pd = avg_x1x2(c, num), avg_x1x2(c, den)
    num[inner] = np.broadcast_to(pn[1:-1], num[inner].shape)
    den[inner] = np.broadcast_to(pd[1:-1], den[inner].shape)
    num[inner] = np.where(num[inner] < 0.0, 0.0, num[inner])
    c.ghost(num, CFLUC)
    c.ghost(den, CFLUC)
    out = np.zeros(g.ghosted, order="F")
    with np.errstate(divide="ignore", invalid="ignore"):
        out[inner] = np.where(den[inner] == 0.0, 1.0e-20, 0.5 * num[inner] / den[inner])
    c.ghost(out, CFLUC)
    out = filter_hf(c, out, CFLUC)
    c.ghost(out, CFLUC)
    return out, dg, modS


def dsm_scalar(c, f, name):
    """DSMrho / DSMscal1 (les/DSMrho.F90:1-240; DSMscal1.F90 is the same
    routine on scal1) of the scalar `name`: the dynamic coefficient."""
    g = c.g
    h = _Shift(g)
    S, M = h.S, h.M
    inner = (slice(1, -1),) * 3
    dg = np.broadcast_to(filter_width(h, abi.DELTA_3ROOT), (g.x.n, g.y.n, g.z.n))
    modS = strain_magnitude(f, h)
    filt_vel = {k: filter2(c, f[k], vt) for k, vt in (("u", VT_U), ("v", VT_V), ("w", VT_W))}
    fmodS = np.zeros(g.ghosted, order="F")
    fmodS[inner] = strain_magnitude(filt_vel, h)
    c.ghost(fmodS, CFLUC)
    q = f[name]
    vel = (f["u"], f["v"], f["w"])
    l4 = np.zeros(g.ghosted, order="F")
    C = np.zeros(g.ghosted, order="F")
    for ij in (1, 2, 3):
        d = ij - 1
        sh = [0, 0, 0]
        sh[d] = 1
        t1 = 0.5 * (S(q) + S(q, *[-v for v in sh]))
        t2 = 0.5 * (S(q) + S(q, *sh))
        rd = M(d, "rdxc")
        l1 = np.zeros(g.ghosted, order="F")
        l1[inner] = (dg * dg) * modS * (t2 - t1) * rd
        c.ghost(l1, CFLUC)
        l2 = filter2(c, l1, CFLUC)
        l1 = np.zeros(g.ghosted, order="F")
        l1[inner] = (t2 - t1) * rd
        c.ghost(l1, CFLUC)
        l3 = filter2(c, l1, CFLUC)
        l1 = fmodS.copy(order="F")
        rr = RATIO * dg
        l2[inner] = l2[inner] - (rr * rr) * l1[inner] * l3[inner]
        c.ghost(l2, CFLUC)
        l1 = np.zeros(g.ghosted, order="F")
        l1[inner] = S(q) * 0.5 * (S(vel[d], *[-v for v in sh]) + S(vel[d]))
        c.ghost(l1, CFLUC)
        l3 = filter2(c, l1, CFLUC)
        fc = filter2(c, center(c, vel[d], d), CFLUC)
        fq = filter2(c, q, CFLUC)
        l3 = l3 - fq * fc
        c.ghost(l3, CFLUC)
        l4 = l4 + l2 * l2
        C = C + l2 * l3
    num, den = C.copy(order="F"), l4.copy(order="F")
    c.ghost(num, CFLUC)
    c.ghost(den, CFLUC)
    pn, pd = avg_x1x2(c, num), avg_x1x2(c, den)
    num[inner] = np.broadcast_to(pn[1:-1], num[inner].shape)
    den[inner] = np.broadcast_to(pd[1:-1], den[inner].shape)
    num[inner] = np.where(num[inner] < 0.0, 0.0, num[inner])
    c.ghost(num, CFLUC)
    c.ghost(den, CFLUC)
    out = np.zeros(g.ghosted, order="F")
    with np.errstate(divide="ignore", invalid="ignore"):
        out[inner] = np.where(den[inner] == 0.0, 1.0e-20, 0.5 * num[inner] / den[inner])
    c.ghost(out, CFLUC)
    out = filter_hf(c, out, CFLUC)
    c.ghost(out, CFLUC)
    return out, dg, modS


@pytest.mark.parametrize("filt", [(1, 1, 1), (1, 0, 1)], ids=["xyz", "xz"])
def test_dynamic_csgs_equals_restatement(filt):
    g = G.shear_layer_grid(16, 8, 16, stretched=False)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=50000.0, g=-0.1, ew=1, scal1_on=1, les=True,
                             models=(abi.MODEL_DSM, abi.MODEL_SSM, abi.MODEL_SSM), test_ratio=RATIO,
                             filt=filt, stretched=(0, 0, 0), interp=abi.DIAG_LITERAL)
    rng = np.random.default_rng(5)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w"):
        f[k][...] = rng.standard_normal(g.ghosted)
    for k in ("nuT", "kappaT", "nappaT"):
        f[k] = np.zeros(g.ghosted, order="F")
    o = OracleNS(g, mgp, nsp, f)
    c = _Ctx(g, nsp, filt)
    for k, vt in (("u", VT_U), ("v", VT_V), ("w", VT_W)):
        c.ghost(f[k], vt)
    csgs, dg, modS = dsm_csgs(c, f)
    o.les_update()
    ref = -(csgs[1:-1, 1:-1, 1:-1] + 0.0) * (dg * dg) * modS + 0.0
    assert np.abs(ref).max() > 0
    np.testing.assert_array_equal(f["nuT"][1:-1, 1:-1, 1:-1], ref)


def test_dynamic_scalar_models_equal_restatement():
    """DSM, DSMrho and DSMscal1 together (the reference runfile's models)."""
    g = G.shear_layer_grid(16, 8, 16, stretched=False)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=50000.0, g=-0.1, ew=1, scal1_on=1, les=True, models=(abi.MODEL_DSM,) * 3,
                             test_ratio=RATIO, filt=(1, 1, 1), stretched=(0, 0, 0), interp=abi.DIAG_LITERAL)
    rng = np.random.default_rng(8)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w", "rho", "scal1"):
        f[k][...] = rng.standard_normal(g.ghosted)
    for k in ("nuT", "kappaT", "nappaT"):
        f[k] = np.zeros(g.ghosted, order="F")
    o = OracleNS(g, mgp, nsp, f)
    c = _Ctx(g, nsp, (1, 1, 1))
    for k, vt in (("u", VT_U), ("v", VT_V), ("w", VT_W), ("rho", 4), ("scal1", 12)):
        c.ghost(f[k], vt)
    o.les_update()
    for name, eddy in (("rho", "kappaT"), ("scal1", "nappaT")):
        C, dg, modS = dsm_scalar(c, f, name)
        ref = -(C[1:-1, 1:-1, 1:-1] + 0.0) * (dg * dg) * modS + 0.0
        assert np.abs(ref).max() > 0
        np.testing.assert_array_equal(f[eddy][1:-1, 1:-1, 1:-1], ref, err_msg=eddy)


@pytest.mark.parametrize("interp", [abi.DIAG_CORRECTED], ids=["corrected"])
def test_dynamic_models_on_stretched_z(interp):
    """The same restatement on a tanh-stretched z axis: the cell-centred
    velocities come from the five-point interpolation, delg varies with k."""
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = abi.make_ns_params(Re=50000.0, g=-0.1, ew=1, scal1_on=1, les=True, models=(abi.MODEL_DSM,) * 3,
                             test_ratio=RATIO, filt=(1, 1, 1), stretched=(0, 0, 1), interp=interp)
    rng = np.random.default_rng(31)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w", "rho", "scal1"):
        f[k][...] = rng.standard_normal(g.ghosted)
    for k in ("nuT", "kappaT", "nappaT"):
        f[k] = np.zeros(g.ghosted, order="F")
    o = OracleNS(g, mgp, nsp, f)
    c = _Ctx(g, nsp, (1, 1, 1))
    for k, vt in (("u", VT_U), ("v", VT_V), ("w", VT_W), ("rho", 4), ("scal1", 12)):
        c.ghost(f[k], vt)
    o.les_update()
    csgs, dg, modS = dsm_csgs(c, f)
    ref = -(csgs[1:-1, 1:-1, 1:-1] + 0.0) * (dg * dg) * modS + 0.0
    np.testing.assert_array_equal(f["nuT"][1:-1, 1:-1, 1:-1], ref, err_msg="nuT")
    for name, eddy in (("rho", "kappaT"), ("scal1", "nappaT")):
        C, dg, modS = dsm_scalar(c, f, name)
        ref = -(C[1:-1, 1:-1, 1:-1] + 0.0) * (dg * dg) * modS + 0.0
        np.testing.assert_array_equal(f[eddy][1:-1, 1:-1, 1:-1], ref, err_msg=eddy)
