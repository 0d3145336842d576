"""The oracle's finest-level multigrid passes, restated from the reference
(CPU only).

- mg_bdry (ANELASTIC_SL/mgMK/mg_bdry.F90:72-190), serial form: the periodic
  wrap of all six ghost planes, then the faces in the order X2max, X3min,
  X2min, X3max, X1min, X1max, each over its whole plane: Neumann
  phi_g = phi_b -/+ phibc * dc (the level's cell size next to the face),
  Dirichlet phi_g = phibc;
- one mg_relaxRB iteration (mgMK/mg_relax.F90:85-179): colour (i+j+k) even,
  boundary pass, colour odd, boundary pass, each cell
  phi = (f - (c1 phi_W + c2 phi_E + c3 phi_S + c4 phi_N + c5 phi_B +
  c6 phi_T)) / c7 in that order, with mgdpfpde's fine coefficients
  (mgMK/mg_pfpde.F90:34-56, literal mode, anelastic r(z));
- one mg_relaxLz iteration (the LJ smoother, mgMK/mg_relax.F90:423-538):
  (i+j) red-black z-lines with mg_coeff's 1-D coefficients and the
  reference's Thomas routine;
- one iteration of this build's ZLINE smoother in metric mode, against its
  description: (i+j) red-black z-lines of the level's own 7-point operator
  (the projection's Psource(Pgrad(.)) with face densities), Thomas order.

All are numpy on whole planes or colours; the oracle's ghost cells and
interior must equal them bit for bit, for periodic-x/y walls-in-z and for
walls everywhere with non-zero boundary values.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleMG

from .helpers import levels_for

CASES = {
    "periodic_xy": ((0, 1, 0, 1, 0, 0), (0.0, 0.3, 0.0, -0.7, 0.0, 0.0)),
    "walls": ((2, 1, 1, 2, 1, 2), (0.4, -0.2, 0.9, 1.3, -0.6, 0.25)),
}


def mg_bdry(phi, g, tbc, vbc):
    p = phi
    p[0, :, :] = p[-2, :, :]
    p[-1, :, :] = p[1, :, :]
    p[:, 0, :] = p[:, -2, :]
    p[:, -1, :] = p[:, 1, :]
    p[:, :, 0] = p[:, :, -2]
    p[:, :, -1] = p[:, :, 1]
    dx, dy, dz = g.x.dxc, g.y.dxc, g.z.dxc
    nx, ny, nz = g.shape
    # X2max, X3min, X2min, X3max, X1min, X1max
    if tbc[0] == 1:
        p[:, -1, :] = p[:, -2, :] + vbc[0] * dy[ny]
    elif tbc[0] == 2:
        p[:, -1, :] = vbc[0]
    if tbc[1] == 1:
        p[:, :, 0] = p[:, :, 1] - vbc[1] * dz[1]
    elif tbc[1] == 2:
        p[:, :, 0] = vbc[1]
    if tbc[2] == 1:
        p[:, 0, :] = p[:, 1, :] - vbc[2] * dy[1]
    elif tbc[2] == 2:
        p[:, 0, :] = vbc[2]
    if tbc[3] == 1:
        p[:, :, -1] = p[:, :, -2] + vbc[3] * dz[nz]
    elif tbc[3] == 2:
        p[:, :, -1] = vbc[3]
    if tbc[4] == 1:
        p[0, :, :] = p[1, :, :] - vbc[4] * dx[1]
    elif tbc[4] == 2:
        p[0, :, :] = vbc[4]
    if tbc[5] == 1:
        p[-1, :, :] = p[-2, :, :] + vbc[5] * dx[nx]
    elif tbc[5] == 2:
        p[-1, :, :] = vbc[5]


def literal_coefficients(g, r):
    """mgdpfpde: c1..c7 on the interior (r ghosted)."""
    nx, ny, nz = g.shape
    t = [1.0 / ((ax.L / float(np.float32(ax.n))) * (ax.L / float(np.float32(ax.n)))) for ax in (g.x, g.y, g.z)]
    rk, rm, rp = r[1:-1, 1:-1, 1:-1], r[1:-1, 1:-1, :-2], r[1:-1, 1:-1, 2:]
    h = float(np.float32(0.5))
    c5 = t[2] * h * (rk + rm) / rm
    c6 = t[2] * h * (rk + rp) / rp
    c7 = -(t[0] + t[0] + t[1] + t[1] + (t[2] * h * (rk + rm) / rk) + (t[2] * h * (rk + rp) / rk))
    return t[0], t[0], t[1], t[1], c5, c6, c7


def rb_iteration(phi, src, g, r, tbc, vbc):
    c1, c2, c3, c4, c5, c6, c7 = literal_coefficients(g, r)
    nx, ny, nz = g.shape
    i, j, k = np.meshgrid(np.arange(2, nx + 2), np.arange(2, ny + 2), np.arange(2, nz + 2), indexing="ij")
    for colour in (0, 1):
        p = phi
        new = (src[1:-1, 1:-1, 1:-1] - (c1 * p[:-2, 1:-1, 1:-1] + c2 * p[2:, 1:-1, 1:-1] + c3 * p[1:-1, :-2, 1:-1]
                                         + c4 * p[1:-1, 2:, 1:-1] + c5 * p[1:-1, 1:-1, :-2]
                                         + c6 * p[1:-1, 1:-1, 2:])) / c7
        mask = (i + j + k) % 2 == colour
        p[1:-1, 1:-1, 1:-1] = np.where(mask, new, p[1:-1, 1:-1, 1:-1])
        mg_bdry(phi, g, tbc, vbc)


def _case(name):
    tbc, vbc = CASES[name]
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    p = abi.make_mg_params(levels_for(g), tbc=tbc, vbc=vbc, mode=abi.MODE_LITERAL)
    o = OracleMG(g, p)
    f = {"r": np.zeros(g.ghosted, order="F"), "densityBG": np.zeros(g.ghosted, order="F")}
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    o.set_density(f["r"])
    return g, o, f["r"], tbc, vbc


@pytest.mark.parametrize("name", list(CASES))
def test_boundary_pass_equals_restatement(name):
    g, o, r, tbc, vbc = _case(name)
    rng = np.random.default_rng(2)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    ref = phi.copy(order="F")
    o.debug_pass(1, phi, np.zeros(g.ghosted, order="F"))
    mg_bdry(ref, g, tbc, vbc)
    np.testing.assert_array_equal(phi, ref)


@pytest.mark.parametrize("name", list(CASES))
def test_rb_iteration_equals_restatement(name):
    g, o, r, tbc, vbc = _case(name)
    rng = np.random.default_rng(4)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    src = np.asfortranarray(rng.standard_normal(g.ghosted))
    ref = phi.copy(order="F")
    o.debug_pass(0, phi, src.copy(order="F"))
    rb_iteration(ref, src, g, r, tbc, vbc)
    np.testing.assert_array_equal(phi, ref)


def pcf_fine(g, tbc):
    """mg_coeff's 1-D line coefficients on the finest level
    (mgMK/mg_coeff.F90:77-145): p1 = 1/(dxc(i) dxe(i-1)), p2 = 1/(dxc(i)
    dxe(i)), and the same in y and z, with the finest level's Neumann
    zeroing of the wall coefficients.  Arrays over the interior."""
    out = []
    for ax, lo, hi in ((g.x, 4, 5), (g.y, 2, 0), (g.z, 1, 3)):
        n = ax.n
        dc, de = ax.dxc[1:n + 1], ax.dxe
        pm = 1.0 / (dc * de[0:n])
        pp = 1.0 / (dc * de[1:n + 1])
        if tbc[lo] == 1:
            pm[0] = 0.0
        if tbc[hi] == 1:
            pp[-1] = 0.0
        out += [pm, pp]
    return out


def lz_iteration(phi, src, g, tbc, vbc):
    """One mg_relaxLz iteration (mgMK/mg_relax.F90:423-538): (i+j)
    red-black z-lines, each the tridiagonal (a = p5, b = -(p1+p2+p3+p4+p5+p6),
    c = p6) with the ghost term inside the neighbour sum of the end rows,
    solved by the reference's Thomas routine; boundary pass per colour."""
    p1, p2, p3, p4, p5, p6 = pcf_fine(g, tbc)
    nx, ny, nz = g.shape
    P1, P2 = p1[:, None, None], p2[:, None, None]
    P3, P4 = p3[None, :, None], p4[None, :, None]
    a = np.broadcast_to(p5[None, None, :], (nx, ny, nz)).copy()
    b = np.broadcast_to(-(P1 + P2 + P3 + P4 + p5[None, None, :] + p6[None, None, :]), (nx, ny, nz)).copy()
    c = np.broadcast_to(p6[None, None, :], (nx, ny, nz)).copy()
    i, j = np.meshgrid(np.arange(2, nx + 2), np.arange(2, ny + 2), indexing="ij")
    for colour in (0, 1):
        p = phi
        W, E = p[:-2, 1:-1, 1:-1], p[2:, 1:-1, 1:-1]
        S_, N = p[1:-1, :-2, 1:-1], p[1:-1, 2:, 1:-1]
        f = src[1:-1, 1:-1, 1:-1]
        rhs = f - (P1 * W + P2 * E + P3 * S_ + P4 * N)
        rhs[:, :, 0] = f[:, :, 0] - (P1[:, :, 0] * W[:, :, 0] + P2[:, :, 0] * E[:, :, 0] + P3[:, :, 0] * S_[:, :, 0]
                                     + P4[:, :, 0] * N[:, :, 0] + p5[0] * p[1:-1, 1:-1, 0])
        rhs[:, :, -1] = f[:, :, -1] - (P1[:, :, 0] * W[:, :, -1] + P2[:, :, 0] * E[:, :, -1]
                                       + P3[:, :, 0] * S_[:, :, -1] + P4[:, :, 0] * N[:, :, -1]
                                       + p6[-1] * p[1:-1, 1:-1, -1])
        aa, bb, G_ = a.copy(), b.copy(), rhs
        for q in range(nz - 1):
            aa[..., q + 1] = -aa[..., q + 1] / bb[..., q]
            bb[..., q + 1] = bb[..., q + 1] + aa[..., q + 1] * c[..., q]
            G_[..., q + 1] = G_[..., q + 1] + aa[..., q + 1] * G_[..., q]
        G_[..., nz - 1] = G_[..., nz - 1] / bb[..., nz - 1]
        for q in range(nz - 2, -1, -1):
            G_[..., q] = (G_[..., q] - c[..., q] * G_[..., q + 1]) / bb[..., q]
        mask = ((i + j) % 2 == colour)[:, :, None]
        p[1:-1, 1:-1, 1:-1] = np.where(mask, G_, p[1:-1, 1:-1, 1:-1])
        mg_bdry(phi, g, tbc, vbc)


@pytest.mark.parametrize("name", list(CASES))
def test_lz_iteration_equals_restatement(name):
    tbc, vbc = CASES[name]
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    p = abi.make_mg_params(levels_for(g), tbc=tbc, vbc=vbc, mode=abi.MODE_LITERAL, smoother=abi.SMOOTHER_LJ)
    o = OracleMG(g, p)
    rng = np.random.default_rng(6)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    src = np.asfortranarray(rng.standard_normal(g.ghosted))
    ref = phi.copy(order="F")
    o.debug_pass(0, phi, src.copy(order="F"))
    lz_iteration(ref, src, g, tbc, vbc)
    np.testing.assert_array_equal(phi, ref)


def metric_coefficients(g, r, tbc):
    """The metric-mode fine operator (this build's extension, the
    projection's Psource(Pgrad(.)) in coefficient form): a1 = rdxc(i)
    rdxe(i-1), a2 = rdxc(i) rdxe(i) and likewise in y and z, a Neumann wall
    face's coefficient zeroed, the z ones weighted by the face densities,
    and the diagonal minus the sum of the six."""
    nx, ny, nz = g.shape

    def pair(ax):
        n = ax.n
        return ax.rdxc[1:n + 1] * ax.rdxe[0:n], ax.rdxc[1:n + 1] * ax.rdxe[1:n + 1]

    (a1, a2), (a3, a4), (a5, a6) = pair(g.x), pair(g.y), pair(g.z)
    a1 = np.broadcast_to(a1[:, None, None], (nx, ny, nz)).copy()
    a2 = np.broadcast_to(a2[:, None, None], (nx, ny, nz)).copy()
    a3 = np.broadcast_to(a3[None, :, None], (nx, ny, nz)).copy()
    a4 = np.broadcast_to(a4[None, :, None], (nx, ny, nz)).copy()
    a5 = np.broadcast_to(a5[None, None, :], (nx, ny, nz)).copy()
    a6 = np.broadcast_to(a6[None, None, :], (nx, ny, nz)).copy()
    if tbc[4] == 1:
        a1[0] = 0.0
    if tbc[5] == 1:
        a2[-1] = 0.0
    if tbc[2] == 1:
        a3[:, 0] = 0.0
    if tbc[0] == 1:
        a4[:, -1] = 0.0
    if tbc[1] == 1:
        a5[:, :, 0] = 0.0
    if tbc[3] == 1:
        a6[:, :, -1] = 0.0
    rp, rb, rt = r[1:-1, 1:-1, 1:-1], r[1:-1, 1:-1, :-2], r[1:-1, 1:-1, 2:]
    w5 = 0.5 * (rp + rb)
    w6 = 0.5 * (rp + rt)
    c7 = -(a1 + a2 + a3 + a4 + a5 * w5 / rp + a6 * w6 / rp)
    return a1, a2, a3, a4, a5 * w5 / rb, a6 * w6 / rt, c7


def zline_iteration(phi, src, g, r, tbc, vbc):
    """One ZLINE iteration: (i+j) red-black z-lines of the level's own
    7-point operator (a = c5, b = c7, c = c6; the ghost terms subtracted
    after the horizontal neighbour sum), the reference's Thomas routine,
    and the boundary pass after each colour."""
    c1, c2, c3, c4, c5, c6, c7 = metric_coefficients(g, r, tbc)
    nx, ny, nz = g.shape
    i, j = np.meshgrid(np.arange(2, nx + 2), np.arange(2, ny + 2), indexing="ij")
    for colour in (0, 1):
        p = phi
        rhs = src[1:-1, 1:-1, 1:-1] - (c1 * p[:-2, 1:-1, 1:-1] + c2 * p[2:, 1:-1, 1:-1] + c3 * p[1:-1, :-2, 1:-1]
                                        + c4 * p[1:-1, 2:, 1:-1])
        rhs[:, :, 0] = rhs[:, :, 0] - c5[:, :, 0] * p[1:-1, 1:-1, 0]
        rhs[:, :, -1] = rhs[:, :, -1] - c6[:, :, -1] * p[1:-1, 1:-1, -1]
        aa, bb, G_ = c5.copy(), c7.copy(), rhs
        for q in range(nz - 1):
            aa[..., q + 1] = -aa[..., q + 1] / bb[..., q]
            bb[..., q + 1] = bb[..., q + 1] + aa[..., q + 1] * c6[..., q]
            G_[..., q + 1] = G_[..., q + 1] + aa[..., q + 1] * G_[..., q]
        G_[..., nz - 1] = G_[..., nz - 1] / bb[..., nz - 1]
        for q in range(nz - 2, -1, -1):
            G_[..., q] = (G_[..., q] - c6[..., q] * G_[..., q + 1]) / bb[..., q]
        mask = ((i + j) % 2 == colour)[:, :, None]
        p[1:-1, 1:-1, 1:-1] = np.where(mask, G_, p[1:-1, 1:-1, 1:-1])
        mg_bdry(phi, g, tbc, vbc)


@pytest.mark.parametrize("name", list(CASES))
def test_zline_iteration_equals_restatement(name):
    """The ZLINE smoother of the metric mode (this build's extension) against
    its description, with an anelastic r(z) on the stretched grid."""
    tbc, vbc = CASES[name]
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    p = abi.make_mg_params(levels_for(g), tbc=tbc, vbc=vbc, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE)
    o = OracleMG(g, p)
    f = {"r": np.zeros(g.ghosted, order="F"), "densityBG": np.zeros(g.ghosted, order="F")}
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    o.set_density(f["r"])
    rng = np.random.default_rng(9)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    src = np.asfortranarray(rng.standard_normal(g.ghosted))
    ref = phi.copy(order="F")
    o.debug_pass(0, phi, src.copy(order="F"))
    zline_iteration(ref, src, g, f["r"], tbc, vbc)
    np.testing.assert_array_equal(phi, ref)
