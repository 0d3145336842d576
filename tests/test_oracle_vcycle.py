"""One V-cycle of the oracle's multigrid, restated from the reference (CPU
only).

mg_cycle (ANELASTIC_SL/mgMK/mg_cycle.F90:44-184) with the RBPGS smoother
in literal mode, in numpy:

- level sizes of MG_init (mgMK/mg_init.F90:70-351), including the levels
  where a direction is no longer coarsened;
- fine coefficients of mgdpfpde and coarse ones of mgdphpde
  (mgMK/mg_phpde.F90:40-142): the index maps km = 2 kstep k - 3 (kstep-1),
  Neumann zeroing of the wall coefficients, and the diagonal evaluated
  with the indices left over from the last cell of the coefficient loop
  (the same r values for every cell of the level);
- mg_relaxRB and mg_bdry per level (homogeneous values below the finest);
- mg_restr (mgMK/mg_restr.F90:114-241): coarse phi and f cleared, the fine
  residual f - (c1..c7 . phi), and the 8-, 4- or 2-child averages in the
  source's order;
- mg_cor (mgMK/mg_cor.F90:96-296): the 27/9/3/1 trilinear weights (and the
  bilinear and linear forms) in the source's term order, on the fine
  interior, then the boundary pass.

The oracle's V-cycle must equal it bit for bit, with full coarsening and
with a direction whose coarsening stops early, on a stretched grid with an
anelastic r(z) and non-zero boundary values on the finest level.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleMG

from .test_oracle_mg_passes import literal_coefficients, mg_bdry

TBC, VBC = (0, 1, 0, 1, 0, 0), (0.0, 0.3, 0.0, -0.7, 0.0, 0.0)


def level_sizes(shape, levels):
    """Interior cells per level k = 1..ngrid: n 2^(max(k+L-ngrid, 1) - L)."""
    ng = max(levels)
    return {k: tuple(n >> (L - max(k + L - ng, 1)) for n, L in zip(shape, levels)) for k in range(1, ng + 1)}


class _Level:
    def __init__(self, n, lengths):
        self.shape = n
        self.ghosted = tuple(v + 2 for v in n)
        self.L = lengths


def coarse_coefficients(fine_shape, nl, lengths, r, tbc):
    """mgdphpde on a level of nl interior cells; r is the finest level's
    ghosted density."""
    nm = [v + 1 for v in nl]          # nodes of the level
    nf = [v + 1 for v in fine_shape]  # nodes of the finest level
    e = [1.0 / ((lengths[d] / float(np.float32(nm[d] - 1))) * (lengths[d] / float(np.float32(nm[d] - 1))))
         for d in range(3)]
    step = [(nf[d] - 1) // (nm[d] - 1) for d in range(3)]
    h = float(np.float32(0.5))
    R = lambda k: r[1, 1, k - 1]     # r depends on z only; Fortran index k
    sh = tuple(nl)
    c1 = np.full(sh, e[0])
    c2 = np.full(sh, e[0])
    c3 = np.full(sh, e[1])
    c4 = np.full(sh, e[1])
    c5 = np.empty(sh)
    c6 = np.empty(sh)
    ks = 0
    for q in range(nl[2]):
        k = q + 2
        km = 2 * step[2] * k - 3 * (step[2] - 1)
        ks = (km - step[2]) // 2
        c5[:, :, q] = e[2] * h * (R(ks) + R(ks - 1)) / R(ks - 1)
        ks = (km + step[2]) // 2
        c6[:, :, q] = e[2] * h * (R(ks) + R(ks + 1)) / R(ks + 1)
    # Neumann zeroing: X2max, X3min, X2min, X3max, X1min, X1max
    if tbc[0] == 1:
        c4[:, -1, :] = 0.0
    if tbc[1] == 1:
        c5[:, :, 0] = 0.0
    if tbc[2] == 1:
        c3[:, 0, :] = 0.0
    if tbc[3] == 1:
        c6[:, :, -1] = 0.0
    if tbc[4] == 1:
        c1[0, :, :] = 0.0
    if tbc[5] == 1:
        c2[-1, :, :] = 0.0
    # the diagonal with the last cell's indices (ks of c6 at k = ezm)
    c7 = -(c1 + c2 + c3 + c4 + (e[2] * h * (R(ks) + R(ks - 1)) / R(ks)) + (e[2] * h * (R(ks) + R(ks + 1)) / R(ks)))
    return c1, c2, c3, c4, c5, c6, c7


def relax(phi, src, c, lv, iters, vbc):
    nx, ny, nz = lv.shape
    i, j, k = np.meshgrid(np.arange(2, nx + 2), np.arange(2, ny + 2), np.arange(2, nz + 2), indexing="ij")
    c1, c2, c3, c4, c5, c6, c7 = c
    for _ in range(iters):
        for colour in (0, 1):
            p = phi
            new = (src[1:-1, 1:-1, 1:-1] - (c1 * p[:-2, 1:-1, 1:-1] + c2 * p[2:, 1:-1, 1:-1]
                                             + c3 * p[1:-1, :-2, 1:-1] + c4 * p[1:-1, 2:, 1:-1]
                                             + c5 * p[1:-1, 1:-1, :-2] + c6 * p[1:-1, 1:-1, 2:])) / c7
            p[1:-1, 1:-1, 1:-1] = np.where((i + j + k) % 2 == colour, new, p[1:-1, 1:-1, 1:-1])
            mg_bdry(phi, lv.grid, TBC, vbc)


def residual(phi, src, c):
    c1, c2, c3, c4, c5, c6, c7 = c
    p = phi
    return src[1:-1, 1:-1, 1:-1] - (c1 * p[:-2, 1:-1, 1:-1] + c2 * p[2:, 1:-1, 1:-1] + c3 * p[1:-1, :-2, 1:-1]
                                    + c4 * p[1:-1, 2:, 1:-1] + c5 * p[1:-1, 1:-1, :-2] + c6 * p[1:-1, 1:-1, 2:]
                                    + c7 * p[1:-1, 1:-1, 1:-1])


def restrict(res, fine_n, coarse_n):
    """Coarse interior f from the fine residual (interior arrays)."""
    cx, cy, cz = (coarse_n[d] < fine_n[d] for d in range(3))

    def child(di, dj, dk):
        sl = []
        for d, (cd, o) in enumerate(zip((cx, cy, cz), (di, dj, dk))):
            sl.append(slice(o, None, 2) if cd else slice(0, None))
        return res[tuple(sl)]

    if cx and cy and cz:
        return 0.125 * (child(0, 0, 0) + child(0, 1, 0) + child(0, 0, 1) + child(0, 1, 1) + child(1, 0, 0)
                        + child(1, 1, 1) + child(1, 1, 0) + child(1, 0, 1))
    if not cx and not cy:
        return 0.5 * (child(0, 0, 0) + child(0, 0, 1))
    if not cx and not cz:
        return 0.5 * (child(0, 0, 0) + child(0, 1, 0))
    if not cy and not cz:
        return 0.5 * (child(0, 0, 0) + child(1, 0, 0))
    if not cx:
        return 0.25 * (child(0, 0, 0) + child(0, 1, 0) + child(0, 0, 1) + child(0, 1, 1))
    if not cy:
        return 0.25 * (child(0, 0, 0) + child(0, 0, 1) + child(1, 0, 0) + child(1, 0, 1))
    return 0.25 * (child(0, 0, 0) + child(1, 0, 0) + child(0, 1, 0) + child(1, 1, 0))


def prolong_add(phif, phic, fine_n, coarse_n):
    """phif interior += mg_cor's correction from the ghosted coarse phic."""
    co = [coarse_n[d] < fine_n[d] for d in range(3)]
    idx, wts = [], []
    for d in range(3):
        f = np.arange(2, fine_n[d] + 2)  # Fortran fine indices
        if co[d]:
            odd = f % 2 == 1
            base = np.where(odd, (f + 1) // 2, f // 2)
            w0 = np.where(odd, 3.0, 1.0)
            w1 = np.where(odd, 1.0, 3.0)
        else:
            base, w0, w1 = f, np.ones(f.size), np.zeros(f.size)
        idx.append(base - 1)  # 0-based coarse index of offset 0
        wts.append((w0, w1))
    ncoarse = sum(co)
    if ncoarse == 3:
        order = [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1), (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)]
        div = 64.0
    elif ncoarse == 2:
        a, b = [d for d in range(3) if co[d]]
        order = []
        for ob in (0, 1):
            for oa in (0, 1):
                o = [0, 0, 0]
                o[a], o[b] = oa, ob
                order.append(tuple(o))
        div = 16.0
    else:
        a = [d for d in range(3) if co[d]][0]
        order = [tuple(1 if d == a and o else 0 for d in range(3)) for o in (0, 1)]
        div = 4.0
    s = None
    for o in order:
        ii = idx[0][:, None, None] + o[0]
        jj = idx[1][None, :, None] + o[1]
        kk = idx[2][None, None, :] + o[2]
        w = 1.0
        for d, od in enumerate(o):
            if co[d]:
                wd = wts[d][od]
                sl = [None, None, None]
                sl[d] = slice(None)
                w = w * wd[tuple(sl)]
        term = w * phic[ii, jj, kk]
        s = term if s is None else s + term
    phif[1:-1, 1:-1, 1:-1] = phif[1:-1, 1:-1, 1:-1] + s / div


def vcycle(phi, src, g, levels, r, pre, post):
    sizes = level_sizes(g.shape, levels)
    ng = max(levels)
    L = (g.x.L, g.y.L, g.z.L)
    coef, lv, P, F = {}, {}, {}, {}
    for k in range(1, ng + 1):
        n = sizes[k]
        lv[k] = _Level(n, L)
        lv[k].grid = G.Grid(G.uniform_axis(n[0], 1.0), G.uniform_axis(n[1], 1.0), G.uniform_axis(n[2], 1.0))
        coef[k] = literal_coefficients(g, r) if k == ng else coarse_coefficients(g.shape, n, L, r, TBC)
    lv[ng].grid = g
    P[ng], F[ng] = phi, src
    zero = (0.0,) * 6

    def down(k):
        relax(P[k], F[k], coef[k], lv[k], pre[k - 1], VBC if k == ng else zero)
        res = residual(P[k], F[k], coef[k])
        P[k - 1] = np.zeros(lv[k - 1].ghosted, order="F")
        F[k - 1] = np.zeros(lv[k - 1].ghosted, order="F")
        F[k - 1][1:-1, 1:-1, 1:-1] = restrict(res, sizes[k], sizes[k - 1])

    for k in range(ng, 1, -1):
        down(k)
    relax(P[1], F[1], coef[1], lv[1], pre[0], zero)
    for k in range(1, ng):
        relax(P[k], F[k], coef[k], lv[k], post[k - 1], zero)
        prolong_add(P[k + 1], P[k], sizes[k + 1], sizes[k])
        mg_bdry(P[k + 1], lv[k + 1].grid, TBC, VBC if k + 1 == ng else zero)
    relax(P[ng], F[ng], coef[ng], lv[ng], post[ng - 1], VBC)


@pytest.mark.parametrize("levels", [(4, 3, 4), (4, 4, 3)], ids=["y_stops", "z_stops"])
def test_vcycle_equals_restatement(levels):
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    pre, post = [1, 2, 1, 2], [2, 1, 2, 1]
    p = abi.make_mg_params(levels, tbc=TBC, vbc=VBC, mode=abi.MODE_LITERAL, pre=pre, post=post)
    o = OracleMG(g, p)
    f = {"r": np.zeros(g.ghosted, order="F"), "densityBG": np.zeros(g.ghosted, order="F")}
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    o.set_density(f["r"])
    rng = np.random.default_rng(12)
    phi = np.asfortranarray(rng.standard_normal(g.ghosted))
    src = np.asfortranarray(rng.standard_normal(g.ghosted))
    o.debug_pass(1, phi, src)  # a ghosted initial guess
    ref = phi.copy(order="F")
    o.debug_pass(2, phi, src.copy(order="F"))
    vcycle(ref, src, g, levels, f["r"], pre, post)
    np.testing.assert_array_equal(phi, ref)
