"""Pin the CPU oracle with the reference's own known-answer cases.

The reference ships no golden outputs; its only known answers are the six
analytic problems of the pressure-solver test program ptest
(ANELASTIC_SL/mgMK/test/test.F90:149-382, exact solutions :471-564, wk = 1
from ANELASTIC_SL/include/modules.F90:259).  Quadratic and linear
solutions are reproduced exactly by the 7-point operator on a uniform grid,
so the oracle must reach them to solver tolerance; the sine cases are
second-order accurate and are checked by their convergence rate.
"""
import math

import numpy as np
import pytest

from anelastic_solve_b200 import abi
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleMG

from .helpers import levels_for, remove_mean

PI = 4.0 * math.atan(1.0)
# direction -> (min face, max face) indices into tbc/vbc
FACES = {"x1": (4, 5), "x2": (2, 0), "x3": (1, 3)}


def _grid(n=(16, 8, 32)):
    return G.Grid(G.uniform_axis(n[0], 1.0), G.uniform_axis(n[1], 1.0), G.uniform_axis(n[2], 2.0, -1.0))


def _axis(g, d):
    return {"x1": g.x, "x2": g.y, "x3": g.z}[d]


def _bcast(v, d, shape):
    sl = [None, None, None]
    sl[{"x1": 0, "x2": 1, "x3": 2}[d]] = slice(None)
    return np.broadcast_to(v[tuple(sl)], shape)


def _solve(g, tbc, vbc, phi0, src, tol=1e-13, maxcy=400):
    p = abi.make_mg_params(levels_for(g), maxcy=maxcy, tolmax=tol, pre=2, post=2, tbc=tbc, vbc=vbc)
    m = OracleMG(g, p)
    phi = np.asfortranarray(phi0.copy())
    it, rm = m.solve(phi, np.asfortranarray(src.copy()))
    return phi, it, rm


@pytest.mark.parametrize("d", ["x1", "x2", "x3"])
@pytest.mark.parametrize("case", ["dirichletBCs", "linearpgrad"])
def test_dirichlet_quadratic(case, d):
    """test.F90:150-227: del^2 p = a1 with p = 1 / 2 at the two ghost centres."""
    g = _grid()
    lo, hi = FACES[d]
    tbc = [0] * 6
    vbc = [0.0] * 6
    tbc[lo] = tbc[hi] = 2
    vbc[lo], vbc[hi] = 1.0, 2.0
    a1 = 2.0 if case == "dirichletBCs" else 0.0
    xc = _axis(g, d).xc
    b1 = (vbc[lo] - vbc[hi]) / (xc[0] - xc[-1]) - a1 / 2 * (xc[0] + xc[-1])
    c1 = (vbc[lo] + vbc[hi]) / 2.0 - a1 / 4.0 * (xc[0] ** 2 + xc[-1] ** 2) - b1 / 2.0 * (xc[0] + xc[-1])
    shape = g.ghosted
    phi, it, rm = _solve(g, tbc, vbc, np.full(shape, 0.5 * (vbc[lo] + vbc[hi])), np.full(shape, a1))
    exact = _bcast(a1 * xc ** 2 / 2.0 + b1 * xc + c1, d, shape)
    err = np.abs(phi - exact)[1:-1, 1:-1, 1:-1].mean()
    assert rm <= 1e-13 and it < 400
    assert err < 1e-10, err


@pytest.mark.parametrize("d", ["x1", "x2", "x3"])
def test_dirichlet_neumann(d):
    """test.F90:229-268: p = 1 at the min ghost centre, dp/dn = 0 at max."""
    g = _grid()
    lo, hi = FACES[d]
    tbc = [0] * 6
    vbc = [0.0] * 6
    tbc[lo], tbc[hi] = 2, 1
    vbc[lo], vbc[hi] = 1.0, 0.0
    a1 = 2.0
    xc = _axis(g, d).xc
    b1 = vbc[hi] - a1 * 0.5 * (xc[-1] + xc[-2])
    c1 = vbc[lo] - a1 * 0.5 * xc[0] ** 2 - b1 * xc[0]
    shape = g.ghosted
    phi, it, rm = _solve(g, tbc, vbc, np.full(shape, 0.5), np.full(shape, a1), maxcy=2000)
    exact = _bcast(a1 * xc ** 2 / 2.0 + b1 * xc + c1, d, shape)
    err = np.abs(phi - exact)[1:-1, 1:-1, 1:-1].mean()
    assert err < 1e-9, err


def test_cfdhw():
    """test.F90:347-380: Dirichlet in y (1, 0), Neumann in z, linear in y,
    started from a field of sines (test.F90:372-380)."""
    g = _grid((8, 16, 16))
    tbc = [2, 1, 2, 1, 0, 0]
    vbc = [0.0, 0.0, 1.0, 0.0, 0.0, 0.0]
    yc = g.y.xc
    zc = g.z.xc
    b1 = (vbc[2] - vbc[0]) / (yc[0] - yc[-1])
    c1 = (vbc[2] + vbc[0]) / 2.0 - b1 / 2.0 * (yc[0] + yc[-1])
    shape = g.ghosted
    phi0 = np.zeros(shape)
    # the reference loops l,m = 1..8 and keeps the last assignment (l = m = 8)
    phi0[:] = np.sin(2 * PI * 8 * yc[None, :, None] / g.y.L + 2 * PI * 8 * zc[None, None, :] / g.z.L)
    phi, it, rm = _solve(g, tbc, vbc, phi0, np.zeros(shape), maxcy=2000)
    exact = _bcast(b1 * yc + c1, "x2", shape)
    err = np.abs(phi - exact)[1:-1, 1:-1, 1:-1].mean()
    assert err < 1e-9, err


@pytest.mark.parametrize("d", ["x1", "x2", "x3"])
def test_1dsine_second_order(d):
    """test.F90:270-324: periodic, del^2 p = -(2 pi)^2 sin(2 pi x_e).  The
    discrete solution matches sin(2 pi x_e) (+ const) to O(h^2)."""
    errs = []
    for n in (16, 32):
        sizes = [8, 8, 8]
        sizes[{"x1": 0, "x2": 1, "x3": 2}[d]] = n
        g = G.Grid(G.uniform_axis(sizes[0], 1.0), G.uniform_axis(sizes[1], 1.0),
                   G.uniform_axis(sizes[2], 1.0))
        xe = _axis(g, d).xe
        c = 2.0 * PI
        shape = g.ghosted
        src = _bcast(-(c ** 2) * np.sin(c * xe), d, shape)
        phi, it, rm = _solve(g, [0] * 6, [0.0] * 6, np.zeros(shape), src, tol=1e-12, maxcy=500)
        exact = _bcast(np.sin(c * xe), d, shape)
        e = remove_mean(np.asfortranarray(phi - exact))
        errs.append(np.abs(e[1:-1, 1:-1, 1:-1]).mean())
    rate = math.log2(errs[0] / errs[1])
    assert 1.8 < rate < 2.2, (errs, rate)


def test_levels_table_reference_runfile():
    """Level maps of the reference runfile's solver block (Sturb.ini:125-135:
    nxlevels=4, nylevels=3, nzlevels=8 on 256 x 64 x 256) follow
    mg_init.F90:125-220: x and y stop coarsening below their own level
    counts and offsets are packed finest first."""
    g = G.Grid(G.uniform_axis(256, 1.0), G.uniform_axis(64, 1.0), G.uniform_axis(256, 1.0))
    p = abi.make_mg_params((4, 3, 8), pre=[14, 10, 4, 4, 2, 2, 2, 2], post=[12, 10, 4, 4, 2, 2, 2, 2],
                           tbc=(0, 1, 0, 1, 0, 0))
    t = OracleMG(g, p).levels()
    assert t.shape == (8, 12)
    nxk = t[:, 0]
    nyk = t[:, 1]
    nzk = t[:, 2]
    assert list(nxk) == [33, 33, 33, 33, 33, 65, 129, 257]
    assert list(nyk) == [17, 17, 17, 17, 17, 17, 33, 65]
    assert list(nzk) == [3, 5, 9, 17, 33, 65, 129, 257]
    # ex = (ex_f - 1)/2 + 1 when coarsened, else unchanged
    assert list(t[:, 4]) == [33, 33, 33, 33, 33, 65, 129, 257]
    assert list(t[:, 8]) == [3, 5, 9, 17, 33, 65, 129, 257]
    # workspace offsets: finest at 1, each next one after the previous level
    assert t[-1, 9] == 1
    G8 = (257 + 1) * (65 + 1) * (257 + 1)
    assert t[-2, 9] == 1 + G8


def test_zline_semicoarsening_converges_faster():
    """The ZLINE extension (z-line smoothing with horizontal
    semi-coarsening) needs far fewer V-cycles than RBPGS with full
    coarsening on the tanh-stretched shear-layer grid."""
    from .helpers import compatible, field, zeros

    g = G.shear_layer_grid(64, 32, 64, stretched=True)
    rng = np.random.default_rng(3)
    src = compatible(field(g, rng), g, abi.MODE_METRIC)
    its = {}
    for sm, lv in ((abi.SMOOTHER_RBPGS, (6, 5, 6)), (abi.SMOOTHER_ZLINE, (6, 5, 1))):
        p = abi.make_mg_params(lv, maxcy=300, tolmax=1e-10, pre=2, post=2, tbc=(0, 1, 0, 1, 0, 0),
                               mode=abi.MODE_METRIC, smoother=sm, stop=abi.STOP_RESID)
        phi = zeros(g)
        its[sm], _ = OracleMG(g, p).solve(phi, src.copy(order="F"))
    assert its[abi.SMOOTHER_ZLINE] * 3 <= its[abi.SMOOTHER_RBPGS], its
