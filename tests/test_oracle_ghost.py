"""The oracle's boundary pass, restated from the reference (CPU only).

ghost() and bound_update() (ANELASTIC_SL/dns/BC.F90:1-187, 334-585) in
their serial form: the full periodic wrap of all six ghost planes, then per
direction and face the boundary code TB(dir, face, l) of the variable's
column l, with the variable's staggering (metric arrays and offsets of1,
of2), the two-point Neumann rows of the scalars (rtype 1), w's edge node
(EW) and its extra point.  The restatement is numpy on whole planes, in the
Fortran order of the assignments.  For every variable type and a set of
boundary-code configurations with non-zero wall values (periodic, Dirichlet,
Neumann, codes 4, 6, 7, 8), the oracle's ghost cells and interior must equal
it bit for bit.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for

# vt -> (name, column l, rtype, staggering) as ghost() selects them
VTYPES = {0: ("u", 1, 0, "u"), 1: ("v", 2, 0, "v"), 2: ("w", 3, 0, "w"), 3: ("p", 4, 0, "c"),
          4: ("rho", 5, 1, "c"), 5: ("cfluc", 6, 0, "c"), 6: ("psource", 7, 0, "c"),
          7: ("utemp", 7, 0, "u"), 8: ("vtemp", 7, 0, "v"), 9: ("wtemp", 7, 0, "w"),
          10: ("rtemp", 7, 0, "c"), 11: ("s1temp", 7, 0, "c"), 12: ("scal1", 8, 1, "c"),
          13: ("scal1temp", 8, 0, "c")}


def _metrics(g, stag):
    """(dxt, dyt, dzt, of1, of2) of bound_update's select on vtype."""
    x, y, z = g.x, g.y, g.z
    if stag == "u":
        return x.dxc, y.dxe, z.dxe, 0, 1
    if stag == "v":
        return x.dxe, y.dxc, z.dxe, 0, 1
    if stag == "w":
        return x.dxe, y.dxe, z.dxc, 0, 1
    return x.dxe, y.dxe, z.dxe, -1, 0


def bound_update(a, g, btype, face, d, value, stag, rt, ew):
    """One call of bound_update on the ghosted array a (0-based index =
    Fortran index - 1); sx = 2, ex = n+1 in Fortran terms."""
    dt_ = _metrics(g, stag)
    dm, of1, of2 = dt_[d - 1], dt_[3], dt_[4]
    n = g.shape[d - 1]
    s_, e_ = 2, n + 1
    iE = ew if (d == 3 and stag == "w") else 0

    def P(k):  # the plane at Fortran index k along d
        sl = [slice(None)] * 3
        sl[d - 1] = k - 1
        return tuple(sl)

    M = lambda k: dm[k - 1]
    if btype == 1:
        if face == 1:
            a[P(s_ - 1)] = value
        else:
            a[P(e_ + 1 - iE)] = value
    elif btype == 2:
        if face == 1:
            if rt == 1:
                a[P(s_)] = a[P(s_ + 1)] - value * M(s_ + 1 + of1)
            a[P(s_ - 1)] = a[P(s_)] - value * M(s_ + of1)
        else:
            if rt == 1:
                a[P(e_ - iE)] = a[P(e_ - 1 - iE)] + value * M(e_ - 1 + of2 - iE)
            a[P(e_ + 1 - iE)] = a[P(e_ - iE)] + value * M(e_ + of2 - iE)
    elif btype == 3:
        a[P(s_ - 1)] = a[P(e_ - iE)]
        a[P(e_ + 1 - iE)] = a[P(s_)]
    elif btype == 4:
        if face == 1:
            a[P(s_ - 1)] = a[P(s_)] - value * M(s_ + of1)
        else:
            a[P(e_ + 1 - iE)] = a[P(e_ - iE)] + value * M(e_ + of2 - iE)
    elif btype == 8 and d == 1:
        if face == 1:
            a[P(s_ - 1)] = 2.0 * a[P(s_)] - a[P(s_ + 1)]
        else:
            a[P(e_ + 1)] = 2.0 * a[P(e_)] - a[P(e_ - 1)]
    elif btype == 6 and d == 3:
        if face == 1:
            a[P(s_ - 1)] = 2.0 * value - 1.0 * a[P(s_)]
        else:
            a[P(e_ + 1 - iE)] = 2.0 * value - 1.0 * a[P(e_ - iE)]
    elif btype == 7 and d == 3:
        if face == 1:
            a[P(s_)] = 0.0
            a[P(s_ - 1)] = -1.0 * a[P(s_ + 1)]
        else:
            a[P(e_)] = 0.0
            a[P(e_ + 1 - iE)] = -1.0 * a[P(e_ - iE - 1)]
    if d == 3 and face == 2 and iE == 1:
        a[P(e_ + 1)] = 0.0  # the extra point


def ghost(a, g, vt, tb, vb, ew):
    _, l, rt, stag = VTYPES[vt]
    a[0, :, :] = a[-2, :, :]
    a[-1, :, :] = a[1, :, :]
    a[:, 0, :] = a[:, -2, :]
    a[:, -1, :] = a[:, 1, :]
    a[:, :, 0] = a[:, :, -2]
    a[:, :, -1] = a[:, :, 1]
    for d in (1, 2, 3):
        for m in (1, 2):
            if tb[d - 1][0][l - 1] != 3 or m == 1:
                bound_update(a, g, tb[d - 1][m - 1][l - 1], m, d, vb[d - 1][m - 1][l - 1], stag, rt, ew)


# (x codes, y codes, z min codes, z max codes) per variable column l = 1..8
CONFIGS = {
    "shear_layer": None,  # the stepping configuration (make_ns_params)
    "walls_everywhere": ((2, 1), (4, 2), (1, 2, 2, 4, 2, 6, 1, 2), (2, 7, 1, 2, 2, 6, 4, 2)),
    "x_extrapolated": ((8, 8), (3, 3), (6, 2, 7, 4, 2, 1, 2, 2), (1, 4, 6, 2, 7, 2, 2, 1)),
}


def _params(config, ew):
    nsp = abi.make_ns_params(ew=ew, scal1_on=1)
    if CONFIGS[config] is None:
        return nsp
    xs, ys, zmin, zmax = CONFIGS[config]
    rng = np.random.default_rng(len(config))
    for l in range(8):
        for m in range(2):
            nsp.tb[0][m][l] = xs[m]
            nsp.tb[1][m][l] = ys[m]
        nsp.tb[2][0][l] = zmin[l]
        nsp.tb[2][1][l] = zmax[l]
        for d in range(3):
            for m in range(2):
                nsp.vb[d][m][l] = float(rng.standard_normal())
    return nsp


@pytest.mark.parametrize("config", list(CONFIGS))
@pytest.mark.parametrize("ew", [1, 0])
def test_ghost_equals_restatement(config, ew):
    g = G.shear_layer_grid(8, 6, 10, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC)
    nsp = _params(config, ew)
    o = OracleNS(g, mgp, nsp, shear.shear_layer_fields(g))
    rng = np.random.default_rng(ew + 10)
    for vt in VTYPES:
        a = np.asfortranarray(rng.standard_normal(g.ghosted))
        b = a.copy(order="F")
        o.ghost(a, vt)
        ghost(b, g, vt, nsp.tb, nsp.vb, ew)
        np.testing.assert_array_equal(a, b, err_msg=f"{config} {VTYPES[vt][0]}")
