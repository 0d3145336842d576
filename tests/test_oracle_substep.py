"""One RK sub-step of the oracle against the restated pieces (CPU only).

rk_ss (ANELASTIC_SL/dns/NSsolver.F90:418-583, the Crank-Nicolson branch)
is composed here from this suite's numpy restatements: the five explicit
right-hand sides, var_advance, the Crank-Nicolson z solves, Psource, a
dense direct solve of the pressure equation (the projection operator
Psource(Pgrad(.)), so no multigrid is involved) and Pgrad
(NSsolver.F90:2023-2085), with the restated boundary pass (ghost,
dns/BC.F90) between them, so no routine of the oracle is used.

The scalars do not see the pressure, so rho and scal1 must equal the
oracle's bit for bit.  The velocities agree to the pressure solve's
accuracy: the oracle's multigrid is solved to a relative residual of 1e-13,
so they are held to 1e-9 relative L2.  The case has a stretched z axis, an
anelastic r(z), random velocities, scalars and RK accumulators, and the
coefficients of the second RK3 sub-step, so every term contributes.

A whole step is composed the same way from the restated calcdt and three
restated sub-steps with the driver's coefficient table; a wrong table entry
fails it.
"""
import numpy as np

from anelastic_solve_b200 import abi, anelastic, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for, rel_l2
from .test_oracle_cn import cn_restated
from .test_oracle_direct import dense_operator, psource_pgrad, _wrap_xy
from .test_oracle_ghost import ghost as ghost_restated
from .test_oracle_projection import psource
from .test_oracle_rhs import _Shift, scalar_rhs, u1_rhs, u2_rhs, u3_rhs

RE, PR, SC, GRAV = 1000.0, 0.7, 2.0, -0.12
# second sub-step of the low-storage RK3 (a1, a2, a3 = a1 + a2 of rk_ss)
A1, A2 = -17.0 / 60.0, 5.0 / 12.0
DT = 0.02
VT = {"u": 0, "v": 1, "w": 2, "rho": 4, "scal1": 12, "q_u": 7, "q_v": 8, "q_w": 9, "q_rho": 10, "q_s": 11}




def restated_substep(n, g, nsp, a1, a2, a3, dt_rk, dt):
    """rk_ss on the state n (in place), from the restated pieces."""
    def gh(name, vt=None):
        ghost_restated(n[name], g, VT[name] if vt is None else vt, nsp.tb, nsp.vb, 1)

    h = _Shift(g)
    rRe = 1.0 / RE
    rhs = {"q_u": u1_rhs(n, h, rRe), "q_v": u2_rhs(n, h, rRe), "q_w": u3_rhs(n, h, rRe, GRAV, ew=1),
           "q_rho": scalar_rhs(n, h, "rho", rRe * (1.0 / PR), True),
           "q_s": scalar_rhs(n, h, "scal1", rRe * (1.0 / SC), False)}
    for q, F in rhs.items():  # var_advance(F, q, a1, a2, dt): q = a1 q + a2 F dt (interior)
        n[q][1:-1, 1:-1, 1:-1] = a1 * n[q][1:-1, 1:-1, 1:-1] + a2 * F * dt
        gh(q)

    def cn(q, name, var):
        n[name][1:-1, 1:-1, 1:-1] = cn_restated(g, nsp, n["r"], n[q], n[name], var, a3, dt_rk)
        gh(name)

    cn("q_u", "u", 1)
    cn("q_v", "v", 2)
    cn("q_w", "w", 3)
    src = psource(n, g) * (1.0 / dt_rk)
    cn("q_rho", "rho", 5)
    cn("q_s", "scal1", 8)
    # pressure: div(r grad(p/r)) = src, solved directly (null vector r)
    r = n["r"]

    def apply(p):
        a = p.copy(order="F")
        _wrap_xy(a)
        return psource_pgrad(a, g, r)

    A = dense_operator(apply, g)
    p_int = np.linalg.lstsq(A, src.reshape(-1, order="F"), rcond=None)[0]
    p = np.zeros(g.ghosted, order="F")
    p[1:-1, 1:-1, 1:-1] = p_int.reshape(g.shape, order="F")
    _wrap_xy(p)
    # Pgrad with dt_rk, each velocity ghosted after its update
    S, M = h.S, h.M
    n["u"][1:-1, 1:-1, 1:-1] = S(n["u"]) - (S(p, 1) / S(r) - S(p) / S(r)) * M(0, "rdxe") * dt_rk
    gh("u", VT["q_u"])
    n["v"][1:-1, 1:-1, 1:-1] = S(n["v"]) - (S(p, 0, 1) / S(r) - S(p) / S(r)) * M(1, "rdxe") * dt_rk
    gh("v", VT["q_v"])
    w = n["w"][1:-1, 1:-1, 1:-1]
    pw = S(p, 0, 0, 1)[:, :, :-1] / S(r, 0, 0, 1)[:, :, :-1] - S(p)[:, :, :-1] / S(r)[:, :, :-1]
    w[:, :, :-1] = w[:, :, :-1] - pw * M(2, "rdxe")[:, :, :-1] * dt_rk  # k = sz..ez-EW
    gh("w", VT["q_w"])
    for k in ("u", "v", "w", "rho", "scal1"):
        gh(k)


def _state(seed, **nskw):
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), maxcy=300, tolmax=1e-13, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=RE, Pr=PR, Sc=SC, g=GRAV, ew=1, scal1_on=1, **nskw)
    rng = np.random.default_rng(seed)
    f = shear.shear_layer_fields(g)
    for k in ("u", "v", "w", "rho", "scal1", "q_u", "q_v", "q_w", "q_rho", "q_s"):
        f[k][...] = 0.1 * rng.standard_normal(g.ghosted)
    anelastic.set_density_bg(f, g, x3center=-1000.0)
    o = OracleNS(g, mgp, nsp, f)
    for k in ("u", "v", "w", "rho", "scal1", "q_u", "q_v", "q_w", "q_rho", "q_s"):
        o.ghost(f[k], VT[k])
    return g, nsp, f, o


def test_substep_equals_restated_composition():
    g, nsp, f, o = _state(17)
    n = {k: v.copy(order="F") for k, v in f.items()}  # the restated state
    a3 = A1 + A2
    dt_rk = a3 * DT
    o.substep(A1, A2, a3, dt_rk, DT)
    restated_substep(n, g, nsp, A1, A2, a3, dt_rk, DT)
    for k in ("rho", "scal1"):
        np.testing.assert_array_equal(n[k][1:-1, 1:-1, 1:-1], f[k][1:-1, 1:-1, 1:-1], err_msg=k)
    for k in ("u", "v", "w"):
        assert 0.0 < rel_l2(n[k], f[k]) < 1e-9, (k, rel_l2(n[k], f[k]))


def test_step_equals_restated_composition():
    """A whole NSsolver step (NSsolver.F90:63-283, DNS): zero_temps, calcdt
    capped by dtmax, then rk_ss three times with the driver's coefficient
    table a1 = 0, -5/9, -153/128; a2 = 1; a3 = 1/3, 15/16, 8/15;
    dt_rk = delt/3, 5 delt/12, delt/4.  The time step is bit-exact; every
    field, the scalars included (they see the velocities of the earlier
    sub-steps), agrees to the pressure solves' 1e-9."""
    g, nsp, f, o = _state(23, cfl=0.5, dtmax=1e9)
    n = {k: v.copy(order="F") for k, v in f.items()}
    rep = o.step()
    for q in ("q_u", "q_v", "q_w", "q_rho", "q_s"):
        n[q][...] = 0.0
    h = _Shift(g)
    S, M = h.S, h.M
    adv = M(0, "rdxc") * np.abs(0.5 * (S(n["u"]) + S(n["u"], -1)))
    adv = adv + M(2, "rdxc") * np.abs(0.5 * (S(n["w"]) + S(n["w"], 0, 0, -1)))
    adv = adv + M(1, "rdxc") * np.abs(0.5 * (S(n["v"]) + S(n["v"], 0, -1)))
    delt = min(0.5 / adv.max(), 1e9)
    assert rep.dt == delt
    for a1, a3, frac in ((0.0, 1.0 / 3.0, 1.0 / 3.0), (-5.0 / 9.0, 15.0 / 16.0, 5.0 / 12.0),
                         (-153.0 / 128.0, 8.0 / 15.0, 1.0 / 4.0)):
        restated_substep(n, g, nsp, a1, 1.0, a3, frac * delt, delt)
    for k in ("u", "v", "w", "rho", "scal1"):
        assert rel_l2(n[k], f[k]) < 1e-9, (k, rel_l2(n[k], f[k]))
