"""Cohort stepping (anel_ns_ctx_step_cohort) on the GPU.

Members of one grid and multigrid setup, each with its own physics (Re,
Ri), time step and state, step together on one stream; each sub-step's
pressure solves are one batched multigrid solve.  A member's fields, time
step, divergence and cycle counts must equal those of the same member
stepped alone, bit for bit.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200.mg import MGSolver
from anelastic_solve_b200.ns import NSSolver

from .helpers import levels_for

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "rho")
MEMBERS = [(1000.0, 0.12, 7), (2500.0, 0.05, 8), (600.0, 0.3, 9)]  # (Re, Ri, seed)


def _params(g, Re, Ri):
    lv = levels_for(g)
    mg = abi.make_mg_params((lv[0], lv[1], 1), maxcy=200, tolmax=1e-10, pre=2, post=2,
                            tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC, stop=abi.STOP_RESID,
                            precision=abi.PREC_MIXED, smoother=abi.SMOOTHER_ZLINE)
    ns = abi.make_ns_params(Re=Re, Pr=1.0, g=-Ri, cfl=0.5, dtmax=1e9, ew=1, scal1_on=0)
    return mg, ns


def _member(g, Re, Ri, seed):
    mg, ns = _params(g, Re, Ri)
    f = shear.shear_layer_fields(g, amp=1e-2, seed=seed)
    s = NSSolver(g, mg, ns)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    s.project()
    return s


@pytest.mark.parametrize("own_batch", [False, True])
def test_cohort_equals_members_alone(own_batch):
    """Three members of 64x32x128 (column cycle), three steps: cohort ==
    alone for u, v, w, p, rho, dt, max|div| and every sub-step's cycle
    count; with the first member's multigrid context as the batch solver
    and with a separate one."""
    g = G.shear_layer_grid(64, 32, 128, stretched=True)
    alone = []
    for Re, Ri, seed in MEMBERS:
        s = _member(g, Re, Ri, seed)
        rep = s.step(3)
        alone.append((s.get_fields(FIELDS), rep.dt, rep.max_div, list(rep.mg_iter)))
        s.close()
    ms = [_member(g, Re, Ri, seed) for Re, Ri, seed in MEMBERS]
    batch = MGSolver(g, _params(g, *MEMBERS[0][:2])[0]) if own_batch else None
    reps = NSSolver.step_cohort(ms, 3, batch=batch)
    for b, (s, rep) in enumerate(zip(ms, reps)):
        f, dt, mdiv, it = alone[b]
        got = s.get_fields(FIELDS)
        print(f"\nmember {b}: dt {rep.dt:.6e} (alone {dt:.6e}), cycles {list(rep.mg_iter)} (alone {it})")
        for k in FIELDS:
            np.testing.assert_array_equal(got[k], f[k], err_msg=f"member {b} {k}")
        assert rep.dt == dt and rep.max_div == mdiv and list(rep.mg_iter) == it
        s.close()
    if batch is not None:
        batch.close()
    assert len({a[1] for a in alone}) == len(alone)  # the members' time steps differ


def test_cohort_refuses_mixed_grids():
    g1 = G.shear_layer_grid(64, 32, 128, stretched=True)
    g2 = G.shear_layer_grid(32, 32, 128, stretched=True)
    a, b = _member(g1, 1000.0, 0.1, 1), _member(g2, 1000.0, 0.1, 2)
    with pytest.raises(Exception):
        NSSolver.step_cohort([a, b], 1)
    a.close()
    b.close()
