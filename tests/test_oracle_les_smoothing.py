"""The driver's periodic smoothing of the LES scalars (CPU only).

Every 50 steps, once the time is positive, the reference driver passes rho
and scal1 through filterHF(.., 2, 1, 1, 1, 'rho' / 'scal1', ..) when their
subgrid models are SSMrho/DSMrho and SSMscal1/DSMscal1
(ANELASTIC_SL/dns/NSsolver.F90:144-164), after the model coefficients and
before the sub-steps.  With the Smagorinsky models the coefficients do not
depend on the scalars, so a step at nstep = 50 from a state S equals a step
at nstep = 51 (no smoothing) from S with its scalars smoothed by the
restated filterHF and ghost pass.  The oracle must satisfy that bit for bit,
and must not smooth at other steps, at time 0, or without scalar models.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for
from .test_oracle_dsm import _Ctx, filter_hf

VT = {"u": 0, "v": 1, "w": 2, "rho": 4, "scal1": 12}
KEYS = ("u", "v", "w", "p", "rho", "scal1")


def _oracle(models, state):
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=50000.0, g=-0.1, ew=1, scal1_on=1, les=True, models=models,
                             stretched=(0, 0, 1), interp=abi.DIAG_CORRECTED)
    f = shear.shear_layer_fields(g, amp=1e-2)
    for k in ("nuT", "kappaT", "nappaT"):
        f[k] = np.zeros(g.ghosted, order="F")
    if state is None:
        rng = np.random.default_rng(50)
        f["rho"][...] += 0.05 * rng.standard_normal(g.ghosted)
        f["scal1"][...] = rng.standard_normal(g.ghosted)
    else:
        for k in KEYS:
            f[k][...] = state[k]
    o = OracleNS(g, mgp, nsp, f)
    if state is None:
        for k in ("u", "v", "w", "rho", "scal1"):
            o.ghost(f[k], VT[k])
        o.project()
    return g, nsp, f, o


def _smoothed(g, nsp, state):
    c = _Ctx(g, nsp, (1, 1, 1))
    out = {k: v.copy(order="F") for k, v in state.items()}
    for k in ("rho", "scal1"):
        out[k] = filter_hf(c, state[k], VT[k])
        c.ghost(out[k], VT[k])
    return out


SSM = (abi.MODEL_SSM,) * 3


def test_step_fifty_smooths_the_scalars():
    g, nsp, f0, o0 = _oracle(SSM, None)
    state = {k: f0[k].copy(order="F") for k in KEYS}
    _, _, fa, oa = _oracle(SSM, state)
    oa.set_clock(0.5, 50)
    oa.step()
    _, _, fb, ob = _oracle(SSM, _smoothed(g, nsp, state))
    ob.set_clock(0.5, 51)
    ob.step()
    for k in KEYS:
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)
    # and the smoothing did something: without it the fields differ
    _, _, fc, oc = _oracle(SSM, state)
    oc.set_clock(0.5, 51)
    oc.step()
    assert any(not np.array_equal(fa[k], fc[k]) for k in ("rho", "scal1"))


@pytest.mark.parametrize("case", ["time0", "step49", "dns_scalars"])
def test_no_smoothing_otherwise(case):
    models = (abi.MODEL_SSM, abi.MODEL_DNS, abi.MODEL_DNS) if case == "dns_scalars" else SSM
    time, nstep = (0.0, 50) if case == "time0" else (0.5, 49 if case == "step49" else 50)
    g, nsp, f0, o0 = _oracle(models, None)
    state = {k: f0[k].copy(order="F") for k in KEYS}
    _, _, fa, oa = _oracle(models, state)
    oa.set_clock(time, nstep)
    oa.step()
    _, _, fb, ob = _oracle(models, state)
    ob.set_clock(time, 51)
    ob.step()
    for k in KEYS:
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)
