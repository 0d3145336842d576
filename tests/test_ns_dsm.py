"""Dynamic Smagorinsky models: DSM (les/DSM.F90), DSMrho and DSMscal1
(les/DSMrho.F90, DSMscal1.F90), with the test filter and filterHF of
les/filter.F90 and the reference's x-y plane averaging of the coefficients.

Every per-cell expression equals the oracle's; the plane averages are a
parallel fixed-order sum on the GPU and a running sum in the oracle, so the
eddy viscosity and diffusivities after a step agree within 1e-9 relative to
their largest magnitude, and the fields after two steps within the
1e-8 relative L2.  Cases: the reference runfile's setup (Vel/Rho/Scal1 =
DSM/DSMrho/DSMscal1, TestGrid_ratio = sqrt(6), filters in x, y and z,
uniform grids; run_dir/Sturb.ini:8-18, 89-91), and a tanh-stretched z axis
with the corrected centring interpolation, the dynamic velocity model and
the Smagorinsky scalar models (SSMrho / SSMscal1 from the dynamic Csgs).
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G

from .helpers import levels_for, rel_l2

pytestmark = pytest.mark.gpu

EDDY = ("nuT", "kappaT", "nappaT")
CMP = ("u", "v", "w", "rho", "scal1")


def _case(stretched, models, interp):
    from oracle.pyoracle import OracleNS

    g_ = G.shear_layer_grid(32, 16, 32, stretched=stretched)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=50000.0, Pr=1.0, g=-0.1, dtmax=0.005, ew=1, scal1_on=1, les=True,
                             models=models, stretched=(0, 0, 1 if stretched else 0), interp=interp)
    f = shear.shear_layer_fields(g_, amp=1e-2)
    f["scal1"][...] = 0.5 * f["rho"]
    for k in EDDY:
        f[k] = np.zeros(g_.ghosted, order="F")
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    return g_, mgp, nsp, f, o


@pytest.mark.parametrize("setup", ["runfile", "stretched"])
def test_dynamic_models_match_oracle(setup):
    from anelastic_solve_b200.ns import NSSolver

    if setup == "runfile":
        g_, mgp, nsp, f, o = _case(False, (abi.MODEL_DSM,) * 3, abi.DIAG_LITERAL)
    else:
        g_, mgp, nsp, f, o = _case(True, (abi.MODEL_DSM, abi.MODEL_SSM, abi.MODEL_SSM), abi.DIAG_CORRECTED)
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    o.step()
    s.step(1)
    got = s.get_fields(EDDY)
    for k in EDDY:
        ref = f[k][1:-1, 1:-1, 1:-1]
        scale = np.abs(ref).max()
        assert scale > 0, k
        np.testing.assert_allclose(got[k][1:-1, 1:-1, 1:-1], ref, rtol=1e-9, atol=1e-9 * scale, err_msg=k)
    o.step()
    s.step(1)
    got = s.get_fields(CMP)
    for k in CMP:
        assert rel_l2(got[k], f[k]) < 1e-8, k
