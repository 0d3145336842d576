"""The oracle's optional clip (CPU only): clipVS (Routines.F90:301-380)
after every sub-step, then the field's ghost pass (NSsolver.F90:206-211).

One oracle step with Clip on from the shear-layer state: the interior of
rho stays in [rho_min, rho_max] and takes both bounds; its ghost cells are
the ghost pass of the clipped interior (a second ghost pass changes
nothing); and a range that contains every value leaves the step unchanged
bit for bit.
"""
import numpy as np

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleNS

from .helpers import levels_for


def _case(clip):
    g = G.shear_layer_grid(16, 8, 16, stretched=True)
    mgp = abi.make_mg_params(levels_for(g), maxcy=200, tolmax=1e-10, pre=2, post=2,
                             tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1, clip=clip)
    f = shear.shear_layer_fields(g, amp=1e-3)
    o = OracleNS(g, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    return o, f


def test_clip_bounds_and_ghosts():
    o, f = _case((-0.7, 0.6, -1.0, 1.0))
    o.step()
    rho = f["rho"]
    inner = rho[1:-1, 1:-1, 1:-1]
    assert inner.min() == -0.7 and inner.max() == 0.6
    again = rho.copy(order="F")
    o.ghost(again, 4)
    np.testing.assert_array_equal(again, rho)


def test_wide_clip_changes_nothing():
    o1, f1 = _case((-10.0, 10.0, -10.0, 10.0))
    o2, f2 = _case(None)
    o1.step()
    o2.step()
    for k in ("u", "v", "w", "p", "rho", "scal1"):
        np.testing.assert_array_equal(f1[k], f2[k], err_msg=k)
