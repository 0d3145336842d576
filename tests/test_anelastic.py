"""Anelastic background profiles (set_densityBG, IC.F90:1062-1096) and the
variable-density paths they drive: the multigrid operator with r(z)
(mgdpfpde / mgdphpde, including the literal mode's stale-index coarse
diagonal) and the RK3 step with r(z), densityBG(z) != 1.

The profiles are host inputs (no GPU arithmetic): their test checks the
single-precision literal semantics and the stratification.  On the GPU the
FP64 multigrid passes and capped solves, and the FP64 steps, must be
bit-identical to the oracle with the same profiles; the mixed-precision
step stays within the 1e-8 relative L2 field tolerance of the FP64 oracle.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, anelastic, shear
from anelastic_solve_b200 import grid as G

from .helpers import compatible, field, levels_for, mg_params, rel_l2


def column_grid():
    """A 8 km deep column: r falls by a factor ~2.3 over the domain."""
    return G.Grid(G.uniform_axis(32, 4000.0), G.uniform_axis(16, 2000.0), G.uniform_axis(32, 8000.0))


def test_profile_literals_and_stratification():
    assert anelastic.RD == float(np.float32(287.1)) != 287.1
    assert anelastic.KAPPA == float(np.float32(np.float32(287.1) / np.float32(1004.0)))
    p = anelastic.background_profiles(np.array([0.0, 100.0]))
    assert p["tz"][0] == 300.0
    assert p["tz"][1] == 300.0 - float(np.float32(0.0065)) * 100.0
    g = column_grid()
    q = anelastic.background_profiles(g.z.xc)
    assert np.all(np.diff(q["r"]) < 0)          # density falls with height
    assert np.all(np.diff(q["densityBG"]) > 0)  # potential temperature rises: stable
    assert 0.4 < q["r"][-1] < 0.6 and 1.1 < q["r"][0] < 1.25


def _density(g):
    f = {"r": np.zeros(g.ghosted, order="F"), "densityBG": np.zeros(g.ghosted, order="F")}
    anelastic.set_density_bg(f, g)
    return f["r"]


def _to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def _to_host(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
@pytest.mark.parametrize("which", [0, 2])
def test_mg_pass_with_density_bitwise(mode, which):
    from anelastic_solve_b200.mg import MGSolver
    from oracle.pyoracle import OracleMG

    g = column_grid()
    p = mg_params(g, mode=mode)
    o, s = OracleMG(g, p), MGSolver(g, p)
    r = _density(g)
    o.set_density(r)
    s.set_density(r)
    rng = np.random.default_rng(31 + which)
    phi, src = field(g, rng), field(g, rng)
    ref = phi.copy(order="F")
    o.debug_pass(which, ref, src.copy(order="F"))
    d = _to_dev(phi)
    s.debug_pass(which, d, _to_dev(src))
    np.testing.assert_array_equal(_to_host(d), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
def test_mg_solve_with_density_bitwise(mode):
    """Eight cycles (converged or not), iteration count and stop metric."""
    from anelastic_solve_b200.mg import MGSolver
    from oracle.pyoracle import OracleMG

    g = column_grid()
    p = mg_params(g, mode=mode, maxcy=8, tolmax=1e-12)
    o, s = OracleMG(g, p), MGSolver(g, p)
    r = _density(g)
    o.set_density(r)
    s.set_density(r)
    rng = np.random.default_rng(7)
    src = compatible(field(g, rng), g, mode)
    ref = np.zeros(g.ghosted, order="F")
    it_o, rm_o = o.solve(ref, src.copy(order="F"))
    d = _to_dev(np.zeros(g.ghosted, order="F"))
    it_g, rm_g = s.solve(d, _to_dev(src))
    assert it_g == it_o and rm_g == rm_o
    np.testing.assert_array_equal(_to_host(d), ref)


def _ns_case(precision):
    from oracle.pyoracle import OracleNS

    g_ = G.shear_layer_grid(32, 16, 32, stretched=True)
    lv = levels_for(g_)
    mgp = abi.make_mg_params(lv, maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC,
                             stop=abi.STOP_RESID)
    mgp_gpu = abi.make_mg_params(lv, maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                                 mode=abi.MODE_METRIC, stop=abi.STOP_RESID, precision=precision)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1)
    f = shear.shear_layer_fields(g_, amp=1e-3)
    # the column's profiles, shifted so the layer sits 1 km up
    anelastic.set_density_bg(f, g_, x3center=-1000.0)
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    return g_, mgp_gpu, nsp, f, o


@pytest.mark.gpu
def test_ns_steps_with_background_bitwise():
    from anelastic_solve_b200.ns import NSSolver

    g_, mgp, nsp, f, o = _ns_case(abi.PREC_FP64)
    assert f["r"].std() > 0 and f["densityBG"].std() > 0
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    for _ in range(3):
        ro, rg = o.step(), s.step(1)
        assert ro.dt == rg.dt and list(ro.mg_iter) == list(rg.mg_iter)
    got = s.get_fields(("u", "v", "w", "p", "rho", "scal1"))
    for k in got:
        np.testing.assert_array_equal(got[k], f[k], err_msg=k)


@pytest.mark.gpu
def test_ns_mixed_with_background_within_tolerance():
    from anelastic_solve_b200.ns import NSSolver

    g_, mgp, nsp, f, o = _ns_case(abi.PREC_MIXED)
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    for _ in range(3):
        o.step()
        s.step(1)
    got = s.get_fields(("u", "v", "w", "rho"))
    for k in got:
        assert rel_l2(got[k], f[k]) < 1e-8, k
