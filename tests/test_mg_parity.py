"""GPU multigrid vs the CPU oracle, through the C-ABI.

The FP64 path must be bit-identical to the oracle (the reference's
algorithm evaluated in its own order): boundary pass, one red-black
iteration, one V-cycle, and whole solves including iteration count and the
reference stop metric.  The mixed-precision path must reach the FP64
oracle's solution within 1e-9 relative L2 (after removing the mean, the
problem being singular) with a true relative residual <= 1e-10.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200.mg import MGSolver
from oracle.pyoracle import OracleMG

from .helpers import compatible, field, levels_for, mg_params, rel_l2, remove_mean, zeros

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def to_host(t):
    return np.asfortranarray(t.cpu().numpy().T)


CASES = {
    # name: (grid, tbc, vbc, levels)
    "shear_uniform": (lambda: G.shear_layer_grid(16, 8, 16, stretched=False), (0, 1, 0, 1, 0, 0),
                      (0, 0, 0, 0, 0, 0), None),
    "shear_stretched_vbc": (lambda: G.shear_layer_grid(32, 16, 32, stretched=True),
                            (0, 1, 0, 1, 0, 0), (0, 0.25, 0, -0.5, 0, 0), None),
    "walls_everywhere": (lambda: G.Grid(G.uniform_axis(16, 1.0), G.uniform_axis(12, 0.75),
                                        G.uniform_axis(8, 0.5)),
                         (1, 2, 2, 1, 1, 2), (0.3, 1.0, -1.0, 0.2, -0.4, 0.5), None),
    "partial_coarsening": (lambda: G.shear_layer_grid(16, 8, 32, stretched=False), (0, 1, 0, 1, 0, 0),
                           (0, 0, 0, 0, 0, 0), (3, 2, 5)),
    "odd_coarse": (lambda: G.Grid(G.uniform_axis(12, 1.0), G.uniform_axis(6, 0.5),
                                  G.uniform_axis(12, 1.0)), (0, 1, 0, 1, 0, 0), (0, 0, 0, 0, 0, 0),
                   (3, 2, 3)),
}


def _pair(name, mode=abi.MODE_LITERAL, **kw):
    mk, tbc, vbc, lv = CASES[name]
    g = mk()
    p = mg_params(g, levels=lv or levels_for(g), tbc=tbc, vbc=vbc, mode=mode, **kw)
    return g, p, OracleMG(g, p), MGSolver(g, p)


@pytest.mark.parametrize("name", list(CASES))
def test_level_tables_match(name):
    g, p, o, s = _pair(name)
    np.testing.assert_array_equal(o.levels(), s.levels())


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("which", [1, 0, 2])
def test_single_pass_bitwise(name, mode, which):
    """which: 1 = mg_bdry, 0 = one RB-GS iteration, 2 = one V-cycle."""
    g, p, o, s = _pair(name, mode)
    rng = np.random.default_rng(11 + which)
    phi = field(g, rng)
    src = field(g, rng)
    ref = phi.copy(order="F")
    o.debug_pass(which, ref, src.copy(order="F"))
    dphi, dsrc = to_dev(phi), to_dev(src)
    s.debug_pass(which, dphi, dsrc)
    got = to_host(dphi)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
@pytest.mark.parametrize("name", list(CASES))
def test_solve_bitwise(name, mode):
    g, p, o, s = _pair(name, mode, maxcy=60, tolmax=1e-9)
    rng = np.random.default_rng(5)
    src = compatible(field(g, rng), g, mode)
    phi0 = field(g, rng, 0.1)
    ref = phi0.copy(order="F")
    it_o, rm_o = o.solve(ref, src.copy(order="F"))
    dphi, dsrc = to_dev(phi0), to_dev(src)
    it_g, rm_g = s.solve(dphi, dsrc)
    assert it_g == it_o
    assert rm_g == rm_o
    np.testing.assert_array_equal(to_host(dphi), ref)
    # the right-hand side is read only on the device path
    np.testing.assert_array_equal(to_host(dsrc), src)


def test_host_path_equals_device_path():
    g, p, o, s = _pair("shear_stretched_vbc", maxcy=40, tolmax=1e-10)
    rng = np.random.default_rng(3)
    src = remove_mean(field(g, rng))
    phi_h = zeros(g)
    it_h, rm_h = s.solve(phi_h, src.copy(order="F"))
    dphi, dsrc = to_dev(zeros(g)), to_dev(src)
    it_d, rm_d = s.solve(dphi, dsrc)
    assert (it_h, rm_h) == (it_d, rm_d)
    np.testing.assert_array_equal(phi_h, to_host(dphi))


def test_nonconvergence_reports_like_reference():
    """maxcy reached: the Fortran DO variable ends at maxcy+1
    (mg_solver.F90:114-133) and the status is ANEL_ERR_NOCONV."""
    g, p, o, s = _pair("shear_uniform", maxcy=1, tolmax=1e-30)
    rng = np.random.default_rng(9)
    src = remove_mean(field(g, rng))
    ref = zeros(g)
    it_o, rm_o = o.solve(ref, src.copy(order="F"))
    dphi = to_dev(zeros(g))
    it_g, rm_g = s.solve(dphi, to_dev(src))
    assert it_o == it_g == 2
    assert rm_g == rm_o
    assert s.last_report.status == abi.ERR_NOCONV
    with pytest.raises(Exception):
        s.solve(to_dev(zeros(g)), to_dev(src), allow_noconv=False)


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
def test_mixed_precision_reaches_fp64_solution(mode):
    g = G.shear_layer_grid(32, 16, 32, stretched=True)
    lv = levels_for(g)
    rng = np.random.default_rng(21)
    src = compatible(field(g, rng), g, mode)
    # FP64 oracle solved to the true-residual target
    po = mg_params(g, levels=lv, mode=mode, maxcy=400, tolmax=1e-14)
    o = OracleMG(g, po)
    ref = zeros(g)
    o.solve(ref, src.copy(order="F"))
    assert o.true_resid(ref, src) < 1e-10
    # (a) residual target 1e-10: FP64-oracle residual accuracy; the
    #     solution error is then bounded by cond(A) * 1e-10, not by 1e-10
    pm = mg_params(g, levels=lv, mode=mode, maxcy=100, tolmax=1e-10,
                   precision=abi.PREC_MIXED, stop=abi.STOP_RESID)
    s = MGSolver(g, pm)
    dphi = to_dev(zeros(g))
    s.solve(dphi, to_dev(src))
    got = to_host(dphi)
    assert s.last_report.status == abi.OK
    assert s.last_report.resid <= 1e-10
    assert o.true_resid(got, src) <= 1.01e-10
    assert rel_l2(remove_mean(got), remove_mean(ref)) < 1e-7
    # (b) residual target 1e-12: pressure within 1e-9 relative L2 of the
    #     FP64 oracle (the FP64 outer loop carries the accuracy, the FP32
    #     inner cycle only has to contract)
    pm.tolmax = 1e-12
    s2 = MGSolver(g, pm)
    dphi = to_dev(zeros(g))
    s2.solve(dphi, to_dev(src))
    got = to_host(dphi)
    assert s2.last_report.status == abi.OK
    assert rel_l2(remove_mean(got), remove_mean(ref)) < 1e-9


# ----------------------------------------------------------------- ZLINE
ZCASES = {
    # horizontal semi-coarsening (no z levels) and full coarsening
    "zline_semi": (lambda: G.shear_layer_grid(32, 16, 32, stretched=True), (5, 4, 1)),
    "zline_full": (lambda: G.shear_layer_grid(32, 16, 32, stretched=True), (5, 4, 5)),
    "zline_odd": (lambda: G.Grid(G.uniform_axis(12, 1.0), G.uniform_axis(6, 0.5),
                                 G.tanh_axis(24)), (3, 2, 1)),
}


def _zpair(name, **kw):
    mk, lv = ZCASES[name]
    g = mk()
    p = mg_params(g, levels=lv, tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC,
                  smoother=abi.SMOOTHER_ZLINE, **kw)
    return g, p, OracleMG(g, p), MGSolver(g, p)


@pytest.mark.parametrize("name", list(ZCASES))
@pytest.mark.parametrize("which", [0, 2])
def test_zline_pass_bitwise(name, which):
    g, p, o, s = _zpair(name)
    rng = np.random.default_rng(31 + which)
    phi = field(g, rng)
    src = field(g, rng)
    ref = phi.copy(order="F")
    o.debug_pass(which, ref, src.copy(order="F"))
    dphi = to_dev(phi)
    s.debug_pass(which, dphi, to_dev(src))
    np.testing.assert_array_equal(to_host(dphi), ref)


@pytest.mark.parametrize("name", list(ZCASES))
@pytest.mark.parametrize("stop", [abi.STOP_RELMAX, abi.STOP_RESID])
def test_zline_solve_bitwise(name, stop):
    g, p, o, s = _zpair(name, maxcy=40, tolmax=1e-10, stop=stop)
    rng = np.random.default_rng(8)
    src = compatible(field(g, rng), g, abi.MODE_METRIC)
    ref = zeros(g)
    it_o, rm_o = o.solve(ref, src.copy(order="F"))
    dphi = to_dev(zeros(g))
    it_g, rm_g = s.solve(dphi, to_dev(src))
    assert it_o == it_g
    if stop == abi.STOP_RELMAX:
        assert rm_o == rm_g
    np.testing.assert_array_equal(to_host(dphi), ref)


# Mixed-precision ZLINE solves.  A level with at most 512 lines of a colour
# is swept by cyclic reduction (one CTA per line), a larger one by the
# partitioned solver: 32x16x32 has 256 lines on its finest level (cyclic
# reduction on every level); 64x32x64 and 64x32x256 have 1024 there
# (partitioned on the finest level, segments of 4 and 16 rows; cyclic
# reduction below).
ZMIX = {
    "cr_32x16x32": ((32, 16, 32), (5, 4, 1), 24),
    "seg_64x32x64": ((64, 32, 64), (6, 5, 1), 30),
    "seg_64x32x256": ((64, 32, 256), (6, 5, 1), 30),
}


@pytest.mark.parametrize("name", list(ZMIX))
def test_zline_mixed_precision(name):
    (nx, ny, nz), lv, max_it = ZMIX[name]
    g = G.shear_layer_grid(nx, ny, nz, stretched=True)
    rng = np.random.default_rng(22)
    src = compatible(field(g, rng), g, abi.MODE_METRIC)
    po = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE,
                   maxcy=100, tolmax=1e-13, stop=abi.STOP_RESID)
    ref = zeros(g)
    OracleMG(g, po).solve(ref, src.copy(order="F"))
    pm = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE,
                   maxcy=60, tolmax=1e-12, stop=abi.STOP_RESID, precision=abi.PREC_MIXED)
    s = MGSolver(g, pm)
    dphi = to_dev(zeros(g))
    s.solve(dphi, to_dev(src))
    assert s.last_report.status == abi.OK and s.last_report.resid <= 1e-12
    assert s.last_report.iter <= max_it
    assert rel_l2(remove_mean(to_host(dphi)), remove_mean(ref)) < 1e-9


# ------------------------------------------------------------------- LJ
# The reference's own z-line smoother (mg_relaxLz with its pcf line
# coefficients, mg_relax.F90:423-595): FP64 bit-identical to the oracle.
LJ_CASES = ["shear_uniform", "shear_stretched_vbc", "partial_coarsening"]


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
@pytest.mark.parametrize("name", LJ_CASES)
@pytest.mark.parametrize("which", [0, 2])
def test_lj_pass_bitwise(name, mode, which):
    g, p, o, s = _pair(name, mode, smoother=abi.SMOOTHER_LJ)
    rng = np.random.default_rng(41 + which)
    phi = field(g, rng)
    src = field(g, rng)
    ref = phi.copy(order="F")
    o.debug_pass(which, ref, src.copy(order="F"))
    dphi = to_dev(phi)
    s.debug_pass(which, dphi, to_dev(src))
    np.testing.assert_array_equal(to_host(dphi), ref)


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
@pytest.mark.parametrize("name", LJ_CASES)
def test_lj_solve_bitwise(name, mode):
    g, p, o, s = _pair(name, mode, smoother=abi.SMOOTHER_LJ, maxcy=40, tolmax=1e-9)
    rng = np.random.default_rng(6)
    src = compatible(field(g, rng), g, mode)
    ref = zeros(g)
    it_o, rm_o = o.solve(ref, src.copy(order="F"))
    dphi = to_dev(zeros(g))
    it_g, rm_g = s.solve(dphi, to_dev(src))
    assert (it_g, rm_g) == (it_o, rm_o)
    np.testing.assert_array_equal(to_host(dphi), ref)


@pytest.mark.parametrize("mode", [abi.MODE_LITERAL, abi.MODE_METRIC])
def test_dropin_mg_solve_equals_oracle(mode):
    """The drop-in anel_mg_init / anel_mg_solve / anel_mg_finalize (host
    arrays by reference, the argument list of mg_solver(phif, rhsf, iter,
    relmax), mgMK/mg_solver.F90:48-141) against the oracle's mg_solver:
    the same solution bit for bit, the same iteration count and relmax,
    on two solves in a row (the second from the first's solution)."""
    import ctypes as C

    from anelastic_solve_b200 import _lib

    name = "shear_stretched_vbc"
    mk, tbc, vbc, lv = CASES[name]
    g = mk()
    p = mg_params(g, levels=levels_for(g), tbc=tbc, vbc=vbc, mode=mode, maxcy=40, tolmax=1e-9)
    o = OracleMG(g, p)
    L = _lib.lib()
    desc, keep = abi.make_grid_desc(g)
    _lib.check(L.anel_mg_init(C.byref(desc), C.byref(p)))
    try:
        rng = np.random.default_rng(61)
        ref = zeros(g)
        phi = zeros(g)
        for _ in range(2):
            src = compatible(field(g, rng), g, mode)
            it_o, rm_o = o.solve(ref, src.copy(order="F"))
            it = C.c_int32(-7)
            rm = C.c_double(-7.0)
            L.anel_mg_solve(abi.dptr(phi), abi.dptr(src.copy(order="F")), C.byref(it), C.byref(rm))
            assert it.value > 0, _lib.last_error()
            assert (it.value, rm.value) == (it_o, rm_o)
            np.testing.assert_array_equal(phi, ref)
    finally:
        L.anel_mg_finalize()


def test_direct_coarse_solve_matches_oracle():
    """The FP64 direct solve the z-line cycle uses on its coarse level
    (real Fourier modes in the periodic x and y, one tridiagonal z-system
    per mode, the constant mode's gauge pinned), applied to a whole fine
    level (debug pass 3): the same solution as the oracle's FP64 multigrid
    solve to 1e-13, modulo the constant, and a true residual at FP64
    rounding level."""
    g = G.shear_layer_grid(32, 16, 128, stretched=True)
    lv = (5, 4, 1)
    rng = np.random.default_rng(71)
    src = compatible(field(g, rng), g, abi.MODE_METRIC)
    po = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, maxcy=200,
                   tolmax=1e-13, stop=abi.STOP_RESID)
    ref = zeros(g)
    o = OracleMG(g, po)
    it_o, _ = o.solve(ref, src.copy(order="F"))
    assert it_o <= 200
    pm = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, precision=abi.PREC_MIXED)
    s = MGSolver(g, pm)
    dphi = to_dev(zeros(g))
    s.debug_pass(3, dphi, to_dev(src))
    got = to_host(dphi)
    from .helpers import remove_vmean

    assert rel_l2(remove_vmean(got, g), remove_vmean(ref, g)) < 1e-10
    assert o.true_resid(got, src) < 1e-12


@pytest.mark.parametrize("n", [(64, 32, 256), (32, 16, 512)])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_column_sweep_variants(variant, n, monkeypatch):
    """Every launch variant of the column-layout z-line sweep (the
    autotuner's candidates, forced here through ANEL_COL_VARIANT; 3 is the
    bulk-copy staged kernel, 4 the one with its factors in registers): the mixed ZLINE solve reaches the oracle's
    FP64 solution within 1e-9."""
    monkeypatch.setenv("ANEL_COL_VARIANT", str(variant))
    g = G.shear_layer_grid(*n, stretched=True)
    lv = levels_for(g)[:2] + (1,)
    rng = np.random.default_rng(23)
    src = compatible(field(g, rng), g, abi.MODE_METRIC)
    po = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, maxcy=100,
                   tolmax=1e-13, stop=abi.STOP_RESID)
    ref = zeros(g)
    OracleMG(g, po).solve(ref, src.copy(order="F"))
    pm = mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, maxcy=60,
                   tolmax=1e-12, stop=abi.STOP_RESID, precision=abi.PREC_MIXED)
    s = MGSolver(g, pm)
    dphi = to_dev(zeros(g))
    s.solve(dphi, to_dev(src))
    assert s.last_report.status == abi.OK and s.last_report.resid <= 1e-12
    assert rel_l2(remove_mean(to_host(dphi)), remove_mean(ref)) < 1e-9
