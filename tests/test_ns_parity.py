"""GPU RK3 stepper vs the CPU oracle (rk_ss / NSsolver restatement).

FP64 with the FP64 multigrid: bit-identical fields after sub-steps and
full steps, for both settings of the w edge-node flag.  Mixed-precision
multigrid: velocity and density within 1e-8 relative L2 of the FP64
oracle after the step count, pressure within 1e-9 after removing the mean.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200.ns import RK3, NSSolver
from oracle.pyoracle import OracleNS

from .helpers import levels_for, rel_l2, remove_mean

pytestmark = pytest.mark.gpu

CMP = ("u", "v", "w", "p", "rho", "scal1")


def setup_case(n=(32, 16, 32), ew=1, precision=abi.PREC_FP64, tol=1e-10, mode=abi.MODE_METRIC,
               scal1_on=1, Re=1000.0, g=-0.12, amp=1e-3, **nskw):
    g_ = G.shear_layer_grid(*n, stretched=True)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=tol, pre=2, post=2,
                             tbc=(0, 1, 0, 1, 0, 0), mode=mode, stop=abi.STOP_RESID,
                             precision=abi.PREC_FP64)
    nsp = abi.make_ns_params(Re=Re, Pr=1.0, g=g, dtmax=0.01, ew=ew, scal1_on=scal1_on, **nskw)
    f = shear.shear_layer_fields(g_, amp=amp)
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    start = {k: v.copy(order="F") for k, v in f.items()}
    mgp_gpu = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=tol, pre=2, post=2,
                                 tbc=(0, 1, 0, 1, 0, 0), mode=mode, stop=abi.STOP_RESID,
                                 precision=precision)
    s = NSSolver(g_, mgp_gpu, nsp)
    s.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    return g_, o, s, f, start


@pytest.mark.parametrize("ew", [1, 0])
def test_substeps_bitwise(ew):
    g_, o, s, f, start = setup_case(ew=ew)
    dt = 0.01
    for q, (a1, a2, a3, ec, fr) in enumerate(RK3):
        it_o, _ = o.substep(a1, a2, a3, fr * dt, dt)
        it_g, _ = s.substep(a1, a2, a3, fr * dt, dt)
        got = s.get_fields(CMP + ("q_u", "q_v", "q_w", "q_rho"))
        for name in CMP:
            np.testing.assert_array_equal(got[name], f[name], err_msg=f"{name} after sub-step {q}")
        for name in ("q_u", "q_v", "q_w", "q_rho"):
            np.testing.assert_array_equal(got[name][1:-1, 1:-1, 1:-1], f[name][1:-1, 1:-1, 1:-1],
                                          err_msg=f"{name} after sub-step {q}")
        assert it_o == it_g


@pytest.mark.parametrize("ew", [1, 0])
def test_steps_bitwise(ew):
    g_, o, s, f, start = setup_case(ew=ew)
    for n in range(3):
        ro = o.step()
        rg = s.step(1)
        assert ro.dt == rg.dt and ro.time == rg.time
        assert list(ro.mg_iter) == list(rg.mg_iter)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)


def test_divergence_bound_after_steps():
    """Divergence bound: max|div u| <= 1e-10 max|u| / dz_min (ew = 1)."""
    g_, o, s, f, start = setup_case(ew=1)
    rep = s.step(3)
    got = s.get_fields(("u", "v", "w"))
    umax = max(np.abs(got[k][1:-1, 1:-1, 1:-1]).max() for k in ("u", "v", "w"))
    dzmin = g_.z.dxc[1:-1].min()
    assert rep.max_div <= 1e-10 * umax / dzmin, (rep.max_div, umax, dzmin)
    avg, mx = s.divergence()
    assert mx == rep.max_div


def test_scal1_off_matches_reference_zero_scalar():
    g_, o, s, f, start = setup_case(scal1_on=0)
    for n in range(2):
        o.step()
        s.step(1)
    got = s.get_fields(CMP)
    for name in ("u", "v", "w", "p", "rho"):
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)
    assert not np.any(got["scal1"]) and not np.any(f["scal1"])


def test_dropin_rk_substep_equals_context():
    """anel_ns_init / anel_bind_fields / anel_rk_substep (host arrays, the
    reference's rk_ss argument list) give the same fields."""
    import ctypes as C

    from anelastic_solve_b200 import _lib

    g_, o, s, f, start = setup_case()
    L = _lib.lib()
    desc, keep = abi.make_grid_desc(g_)
    _lib.check(L.anel_ns_init(C.byref(desc), C.byref(s.mgp), C.byref(s.nsp)))
    host = {k: v.copy(order="F") for k, v in start.items()}
    fs = abi.Fields()
    for n in abi.FIELD_NAMES:
        if n in host and n not in ("nuT", "kappaT", "nappaT"):
            setattr(fs, n, abi.dptr(host[n]))
    _lib.check(L.anel_bind_fields(C.byref(fs)))
    dt = 0.01
    for (a1, a2, a3, ec, fr) in RK3:
        args = [C.c_double(x) for x in (a1, a2, a3, ec, fr * dt, dt)]
        ps = C.c_int32(1)
        st = C.c_int32(-99)
        L.anel_rk_substep(*[C.byref(a) for a in args], C.byref(ps), C.byref(st))
        assert st.value == 0, _lib.last_error()
        s.substep(a1, a2, a3, fr * dt, dt)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(host[name], got[name], err_msg=name)
    L.anel_ns_finalize()


def test_shear_layer_config0_20_steps():
    """64x32x64 shear layer, Re=1000, Pr=1, Ri=0.12, 20 steps at dt=0.01, MG
    to relative residual 1e-10 each sub-step: FP64 GPU == oracle bitwise."""
    g_, o, s, f, start = setup_case(n=(64, 32, 64))
    for n in range(20):
        o.step()
    s.step(20)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)


def test_mixed_precision_stepper_within_tolerance():
    """Mixed-precision MG inside the projection (the DNS and LES form): fields
    within 1e-8 rel L2 of the FP64 oracle after 5 steps; MG solved to
    1e-12 so the projection error stays below the tolerance."""
    g_, o, s, f, start = setup_case(precision=abi.PREC_MIXED, tol=1e-12)
    for n in range(5):
        o.step()
    s.step(5)
    got = s.get_fields(CMP)
    for name in ("u", "v", "w", "rho"):
        assert rel_l2(got[name], f[name]) < 1e-8, name
    assert rel_l2(remove_mean(got["p"]), remove_mean(f["p"])) < 1e-9


# ------------------------------------------------------------------- LES
LES_CASES = {
    # SSM with f_damp = 1 and the cube-root filter width, model on from step 1
    "ssm": dict(),
    # wall damping with the REAL(4) literals, 2-norm filter width, model
    # coefficients on a cadence of 2 from step 2 (nuT = 0 before)
    "ssm_damped_cadence": dict(les_damp=abi.DAMP_LITERAL, les_delta=abi.DELTA_2ROOT, les_start=2,
                               les_freq=2),
}


@pytest.mark.parametrize("case", list(LES_CASES))
def test_les_steps_bitwise(case):
    """LES of the shear layer (the 768x384x384 LES setup: SSM_const 0.0289, Pr_sgs 0.7,
    Re 50000, Ri 0.1, amplitude 1e-2): SGSdiff, the eddy terms of every RHS
    and the per-column LES Crank-Nicolson solve, FP64 GPU == oracle bitwise
    after four steps, eddy viscosities included."""
    g_, o, s, f, start = setup_case(Re=50000.0, g=-0.1, amp=1e-2, les=True, **LES_CASES[case])
    for n in range(4):
        ro = o.step()
        rg = s.step(1)
        assert ro.dt == rg.dt
        assert list(ro.mg_iter) == list(rg.mg_iter)
    names = CMP + ("nuT", "kappaT", "nappaT")
    got = s.get_fields(names)
    assert np.abs(f["nuT"]).max() > 0.0
    for name in names:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)


def test_les_step_fifty_smooths_scalars_like_oracle():
    """At nstep = 50 with time > 0 the driver smooths rho and scal1 with
    filterHF under the LES scalar models (NSsolver.F90:144-164): the GPU
    step equals the oracle's bit for bit, and the smoothing changed the
    scalars (a step at nstep = 51 differs)."""
    g_, o, s, f, start = setup_case(Re=50000.0, g=-0.1, amp=1e-2, les=True)
    # scalars with local extrema, so that filterHF has something to do
    rng = np.random.default_rng(50)
    f["rho"][...] += 0.05 * rng.standard_normal(g_.ghosted)
    f["scal1"][...] = rng.standard_normal(g_.ghosted)
    for name, vt in (("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    start = {k: v.copy(order="F") for k, v in f.items()}
    s.set_fields({k: start[k] for k in ("rho", "scal1")})
    o.set_clock(0.5, 50)
    s.set_clock(0.5, 50)
    o.step()
    s.step(1)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)
    s.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1")})
    s.set_clock(0.5, 51)
    s.step(1)
    other = s.get_fields(("rho",))
    assert not np.array_equal(other["rho"], got["rho"])


def test_les_mixed_precision_within_tolerance():
    """LES with the mixed-precision multigrid: fields within 1e-8 relative
    L2 of the FP64 oracle after three steps."""
    g_, o, s, f, start = setup_case(Re=50000.0, g=-0.1, amp=1e-2, les=True,
                                    precision=abi.PREC_MIXED, tol=1e-12)
    for n in range(3):
        o.step()
    s.step(3)
    got = s.get_fields(CMP + ("nuT",))
    for name in ("u", "v", "w", "rho", "nuT"):
        assert rel_l2(got[name], f[name]) < 1e-8, name


def test_step_host_equals_device_steps():
    """anel_ns_ctx_step_host (host state in and out, copies overlapped with
    the step) gives the same fields as set_fields + step + get_fields."""
    import torch

    g_, o, s, f, start = setup_case(ew=1, precision=abi.PREC_MIXED)
    keys = ("u", "v", "w", "p", "rho", "scal1")
    host = {k: np.asfortranarray(torch.zeros(g_.ghosted[::-1], dtype=torch.float64).pin_memory().numpy().T)
            for k in keys}
    for k in keys:
        host[k][...] = start[k]
    for _ in range(2):
        s.step_host(host, host, 1)
    ref = setup_case(ew=1, precision=abi.PREC_MIXED)[2]  # same start, device-resident steps
    ref.step(2)
    got = ref.get_fields(keys)
    for k in keys:
        np.testing.assert_array_equal(host[k], got[k], err_msg=k)


def test_divergence_matches_oracle():
    """anel_ns_ctx_divergence against the oracle's divergence
    (Routines.F90:54-183): the largest |div| bit for bit and the
    volume-weighted mean |div| within summation-order rounding, after FP64
    steps (identical fields) and on a field that is not divergence-free."""
    g_, o, s, f, start = setup_case()
    for _ in range(2):
        o.step()
    s.step(2)
    avg_g, max_g = s.divergence()
    avg_o, max_o = o.divergence()
    assert max_g == max_o and max_g > 0.0
    assert abs(avg_g - avg_o) <= 1e-12 * abs(avg_o)
    # a perturbed (not solenoidal) velocity, ghosted by both sides
    rng = np.random.default_rng(27)
    f["u"][...] += 1e-2 * rng.standard_normal(g_.ghosted)
    o.ghost(f["u"], 0)
    s.set_fields({"u": f["u"]})
    assert np.array_equal(s.get_fields(("u",))["u"], f["u"])
    avg_g, max_g = s.divergence()
    avg_o, max_o = o.divergence()
    assert max_g == max_o and max_g > 1e-3
    assert abs(avg_g - avg_o) <= 1e-12 * abs(avg_o)


def test_gravity_ramp_steps_bitwise():
    """Gravity switched on by the ramp of Routines.F90:27-52 (Ginit = 0,
    Gfinal = -Ri, GT1 = 0.01, GT2 = 0.045, dt = 0.01): g = 0 before GT1, the
    kept value at time == GT1, the linear ramp in between and Gfinal from
    GT2 on.  Six FP64 steps cover every branch; fields bit for bit."""
    import ctypes as C

    g_ = G.shear_layer_grid(32, 16, 32, stretched=True)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=1e-10, pre=2, post=2,
                             tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1)
    nsp.g_init, nsp.g_final, nsp.gt1, nsp.gt2 = 0.0, -0.12, 0.01, 0.045
    f = shear.shear_layer_fields(g_, amp=1e-3)
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    start = {k: v.copy(order="F") for k, v in f.items()}
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    for n in range(6):
        ro = o.step()
        rg = s.step(1)
        assert ro.time == rg.time and ro.dt == rg.dt
        assert list(ro.mg_iter) == list(rg.mg_iter)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)
    # the ramp changed the flow: constant gravity from t = 0 gives other fields
    nsp2 = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1)
    s2 = NSSolver(g_, mgp, nsp2)
    s2.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    s2.step(6)
    assert not np.array_equal(s2.get_fields(("w",))["w"], got["w"])


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_cn_launch_variants_bitwise(variant, monkeypatch):
    """Every launch variant of the DNS Crank-Nicolson column solve (rows per
    load batch, columns per block: the autotuner's candidates, forced here
    through ANEL_CN_VARIANT) gives the oracle's fields bit for bit over two
    steps."""
    monkeypatch.setenv("ANEL_CN_VARIANT", str(variant))
    g_, o, s, f, start = setup_case()
    for _ in range(2):
        o.step()
        s.step(1)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)


def test_clip_steps_bitwise():
    """The driver's optional clip (Clip=yes: clipVS of rho and scal1 after
    every sub-step, NSsolver.F90:206-211, Routines.F90:301-380): three FP64
    steps with a rho range that cuts the shear layer's tails, GPU == oracle
    bit for bit; the clipped rho stays in range and differs from the
    unclipped run."""
    g_ = G.shear_layer_grid(32, 16, 32, stretched=True)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=1e-10, pre=2, post=2,
                             tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    clip = (-0.8, 0.8, -0.5, 0.5)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1, clip=clip)
    f = shear.shear_layer_fields(g_, amp=1e-3)
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    start = {k: v.copy(order="F") for k, v in f.items()}
    s = NSSolver(g_, mgp, nsp)
    s.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    for _ in range(3):
        ro = o.step()
        rg = s.step(1)
        assert ro.dt == rg.dt and list(ro.mg_iter) == list(rg.mg_iter)
    got = s.get_fields(CMP)
    for name in CMP:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)
    rho = got["rho"][1:-1, 1:-1, 1:-1]
    assert rho.min() >= clip[0] and rho.max() <= clip[1]
    s2 = NSSolver(g_, mgp, abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1))
    s2.set_fields({k: start[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    s2.step(3)
    assert s2.get_fields(("rho",))["rho"][1:-1, 1:-1, 1:-1].min() < clip[0]


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_les_cn_launch_variants_bitwise(variant, monkeypatch):
    """Every launch variant of the LES Crank-Nicolson column solve (rows per
    load batch, columns per block: the autotuner's candidates, forced here
    through ANEL_CN_LES_VARIANT) gives the oracle's fields bit for bit over
    two LES steps."""
    monkeypatch.setenv("ANEL_CN_LES_VARIANT", str(variant))
    g_, o, s, f, start = setup_case(Re=50000.0, g=-0.1, amp=1e-2, les=True, **LES_CASES[list(LES_CASES)[0]])
    for _ in range(2):
        o.step()
        s.step(1)
    names = CMP + ("nuT", "kappaT", "nappaT")
    got = s.get_fields(names)
    for name in names:
        np.testing.assert_array_equal(got[name], f[name], err_msg=name)
