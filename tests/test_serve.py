"""Serving engine (anel_serve_*): members queued, admitted against an HBM
budget and run concurrently -- as cohorts of one bucket with batched
pressure solves where the multigrid is the column-layout z-line cycle,
member by member on their own streams otherwise.

* a served member equals the direct context path (set_fields of the
  shear.py state, project, step) bit for bit, which also pins the device
  initial-state generator to shear.py;
* a member's fields are the same alone and in a mix of overlapping members
  (here bit-identical);
* admission: a budget for one context serialises members of one bucket by
  re-using the context; a member larger than the budget fails with
  ANEL_ERR_NOMEM without blocking the others.
"""
import numpy as np
import pytest

from anelastic_solve_b200 import abi, shear
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200.ns import NSSolver
from anelastic_solve_b200.serve import ServeEngine

from .helpers import levels_for

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "rho")


def _params(g, Re=1000.0, Ri=0.12):
    lv = levels_for(g)
    mg = abi.make_mg_params((lv[0], lv[1], 1), maxcy=200, tolmax=1e-10, pre=2, post=2,
                            tbc=(0, 1, 0, 1, 0, 0), mode=abi.MODE_METRIC, stop=abi.STOP_RESID,
                            precision=abi.PREC_MIXED, smoother=abi.SMOOTHER_ZLINE)
    ns = abi.make_ns_params(Re=Re, Pr=1.0, g=-Ri, cfl=0.5, dtmax=1e9, ew=1, scal1_on=0)
    return mg, ns


def _bytes(g):
    G_ = (g.x.n + 2) * (g.y.n + 2) * (g.z.n + 2)
    return G_ * (8 * 14 + 32) + (64 << 20)


def _wait(e, ids):
    e.drain()
    out = {}
    while len(out) < len(ids):
        for r in e.poll(wait_ms=100):
            out[r["id"]] = r
    return out


def test_served_member_equals_direct_context():
    g = G.shear_layer_grid(32, 16, 32, stretched=True)
    mg, ns = _params(g)
    e = ServeEngine(hbm_budget_bytes=8 << 30, max_active=2)
    rid = e.submit(g, mg, ns, nsteps=3, seed=77, amp=1e-2, want_fields=True)
    res = _wait(e, [rid])[rid]
    e.close()
    assert res["status"] == abi.OK
    f = shear.shear_layer_fields(g, amp=1e-2, seed=77)
    s = NSSolver(g, mg, ns)
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    s.project()
    rep = s.step(3)
    got = s.get_fields(FIELDS)
    for k in FIELDS:
        np.testing.assert_array_equal(res["fields"][k], got[k], err_msg=k)
    assert res["max_div"] == rep.max_div and res["dt_last"] == rep.dt


def test_same_alone_and_in_mix():
    sizes = [(32, 16, 32), (64, 32, 64), (48, 24, 48), (32, 32, 32)]
    grids = {n: G.shear_layer_grid(*n, stretched=True) for n in sizes}
    ga = grids[(64, 32, 64)]
    mg_a, ns_a = _params(ga, Re=2000.0, Ri=0.2)
    e = ServeEngine(hbm_budget_bytes=16 << 30, max_active=4)
    rid = e.submit(ga, mg_a, ns_a, nsteps=4, seed=4242, amp=1e-2, want_fields=True)
    alone = _wait(e, [rid])[rid]
    assert alone["status"] == abi.OK
    ids, target = [], None
    rng = np.random.default_rng(5)
    for q in range(10):
        if q == 4:
            target = e.submit(ga, mg_a, ns_a, nsteps=4, seed=4242, amp=1e-2, want_fields=True)
            ids.append(target)
            continue
        n = sizes[q % len(sizes)]
        mg, ns = _params(grids[n], Re=float(rng.uniform(500, 4000)), Ri=float(rng.uniform(0.05, 0.3)))
        ids.append(e.submit(grids[n], mg, ns, nsteps=3, seed=100 + q, amp=1e-3))
    res = _wait(e, ids)
    st = e.stats()
    e.close()
    assert all(r["status"] == abi.OK for r in res.values())
    assert st["peak_active"] > 1  # members overlapped on the device
    for k in FIELDS:
        np.testing.assert_array_equal(res[target]["fields"][k], alone["fields"][k], err_msg=k)


def test_cohort_members_equal_direct_contexts():
    """Six members of one column-cycle bucket (64x32x128), physics and step
    counts of their own, submitted at once to one worker: they step as a
    cohort (batched pressure solves; members join and leave at step
    boundaries), and each equals its own direct context bit for bit."""
    g = G.shear_layer_grid(64, 32, 128, stretched=True)
    rng = np.random.default_rng(11)
    members = [(float(rng.uniform(500, 4000)), float(rng.uniform(0.05, 0.3)), 300 + q, 2 + q % 3)
               for q in range(6)]
    e = ServeEngine(hbm_budget_bytes=32 << 30, max_active=1)
    ids = []
    for Re, Ri, seed, nsteps in members:
        mg, ns = _params(g, Re=Re, Ri=Ri)
        ids.append(e.submit(g, mg, ns, nsteps=nsteps, seed=seed, amp=1e-2, want_fields=True))
    res = _wait(e, ids)
    st = e.stats()
    e.close()
    print(f"\npeak cohort {st['peak_cohort']}, peak active {st['peak_active']}")
    assert st["peak_cohort"] > 1
    for rid, (Re, Ri, seed, nsteps) in zip(ids, members):
        r = res[rid]
        assert r["status"] == abi.OK
        mg, ns = _params(g, Re=Re, Ri=Ri)
        f = shear.shear_layer_fields(g, amp=1e-2, seed=seed)
        s = NSSolver(g, mg, ns)
        s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
        s.project()
        rep = s.step(nsteps)
        got = s.get_fields(FIELDS)
        s.close()
        for k in FIELDS:
            np.testing.assert_array_equal(r["fields"][k], got[k], err_msg=f"member {rid} {k}")
        assert r["max_div"] == rep.max_div and r["dt_last"] == rep.dt


def test_budget_admission_and_oversized_member():
    g = G.shear_layer_grid(48, 24, 48, stretched=True)
    big = G.shear_layer_grid(128, 64, 128, stretched=True)
    mg, ns = _params(g)
    mgb, nsb = _params(big)
    budget = int(1.2 * _bytes(g))
    e = ServeEngine(hbm_budget_bytes=budget, max_active=4)
    ids = [e.submit(g, mg, ns, nsteps=2, seed=s) for s in (1, 2, 3)]
    ids.append(e.submit(big, mgb, nsb, nsteps=1, seed=9))
    res = _wait(e, ids)
    st = e.stats()
    e.close()
    assert [res[i]["status"] for i in ids[:3]] == [abi.OK] * 3
    assert res[ids[3]]["status"] == abi.ERR_NOMEM
    # one context at a time, re-used by the three members of its bucket
    assert st["peak_active"] == 1 and st["peak_bytes"] <= budget


def test_poisson_requests_batched_equal_alone():
    """Standalone pressure solves served as one bucket (64x32x128, mixed
    ZLINE, 1e-10): submitted at once to one worker they are solved in one
    batched solve, and each solution, cycle count and residual equals the
    one-member solve of its own context, bit for bit; a request with an
    initial guess starts from it."""
    import torch

    from anelastic_solve_b200.mg import MGSolver

    from .helpers import compatible, field

    g = G.shear_layer_grid(64, 32, 128, stretched=True)
    mg, _ = _params(g)
    rng = np.random.default_rng(17)
    rhs = [compatible(field(g, rng), g, abi.MODE_METRIC) for _ in range(5)]
    guess = 1e-3 * field(g, np.random.default_rng(3))
    e = ServeEngine(hbm_budget_bytes=16 << 30, max_active=1)
    ids = [e.submit_poisson(g, mg, r, phi0=(guess if q == 2 else None)) for q, r in enumerate(rhs)]
    res = _wait(e, ids)
    st = e.stats()
    e.close()
    print(f"\npoisson requests: peak cohort {st['peak_cohort']}, cycles {[res[i]['mg_iter'] for i in ids]}")
    assert st["peak_cohort"] > 1
    s = MGSolver(g, mg)
    for q, rid in enumerate(ids):
        r = res[rid]
        assert r["status"] == abi.OK and r["resid"] <= 1e-10
        p0 = guess if q == 2 else np.zeros(g.ghosted, order="F")
        d = torch.from_numpy(np.ascontiguousarray(p0.T)).cuda()
        s.solve(d, torch.from_numpy(np.ascontiguousarray(rhs[q].T)).cuda())
        alone = np.asfortranarray(d.cpu().numpy().T)
        assert r["mg_iter"] == s.last_report.iter and r["resid"] == s.last_report.resid
        np.testing.assert_array_equal(r["fields"]["p"], alone, err_msg=f"request {q}")
    s.close()
