"""Batched multigrid solves (anel_mg_ctx_solve_batch) on the GPU.

Several independent pressure problems on one grid are solved together: one
launch per kernel for all members still iterating, the defect-correction
loop as one CUDA graph, each member stopping at its own tolerance test.
A member's result must not depend on the batch: every member is compared
bit for bit (solution, cycle count, residual) with the one-member solve of
the same problem, and one member with the CPU oracle's FP64 solution.
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


def problems(g, n, seed=31):
    """n seeded right-hand sides and initial guesses; member 1 starts from
    a good guess (fewer cycles), so members stop at different cycles."""
    rng = np.random.default_rng(seed)
    rhs = [compatible(field(g, rng), g, abi.MODE_METRIC) for _ in range(n)]
    phi0 = [zeros(g) for _ in range(n)]
    return rhs, phi0


def batch_params(g, tol=1e-10):
    lv = levels_for(g)[:2] + (1,)
    return mg_params(g, levels=lv, mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE, maxcy=60,
                     tolmax=tol, stop=abi.STOP_RESID, precision=abi.PREC_MIXED)


@pytest.mark.parametrize("variant", [None, 1, 3, 4])
def test_batch_equals_members_alone(variant, monkeypatch):
    """Four members of 64x32x256 (column cycle, 8 rows per lane) with the
    autotuned sweep variants and with variants 1, 3 (bulk-copy staged) and
    4 (register factors) forced: batched == alone, bit for bit."""
    if variant is not None:
        monkeypatch.setenv("ANEL_COL_VARIANT", str(variant))
    g = G.shear_layer_grid(64, 32, 256, stretched=True)
    n = 4
    rhs, phi0 = problems(g, n)
    s = MGSolver(g, batch_params(g))
    # member 1: a head start (a solution to 1e-4 of this problem)
    loose = MGSolver(g, batch_params(g, tol=1e-4))
    d1 = to_dev(phi0[1])
    loose.solve(d1, to_dev(rhs[1]))
    phi0[1] = to_host(d1)
    loose.close()
    alone, reps_alone = [], []
    for b in range(n):
        d = to_dev(phi0[b])
        s.solve(d, to_dev(rhs[b]))
        alone.append(to_host(d))
        reps_alone.append(s.last_report)
    dphis = [to_dev(phi0[b]) for b in range(n)]
    drhs = [to_dev(rhs[b]) for b in range(n)]
    reps = s.solve_batch(dphis, drhs)
    s.close()
    iters = [(r.iter, ra.iter) for r, ra in zip(reps, reps_alone)]
    print(f"\nbatch of {n} (variant {variant}): cycles batched/alone {iters}")
    assert reps_alone[1].iter < reps_alone[0].iter  # members stopped at different cycles
    for b in range(n):
        assert reps[b].status == abi.OK
        assert reps[b].iter == reps_alone[b].iter
        assert reps[b].resid == reps_alone[b].resid
        np.testing.assert_array_equal(to_host(dphis[b]), alone[b], err_msg=f"member {b}")


def test_batch_of_one_and_oracle():
    """A batch of one is the one-member solve; its solution agrees with the
    oracle's FP64 solve (to 1e-13) within 1e-9 after mean removal."""
    g = G.shear_layer_grid(32, 16, 128, stretched=True)
    rhs, phi0 = problems(g, 1, seed=5)
    po = mg_params(g, levels=levels_for(g)[:2] + (1,), mode=abi.MODE_METRIC, smoother=abi.SMOOTHER_ZLINE,
                   maxcy=100, tolmax=1e-13, stop=abi.STOP_RESID)
    ref = zeros(g)
    OracleMG(g, po).solve(ref, rhs[0].copy(order="F"))
    s = MGSolver(g, batch_params(g, tol=1e-12))
    d_alone = to_dev(phi0[0])
    s.solve(d_alone, to_dev(rhs[0]))
    d = to_dev(phi0[0])
    (rep,) = s.solve_batch([d], [to_dev(rhs[0])])
    s.close()
    got = to_host(d)
    np.testing.assert_array_equal(got, to_host(d_alone))
    e = rel_l2(remove_mean(got), remove_mean(ref))
    print(f"\nbatch of one: {rep.iter} cycles, resid {rep.resid:.3e}, rel-L2 vs oracle {e:.3e}")
    assert rep.status == abi.OK and rep.resid <= 1e-12
    assert e < 1e-9


def test_batch_refuses_row_major_context():
    """A context without the column cycle (RBPGS smoother) refuses."""
    g = G.shear_layer_grid(16, 8, 16, stretched=False)
    s = MGSolver(g, mg_params(g, precision=abi.PREC_MIXED))
    rhs, phi0 = problems(g, 2)
    with pytest.raises(Exception):
        s.solve_batch([to_dev(p) for p in phi0], [to_dev(r) for r in rhs])
    s.close()
