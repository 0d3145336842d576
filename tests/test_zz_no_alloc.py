"""anel_divergence_noalloc: the divergence diagnostic that allocates no
device memory, called through the C-ABI and checked against the context
entry point anel_ns_ctx_divergence on the same fields.

The file name makes pytest collect it last; it also passes on its own in a
fresh process.  The tensors below are allocated by the test, not by the
entry point under test.
"""
import ctypes as C

import numpy as np
import pytest

from anelastic_solve_b200 import _lib, abi, shear
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200.ns import NSSolver

from .helpers import levels_for

pytestmark = pytest.mark.gpu

# mean |div|: plane-wise sums vs block-wise sums of the context path
MEAN_RTOL = 1e-12


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda()


def _ptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def _noalloc(g, u, v, w, rdxc, rdyc, rdzc, nz=None):
    out = (C.c_double * 2)(-1.0, -1.0)
    st = _lib.lib().anel_divergence_noalloc(g.x.n, g.y.n, g.z.n if nz is None else nz, _ptr(u), _ptr(v),
                                            _ptr(w), _ptr(rdxc), _ptr(rdyc), _ptr(rdzc), out, None)
    return st, (out[0], out[1])


@pytest.fixture(scope="module")
def case():
    g = G.shear_layer_grid(64, 32, 48, stretched=True)
    f = shear.shear_layer_fields(g, amp=1e-2, seed=4321)
    mgp = abi.make_mg_params(levels_for(g), maxcy=50, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    s = NSSolver(g, mgp, abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01))
    s.set_fields({k: f[k] for k in ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")})
    ref = s.divergence()
    fields = s.get_fields(("u", "v", "w"))
    dev = [_dev(fields[k]) for k in ("u", "v", "w")]
    met = [_dev(a.rdxc) for a in (g.x, g.y, g.z)]
    return g, ref, dev, met


def test_two_calls_match_context_entry_point(case):
    g, ref, (u, v, w), (rx, ry, rz) = case
    assert ref[1] > 0.0  # the perturbed field is not solenoidal
    st1, a = _noalloc(g, u, v, w, rx, ry, rz)
    st2, b = _noalloc(g, u, v, w, rx, ry, rz)
    assert st1 == abi.OK and st2 == abi.OK, _lib.last_error()
    for got in (a, b):
        assert got[1] == ref[1]  # max |div| is exact in any order
        assert abs(got[0] - ref[0]) <= MEAN_RTOL * abs(ref[0])
    # the maximum accumulator is cleared between calls: identical results
    assert a == b


def test_further_calls_leave_device_memory_unchanged(case):
    """What the entry point is for: after a first call on the device, more
    calls leave the device's free memory exactly as it was (no cudaMalloc,
    no allocating library routine)."""
    import torch

    g, ref, (u, v, w), (rx, ry, rz) = case
    st, first = _noalloc(g, u, v, w, rx, ry, rz)
    assert st == abi.OK, _lib.last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        st, got = _noalloc(g, u, v, w, rx, ry, rz)
        assert st == abi.OK and got == first
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_rejects_nz_beyond_fixed_scratch(case):
    g, ref, (u, v, w), (rx, ry, rz) = case
    st, out = _noalloc(g, u, v, w, rx, ry, rz, nz=4097)
    assert st == abi.ERR_SIZE
    assert "4096" in _lib.last_error()
    assert out == (-1.0, -1.0)
