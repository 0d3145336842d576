"""Argument checks of the C-ABI that the library makes before it touches
the GPU, so they run on the CPU (no device needed).

The reference's solver setup reports size violations through
mg_check_size's codes (ANELASTIC_SL/mgMK/mg_check_size.F90:77-151) and
stops on unknown boundary types (mgMK/mg_read_params.F90:122-123); here the
same inputs return ANEL_ERR_SIZE / ANEL_ERR_BC with a message, a NULL
context, and never exit the process.  Inputs the reference accepts but this
build does not handle return ANEL_ERR_UNSUPPORTED; bad enums ANEL_ERR_ARG.
"""
import ctypes as C

import pytest

from anelastic_solve_b200 import abi
from anelastic_solve_b200 import grid as G
from anelastic_solve_b200._lib import lib

GRID = G.shear_layer_grid(16, 8, 16)


def _mg(levels=(4, 3, 4), **kw):
    d, keep = abi.make_grid_desc(GRID)
    p = abi.make_mg_params(levels, **kw)
    st = C.c_int32(0)
    h = lib().anel_mg_create(C.byref(d), C.byref(p), 0, C.byref(st))
    return h, st.value, lib().anel_last_error().decode()


def _ns(grid=GRID, levels=(4, 3, 4), tb=None, **kw):
    d, keep = abi.make_grid_desc(grid)
    p = abi.make_mg_params(levels)
    n = abi.make_ns_params(**kw)
    for (dd, m, l), v in (tb or {}).items():
        n.tb[dd][m][l] = v
    st = C.c_int32(0)
    h = lib().anel_ns_create(C.byref(d), C.byref(p), C.byref(n), 0, C.byref(st))
    return h, st.value, lib().anel_last_error().decode()


MG_CASES = [
    ("unknown smoother", dict(smoother=7), abi.ERR_ARG, "unknown smoother"),
    ("unknown mode", dict(mode=5), abi.ERR_ARG, "unknown mode"),
    ("unknown precision", dict(precision=3), abi.ERR_ARG, "unknown precision"),
    ("no cycles", dict(maxcy=0), abi.ERR_ARG, "maxcy"),
    ("single level", dict(levels=(1, 1, 1)), abi.ERR_SIZE, "levels"),
    ("n not nC 2^(L-1)", dict(levels=(9, 4, 5)), abi.ERR_SIZE, "mg_check_size codes 4-6"),
    ("no finest coarsening", dict(levels=(4, 3, 0)), abi.ERR_SIZE, "mg_check_size codes 10-12"),
    ("bad boundary type", dict(tbc=(0, 5, 0, 1, 0, 0)), abi.ERR_BC, "bad boundary type tbc(2) = 5"),
    ("periodic and wall", dict(tbc=(0, 1, 0, 1, 0, 1)), abi.ERR_BC, "mixes periodic and wall"),
]


@pytest.mark.parametrize("name,kw,code,msg", MG_CASES, ids=[c[0] for c in MG_CASES])
def test_mg_create_refuses(name, kw, code, msg):
    h, st, err = _mg(**kw)
    assert not h and st == code and msg in err, (st, err)


NS_CASES = [
    ("unknown model", dict(models=(7, 0, 0)), abi.ERR_ARG, "unknown subgrid model"),
    ("dynamic test ratio", dict(les=True, models=(2, 2, 2), test_ratio=-1.0), abi.ERR_ARG, "test_ratio"),
    ("les_freq 0", dict(les=True, les_freq=0), abi.ERR_ARG, "les_freq"),
    ("unknown les_delta", dict(les=True, les_delta=9), abi.ERR_ARG, "les_delta"),
    ("x wall", dict(tb={(0, 0, 0): 1}), abi.ERR_UNSUPPORTED, "x and y periodic"),
    ("no CN row", dict(tb={(2, 0, 0): 4}), abi.ERR_BC, "no Crank-Nicolson row"),
]


@pytest.mark.parametrize("name,kw,code,msg", NS_CASES, ids=[c[0] for c in NS_CASES])
def test_ns_create_refuses(name, kw, code, msg):
    h, st, err = _ns(**kw)
    assert not h and st == code and msg in err, (st, err)


def test_dynamic_models_need_four_cells():
    small = G.shear_layer_grid(16, 8, 2)
    h, st, err = _ns(grid=small, levels=(4, 3, 2), les=True, models=(2, 2, 2))
    assert not h and st == abi.ERR_SIZE and "at least 4 cells" in err
