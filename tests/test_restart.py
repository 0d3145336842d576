"""Restart files in the reference's layout (Restart.F90).

The library's codec is checked against an independent reader and writer of
Fortran sequential unformatted records (a 4-byte little-endian length
before and after each payload), with the record sequence of
write_flow_small / Greadfile (SMALL) and write_flow_big / start_big (BIG).
No file written by the reference is available, so the layout is pinned to
those routines' write and read statements.  On the GPU: a context's fields
survive a write / read round trip bit for bit, the read ghosts them as the
reference's start_* routines do (checked against the oracle's ghost), and a
run continued from a restart is bit-identical to the uninterrupted one.
"""
import struct

import numpy as np
import pytest

from anelastic_solve_b200 import abi, restart
from anelastic_solve_b200._lib import AnelError


def records(path):
    data = open(path, "rb").read()
    out, o = [], 0
    while o < len(data):
        (n,) = struct.unpack_from("<i", data, o)
        payload = data[o + 4:o + 4 + n]
        (m,) = struct.unpack_from("<i", data, o + 4 + n)
        assert m == n
        out.append(payload)
        o += n + 8
    return out


def write_records(path, recs):
    with open(path, "wb") as f:
        for r in recs:
            f.write(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)))


def sample(n=(6, 4, 5), seed=0):
    rng = np.random.default_rng(seed)
    shape = tuple(v + 2 for v in n)
    return {k: np.asfortranarray(rng.standard_normal(shape)) for k in abi.RESTART_FIELDS}


HDR = dict(nstep=37, time=1.25, delt=0.0125, g=-0.12, rho_0=1.0, scal1_0=0.5, Re=1000.0, Pr=1.0, Sc=0.7)


@pytest.mark.parametrize("layout", [abi.RESTART_SMALL, abi.RESTART_BIG])
def test_written_layout(tmp_path, layout):
    n = (6, 4, 5)
    f = sample(n)
    p = tmp_path / "flow"
    restart.write(p, f, restart.header(**HDR), layout)
    recs = records(p)
    assert len(recs) == 8
    hd = struct.unpack("<i8d", recs[0])
    assert hd == (HDR["nstep"], HDR["time"], HDR["delt"], HDR["g"], HDR["rho_0"], HDR["scal1_0"],
                  HDR["Re"], HDR["Pr"], HDR["Sc"])
    ext = struct.unpack(f"<{len(recs[1]) // 4}i", recs[1])
    if layout == abi.RESTART_SMALL:
        assert ext == (n[0] + 2, n[1] + 2, n[2] + 2)
    else:
        assert ext == (2, n[0] + 1, 2, n[1] + 1, 2, n[2] + 1)
    for q, k in enumerate(abi.RESTART_FIELDS):
        a = np.frombuffer(recs[2 + q], dtype="<f8").reshape(f[k].shape, order="F")
        np.testing.assert_array_equal(a, f[k])


@pytest.mark.parametrize("layout", [abi.RESTART_SMALL, abi.RESTART_BIG])
def test_read_independent_writer(tmp_path, layout):
    n = (5, 3, 4)
    f = sample(n, seed=1)
    ext = (n[0] + 2, n[1] + 2, n[2] + 2) if layout == abi.RESTART_SMALL else (2, n[0] + 1, 2, n[1] + 1, 2, n[2] + 1)
    recs = [struct.pack("<i8d", 12, 0.5, 0.01, -0.1, 1.0, 0.0, 500.0, 1.0, 1.0),
            struct.pack(f"<{len(ext)}i", *ext)]
    recs += [np.asfortranarray(f[k]).tobytes(order="F") for k in abi.RESTART_FIELDS]
    p = tmp_path / "dump"
    write_records(p, recs)
    h, got = restart.read(p, n, layout)
    assert (h.nstep, h.time, h.delt, h.g, h.Re) == (12, 0.5, 0.01, -0.1, 500.0)
    for k in abi.RESTART_FIELDS:
        np.testing.assert_array_equal(got[k], f[k])


def test_read_refuses_bad_files(tmp_path):
    n = (4, 4, 4)
    f = sample(n)
    p = tmp_path / "ok"
    restart.write(p, f, restart.header(**HDR), abi.RESTART_SMALL)
    with pytest.raises(AnelError) as e:  # other sizes (Greadfile's size check)
        restart.read(p, (4, 4, 6), abi.RESTART_SMALL)
    assert e.value.code == abi.ERR_SIZE
    with pytest.raises(AnelError):  # a SMALL file read as BIG: 12-byte extents record
        restart.read(p, n, abi.RESTART_BIG)
    data = open(p, "rb").read()
    t = tmp_path / "truncated"
    t.write_bytes(data[:-100])
    with pytest.raises(AnelError):
        restart.read(t, n, abi.RESTART_SMALL)
    b = tmp_path / "badmarker"
    b.write_bytes(data[:-4] + struct.pack("<i", 7))
    with pytest.raises(AnelError):
        restart.read(b, n, abi.RESTART_SMALL)


def test_filenames():
    assert restart.filename("flow_", 200) == "flow_200"
    assert restart.filename("big", 7, coords=(0, 1, 2)) == "big0_1_2.7"


# ------------------------------------------------------------------ GPU
def _case():
    from anelastic_solve_b200 import grid as G
    from anelastic_solve_b200 import shear
    from oracle.pyoracle import OracleNS

    from .helpers import levels_for

    g_ = G.shear_layer_grid(32, 16, 32, stretched=True)
    mgp = abi.make_mg_params(levels_for(g_), maxcy=200, tolmax=1e-10, tbc=(0, 1, 0, 1, 0, 0),
                             mode=abi.MODE_METRIC, stop=abi.STOP_RESID)
    nsp = abi.make_ns_params(Re=1000.0, Pr=1.0, g=-0.12, dtmax=0.01, ew=1, scal1_on=1)
    f = shear.shear_layer_fields(g_, amp=1e-3)
    o = OracleNS(g_, mgp, nsp, f)
    for name, vt in (("u", 0), ("v", 1), ("w", 2), ("rho", 4), ("scal1", 12)):
        o.ghost(f[name], vt)
    o.project()
    return g_, mgp, nsp, f, o


@pytest.mark.gpu
@pytest.mark.parametrize("layout", [abi.RESTART_SMALL, abi.RESTART_BIG])
def test_gpu_restart_continues_bitwise(tmp_path, layout):
    from anelastic_solve_b200.ns import NSSolver

    g_, mgp, nsp, f, o = _case()
    keys = ("u", "v", "w", "p", "rho", "scal1", "r", "densityBG")
    a = NSSolver(g_, mgp, nsp)
    a.set_fields({k: f[k] for k in keys})
    rep = a.step(2)
    p = tmp_path / restart.filename("flow_", rep.nstep + 1, (0, 0, 0) if layout == abi.RESTART_BIG else None)
    a.write_restart(p, restart.header(nstep=rep.nstep + 1, time=rep.time, delt=rep.dt, g=-0.12, Re=1000.0),
                    layout)
    b = NSSolver(g_, mgp, nsp)
    b.set_fields({k: f[k] for k in ("r", "densityBG")})
    h = b.read_restart(p, layout, icparam=True)
    assert h.nstep == rep.nstep + 1 and h.time == rep.time
    ga, gb = a.get_fields(abi.RESTART_FIELDS), b.get_fields(abi.RESTART_FIELDS)
    for k in abi.RESTART_FIELDS:
        np.testing.assert_array_equal(gb[k], ga[k], err_msg=f"{k} after read")
    # the read ghosts the file's fields as start_small does: compare with
    # the oracle's ghost() of the raw file contents
    _, raw = restart.read(p, (g_.x.n, g_.y.n, g_.z.n), layout)
    for k, vt in (("u", 0), ("v", 1), ("w", 2), ("p", 3), ("rho", 4), ("scal1", 12)):
        o.ghost(raw[k], vt)
        np.testing.assert_array_equal(gb[k], raw[k], err_msg=f"{k} ghosting")
    ra, rb = a.step(1), b.step(1)
    assert ra.time == rb.time and ra.nstep == rb.nstep
    ga, gb = a.get_fields(abi.RESTART_FIELDS), b.get_fields(abi.RESTART_FIELDS)
    for k in abi.RESTART_FIELDS:
        np.testing.assert_array_equal(gb[k], ga[k], err_msg=f"{k} after the continued step")
