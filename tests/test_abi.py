"""The C-ABI library loads and exports every symbol include/*.h declares
(CPU only: no compute call is made)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from anelastic_solve_b200 import _lib, abi
from anelastic_solve_b200 import grid as G

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(anel_[a-z0-9_]+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_signature_table_covers_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_struct_layouts_match_header():
    # anel_grid_desc: 3 int32 + pad + 3 double + 18 pointers
    assert C.sizeof(abi.GridDesc) == 4 * 3 + 4 + 8 * 3 + 8 * 18
    assert C.sizeof(abi.MGReport) == 4 + 4 + 8 + 8 + 8 + 8 + 4 + 4 + 8
    # anel_mg_params: offsets of the first and last fields
    assert abi.MGParams.tolmax.offset == 16
    assert abi.MGParams.verbose.offset == C.sizeof(abi.MGParams) - 4 - 4 or \
        abi.MGParams.verbose.offset == C.sizeof(abi.MGParams) - 4


def test_version_and_error_without_gpu():
    L = _lib.lib()
    assert L.anel_version() >= 100
    assert isinstance(_lib.last_error(), str)


def test_grid_file_roundtrip(tmp_path):
    ax = G.tanh_axis(64, 10.0, 2.0)
    f = tmp_path / "x3_grid.in"
    G.write_grid_file(f, ax, "X3")
    bx = G.read_grid_file(f)
    for a, b in zip(ax.arrays(), bx.arrays()):
        np.testing.assert_array_equal(a, b)
    assert bx.n == 64 and abs(bx.L - 20.0) < 1e-12


def test_tanh_grid_shape():
    ax = G.tanh_axis(64, 10.0, 2.0)
    assert abs(ax.xe[0] + 10.0) < 1e-12 and abs(ax.xe[64] - 10.0) < 1e-12
    dz = ax.dxc[1:-1]
    # ze = 10 tanh(2 s)/tanh(2): widest cells about z = 0, narrowest at the
    # walls, symmetric
    assert dz.argmax() in (31, 32)
    assert dz.argmin() in (0, 63)
    np.testing.assert_allclose(dz, dz[::-1], rtol=1e-12)
    np.testing.assert_allclose(ax.xc[1:-1], 0.5 * (ax.xe[1:-1] + ax.xe[:-2]), rtol=0, atol=1e-14)
