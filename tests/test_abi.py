"""The C-ABI library loads and exports every symbol include/*.h declares
(CPU only: no compute call is made)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

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


def test_struct_sizes_match_the_c_header(tmp_path):
    """ctypes mirrors of every struct have the C compiler's size, and the
    header compiles as strict C99."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    names = {"anel_grid_desc": abi.GridDesc, "anel_mg_params": abi.MGParams,
             "anel_mg_report": abi.MGReport, "anel_ns_params": abi.NSParams,
             "anel_fields": abi.Fields, "anel_step_report": abi.StepReport,
             "anel_request": abi.Request, "anel_result": abi.Result,
             "anel_serve_stats": abi.ServeStats, "anel_restart_header": abi.RestartHeader}
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "anel.h"\nint main(void){\n' +
                   "".join(f'printf("%zu\\n", sizeof({n}));\n' for n in names) + "return 0;}\n")
    exe = tmp_path / "sz"
    # the header is plain C99 and compiles without warnings
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"),
                    str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                            check=True).stdout.split()]
    for (n, cls), got in zip(names.items(), sizes):
        assert C.sizeof(cls) == got, (n, C.sizeof(cls), got)


def test_header_compiles_as_cpp(tmp_path):
    """The header is usable from C++ too (extern "C" linkage, no C-only
    constructs): a translation unit that takes the address of one drop-in
    entry point compiles cleanly with g++."""
    import shutil
    import subprocess

    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    src = tmp_path / "h.cpp"
    src.write_text('#include "anel.h"\nvoid (*fp)(double*, double*, int32_t*, double*) = anel_mg_solve;\n'
                   "int main() { return fp ? 0 : 1; }\n")
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), "-c",
                    str(src), "-o", str(tmp_path / "h.o")], check=True)
