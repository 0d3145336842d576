"""Grid-file format pinned on the reference's own fixtures (copied by
tests/golden/make_grid_fixtures.py from ANELASTIC_SL/run_dir/x?_grid.in,
the 256 x 64 x 256 grid of its runfile; format of loadGrid.F90:38-90)."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from anelastic_solve_b200 import abi
from anelastic_solve_b200 import grid as G
from oracle.pyoracle import OracleMG

GOLDEN = Path(__file__).resolve().parent / "golden"
SIZES = {1: 256, 2: 64, 3: 256}


def _sha_ok():
    for line in (GOLDEN / "ref_grids.sha256").read_text().split("\n"):
        if line.strip():
            h, name = line.split()
            assert hashlib.sha256((GOLDEN / name).read_bytes()).hexdigest() == h, name


@pytest.mark.parametrize("d", [1, 2, 3])
def test_reference_grid_file_parses_and_roundtrips(d, tmp_path):
    _sha_ok()
    a = G.read_grid_file(GOLDEN / f"ref_x{d}_grid.in")
    assert a.n == SIZES[d] and a.gridtype == "uniform"
    # metric identities of the file (16 printed digits)
    np.testing.assert_allclose(np.diff(a.xe), a.dxc[1:], rtol=1e-12)
    np.testing.assert_allclose(a.rdxc, 1.0 / a.dxc, rtol=1e-12)
    np.testing.assert_allclose(a.rdxe, 1.0 / a.dxe, rtol=1e-12)
    # loadGrid.F90:79-90 end fix-ups
    n = a.n
    assert a.dxc[n + 1] == a.dxc[n] and a.rdxc[n + 1] == a.rdxc[n]
    assert a.dxe[0] == a.dxe[1] and a.rdxe[0] == a.rdxe[1]
    assert a.xe[n + 1] == a.xe[n] + a.dxc[n + 1]
    # our writer and reader reproduce the arrays exactly
    out = tmp_path / "g.in"
    G.write_grid_file(out, a, label=f"X{d}")
    b = G.read_grid_file(out)
    for x, y in zip(a.arrays(), b.arrays()):
        np.testing.assert_array_equal(x, y)


def test_runfile_level_table_on_reference_grid():
    """mg_init level maps (mg_init.F90:125-220) for the runfile's solver
    block (Sturb.ini:125-135: nxlevels=4, nylevels=3, nzlevels=8) on the
    reference's own grid files."""
    g = G.Grid(*(G.read_grid_file(GOLDEN / f"ref_x{d}_grid.in") for d in (1, 2, 3)))
    p = abi.make_mg_params((4, 3, 8), pre=[14, 10, 4, 4, 2, 2, 2, 2], post=[12, 10, 4, 4, 2, 2, 2, 2],
                           tbc=(0, 1, 0, 1, 0, 0))
    t = OracleMG(g, p).levels()
    assert list(t[:, 0]) == [33, 33, 33, 33, 33, 65, 129, 257]
    assert list(t[:, 1]) == [17, 17, 17, 17, 17, 17, 33, 65]
    assert list(t[:, 2]) == [3, 5, 9, 17, 33, 65, 129, 257]
