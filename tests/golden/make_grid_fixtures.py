"""Copy the reference's grid-file fixtures (ANELASTIC_SL/run_dir/x?_grid.in:
the 256 x 64 x 256 uniform grid of its runfile, in the format load_grid
reads, ANELASTIC_SL/utils/loadGrid.F90:38-90) into tests/golden/ as
ref_x?_grid.in, with their SHA-256 in ref_grids.sha256.  Run once, in a
checkout that has the reference source tree next to it:

    python tests/golden/make_grid_fixtures.py /path/to/reference
"""
import hashlib
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    src = Path(ref_root) / "ANELASTIC_SL" / "run_dir"
    lines = []
    for d in (1, 2, 3):
        f = src / f"x{d}_grid.in"
        dst = HERE / f"ref_x{d}_grid.in"
        shutil.copyfile(f, dst)
        lines.append(f"{hashlib.sha256(dst.read_bytes()).hexdigest()}  {dst.name}")
    (HERE / "ref_grids.sha256").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_grid_fixtures.py <reference source root>")
    main(sys.argv[1])
