"""Regenerates quadrature_tables.json from the reference's include/*.dat files.

The triangle rules (tri2_<ng>.dat: weight, x, y on the reference triangle
(-1,-1),(1,-1),(-1,1), weights summing to 2) and the Gauss-Legendre edge rules
(legen<ngf>.dat: weight, t) are data that the reference reads at run time
(src/readgauss.f:21-35).  Parity with the reference requires the identical
points, so they are imported verbatim: every entry keeps the decimal text of
the .dat file, and is parsed at load time with a correctly rounded conversion,
as Fortran list-directed input does.

Usage: python spoc_b200/data/import_reference_tables.py REFERENCE_INCLUDE_DIR
(the reference checkout's include/ directory, which holds the .dat files)
"""
import json
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "quadrature_tables.json"


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    SRC = Path(sys.argv[1])
    if not any(SRC.glob("tri2_*.dat")):
        sys.exit(f"no tri2_*.dat in {SRC}")
    tables = {"triangle": {}, "edge": {}}
    for f in sorted(SRC.glob("tri2_*.dat")):
        ng = int(f.stem.split("_")[1])
        rows = [line.split() for line in f.read_text().splitlines() if line.strip()]
        assert len(rows) == ng and all(len(r) == 3 for r in rows), f
        tables["triangle"][str(ng)] = rows
    for f in sorted(SRC.glob("legen*.dat")):
        ngf = int(f.stem[5:])
        rows = [line.split() for line in f.read_text().splitlines() if line.strip()]
        assert len(rows) == ngf and all(len(r) == 2 for r in rows), f
        tables["edge"][str(ngf)] = rows
    tables["source"] = "dupontf/SPOC include/tri2_*.dat, include/legen*.dat"
    OUT.write_text(json.dumps(tables, indent=1) + "\n")
    print(f"wrote {OUT}: {sorted(map(int, tables['triangle']))} / {sorted(map(int, tables['edge']))}")


if __name__ == "__main__":
    main()
