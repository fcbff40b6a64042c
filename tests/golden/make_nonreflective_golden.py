"""Stored histories of the reference's non-reflective boundary study.

Reads cases/nonReflectiveTest/{dirichlet,characteristic,impedance2e-5,
impedance2e-6,impedance2e-7}.txt of the reference (50,000 steps each: the
area-averaged inlet velocity in m/s and pressure in Pa after every step of
cases/nonReflectiveTest/nonReflectiveTestMain.cu) and keeps the first 5,000
steps, every step up to 200, every 10th up to 2,000 and every 100th after,
as nonreflective_<name>.txt (iteration;velocity;pressure).

Usage: python tests/golden/make_nonreflective_golden.py /path/to/reference
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
NAMES = ["dirichlet", "characteristic", "impedance2e-5", "impedance2e-6", "impedance2e-7"]


def keep(it: int) -> bool:
    return it <= 200 or (it <= 2000 and it % 10 == 0) or (it <= 5000 and it % 100 == 0)


def main(ref: Path):
    for name in NAMES:
        src = ref / "cases" / "nonReflectiveTest" / f"{name}.txt"
        rows = src.read_text().splitlines()[1:]
        out = [f"# {src.relative_to(ref)}: iteration;inlet velocity [m/s];inlet pressure [Pa]"]
        for line in rows:
            it, u, p, _ = line.split(";")
            if keep(int(it)):
                out.append(f"{it};{u};{p}")
        (HERE / f"nonreflective_{name}.txt").write_text("\n".join(out) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(Path(sys.argv[1]))
