"""Regenerate the golden fixtures in this folder from the reference project.

Reads the reference's own stored Taylor–Green kinetic-energy histories
(cases/taylorGreenVortex/results/{COARSE,FINE,QUADRATIC}_kineticEnergy.txt,
produced by the reference driver cases/taylorGreenVortex/taylorGreenVortexMain.cu
at Re 1600, Ma 0.1: 128^3 and 256^3 on one grid level, and 128^3 with the
central cube on a second level with the quadratic interface) and writes
them unchanged, as "t_star;energy" lines, to tgv_re1600_*_energy.txt.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = {
    "tgv_re1600_128_energy.txt": "cases/taylorGreenVortex/results/COARSE_kineticEnergy.txt",
    "tgv_re1600_256_energy.txt": "cases/taylorGreenVortex/results/FINE_kineticEnergy.txt",
    "tgv_re1600_128_refined_energy.txt": "cases/taylorGreenVortex/results/QUADRATIC_kineticEnergy.txt",
}


def main(ref_root: str) -> None:
    root = Path(ref_root)
    for out, rel in SOURCES.items():
        lines = (root / rel).read_text().splitlines()
        header, rows = lines[0], [l for l in lines[1:] if l.strip()]
        text = "# source: " + rel + "\n# " + header + "\n" + "\n".join(rows) + "\n"
        (HERE / out).write_text(text)
        print(f"{out}: {len(rows)} samples")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
