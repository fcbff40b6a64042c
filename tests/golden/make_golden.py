"""Regenerate the golden fixtures in this folder from the reference project.

Reads the reference's own stored Taylor–Green kinetic-energy histories
(cases/taylorGreenVortex/results/{COARSE,FINE}_kineticEnergy.txt, produced by
the reference driver cases/taylorGreenVortex/taylorGreenVortexMain.cu at
Re 1600, Ma 0.1, one grid level) and writes them unchanged, as
"t_star;energy" lines, to tgv_re1600_{128,256}_energy.txt.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = {
    "tgv_re1600_128_energy.txt": "cases/taylorGreenVortex/results/COARSE_kineticEnergy.txt",
    "tgv_re1600_256_energy.txt": "cases/taylorGreenVortex/results/FINE_kineticEnergy.txt",
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
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
