"""Golden vectors of the reference's moment-based open boundary.

Reads the reference's generated headers
include/boundaryConditions/{applyMBBC,restoreRho,restoreUxUyUz}.h, turns each
normalCode branch into a Python function that evaluates the same expressions
in float32 (numpy float32 scalars round every operation, left to right, as
the C code does without contraction), runs them on seeded random inputs for
all 26 outer normals, and writes mbbc_vectors.json.

Usage: python tests/golden/make_mbbc_golden.py /path/to/reference
"""
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
F = np.float32


def c_to_py(expr: str) -> str:
    expr = expr.strip().rstrip(";")
    # keep array subscripts f[12] as they are
    expr = re.sub(r"f\[(\d+)\]", r"f<\1>", expr)
    # float literals like 1.f, 2.f, (1.f/3.f) and bare integers
    expr = re.sub(r"(\d+)\.f\b", r"F(\1.0)", expr)
    expr = re.sub(r"(?<![\w.<])(\d+)(?![\w.>])", r"F(\1.0)", expr)
    return re.sub(r"f<(\d+)>", r"f[\1]", expr)


def branches(text: str):
    """Yield (normalCode, [statement lines]) for every branch of a header."""
    parts = re.split(r"(?:else )?if \( normalCode == (\d+) \)", text)
    for k in range(1, len(parts), 2):
        code = int(parts[k])
        body = parts[k + 1]
        body = body[body.index("{") + 1:]
        depth, out = 1, []
        for line in body.splitlines():
            s = line.strip()
            if s.startswith("}"):
                break
            if s and not s.startswith("//"):
                out.append(s)
        yield code, out


def compile_branch(stmts):
    lines = []
    for s in stmts:
        s = s.rstrip(";")
        if s.startswith("const float "):
            s = s[len("const float "):]
        lhs, rhs = s.split("=", 1)
        lines.append(f"{lhs.strip()} = {c_to_py(rhs)}")
    return lines


def build_functions(ref: Path):
    inc = ref / "include" / "boundaryConditions"
    funcs = {}
    for name in ("applyMBBC", "restoreRho", "restoreUxUyUz"):
        text = (inc / f"{name}.h").read_text()
        funcs[name] = {code: compile_branch(stmts) for code, stmts in branches(text)}
    return funcs


def run(lines, env):
    for line in lines:
        exec(line, {"F": F}, env)
    return env


def main(ref_root: str):
    funcs = build_functions(Path(ref_root))
    rng = np.random.default_rng(20240607)
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8, dtype=np.float32)
    cases = []
    for code in sorted(funcs["applyMBBC"]):
        for trial in range(3):
            f = (w * (1 + 0.2 * rng.standard_normal(27))).astype(np.float32)
            rho = F(1.0 + 0.01 * rng.standard_normal())
            u = (0.05 * rng.standard_normal(3)).astype(np.float32)
            # applyMBBC
            env = {"f": f.copy(), "rho": rho, "ux": u[0], "uy": u[1], "uz": u[2]}
            run(funcs["applyMBBC"][code], env)
            f_out = env["f"]
            # restoreRho: rho from known populations and u
            env = {"f": f.copy(), "rho": rho, "ux": u[0], "uy": u[1], "uz": u[2]}
            run(funcs["restoreRho"][code], env)
            rho_out = env["rho"]
            # restoreUxUyUz: u from known populations and rho
            env = {"f": f.copy(), "rho": rho, "ux": u[0], "uy": u[1], "uz": u[2]}
            run(funcs["restoreUxUyUz"][code], env)
            u_out = [env["ux"], env["uy"], env["uz"]]
            cases.append({"code": code, "f": [float(x) for x in f], "rho": float(rho),
                          "u": [float(x) for x in u], "f_out": [float(x) for x in f_out],
                          "rho_out": float(rho_out), "u_out": [float(x) for x in u_out]})
    out = {"source": "include/boundaryConditions/{applyMBBC,restoreRho,restoreUxUyUz}.h", "cases": cases}
    (HERE / "mbbc_vectors.json").write_text(json.dumps(out))
    print(f"mbbc_vectors.json: {len(cases)} cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_mbbc_golden.py /path/to/reference")
    main(sys.argv[1])
