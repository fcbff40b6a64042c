"""Generate mbbc_tables.h: coefficient tables of the moment-based open boundary.

For every outer normal n of a boundary cell (6 faces, 12 edges, 8 corners)
the populations split into known ones (c_a n_a >= 0 on every axis) and
unknown ones.  The boundary closes the unknowns from equilibrium moments:

* applyMBBC: pick, greedily by rank, as many moments (from the 23 central
  D3Q27 moments, in a fixed order) as there are unknowns; the unknowns then
  solve  (S Mfu) f_u = m_eq(S) - (S Mfk) f_k.
* restoreRho / restoreUxUyUz: moments that do not involve the unknowns at all
  (the left null space of Mfu) give relations between the known populations
  and (rho, rho u); one relation (rho) or three (u) are selected the same
  greedy way and solved.  Faces restore u with the closed form of the
  reference's face generator instead (normal velocity from rhoZ, tangential
  from k_nnt = 0).

This restates the algorithm of the reference's generator
(tools/CppCodeGeneratorForMBBC/helperMain.py:115-341, applyMBBC.py,
restoreRho.py, restoreUxUyUz.py, restoreFaceUxUyUz.py) and writes tables
instead of unrolled code.  Run:  python lbm3_b200/csrc/gen_mbbc.py
"""
from __future__ import annotations

from fractions import Fraction
from pathlib import Path

import sympy as sp

CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]
CY = [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1]

# the 23 moment exponents (a, b, c) in the order the selection walks them
MOMENTS = ["000", "100", "010", "001", "200", "020", "002", "011", "101", "110", "111", "210", "201", "120",
           "021", "102", "012", "022", "202", "220", "211", "121", "112"]
ORDER = [sum(int(ch) for ch in m) for m in MOMENTS]

# normals in the reference's enumeration order
NORMALS = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1],
           [0, 1, 1], [1, 0, 1], [1, 1, 0], [0, -1, -1], [-1, 0, -1], [-1, -1, 0],
           [0, 1, -1], [1, 0, -1], [1, -1, 0], [0, -1, 1], [-1, 0, 1], [-1, 1, 0],
           [1, 1, 1], [-1, -1, -1], [-1, 1, 1], [1, -1, 1], [1, 1, -1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]]


def linear_parts():
    """Constant (rho) and first-order (rho u) parts of the equilibrium
    moment M_a(ux) M_b(uy) M_c(uz) rho with M_0 = 1, M_1 = u, M_2 = 1/3 + u^2."""
    const = {0: sp.Integer(1), 1: sp.Integer(0), 2: sp.Rational(1, 3)}
    Q, Qu, Qrho = [], [], []
    for m in MOMENTS:
        e = [int(ch) for ch in m]
        rho = sp.prod([const[x] for x in e])
        lin = []
        for a in range(3):
            if e[a] != 1:
                lin.append(sp.Integer(0))
                continue
            lin.append(sp.prod([const[e[b]] for b in range(3) if b != a]))
        Q.append([rho] + lin)
        Qu.append(lin)
        Qrho.append([rho])
    return sp.Matrix(Q), sp.Matrix(Qu), sp.Matrix(Qrho)


def greedy_rows(M, count, first=0):
    rows = [first]
    i = first + 1
    while len(rows) < count:
        if i >= M.rows:
            raise RuntimeError("ran out of independent rows")
        if M.extract(rows + [i], list(range(M.cols))).rank() > M.extract(rows, list(range(M.cols))).rank():
            rows.append(i)
        i += 1
    return rows


def normal_data(n):
    known = [d for d in range(27) if min(CX[d] * n[0], CY[d] * n[1], CZ[d] * n[2]) >= 0]
    unknown = [d for d in range(27) if d not in known]
    pw = [[CX[d] ** int(m[0]) * CY[d] ** int(m[1]) * CZ[d] ** int(m[2]) for d in range(27)] for m in MOMENTS]
    Mk = sp.Matrix([[row[d] for d in known] for row in pw])
    Mu = sp.Matrix([[row[d] for d in unknown] for row in pw])
    Q, Qu, Qrho = linear_parts()
    S = greedy_rows(Mu, len(unknown))
    Su_mfu = Mu.extract(S, list(range(Mu.cols)))
    inv = Su_mfu.inv()
    Smfk = Mk.extract(S, list(range(Mk.cols)))
    # moment relations free of the unknowns, lowest moment order first
    null = Mu.T.nullspace()
    null = sorted(null, key=lambda v: sum(ORDER[i] for i in range(len(v)) if v[i] != 0))
    C = sp.Matrix.hstack(*null)
    CQu = C.T * Qu
    su = greedy_rows(CQu, 3)
    Su = sp.eye(CQu.rows).extract(su, list(range(CQu.rows)))
    u_inv = (Su * C.T * Qu).inv()
    u_mfk = Su * C.T * Mk
    u_q = Su * C.T * Qrho
    Srho = sp.eye(C.cols).extract([0], list(range(C.cols)))
    r_q = (Srho * C.T * Qrho)[0, 0]
    r_mfk = Srho * C.T * Mk
    r_qu = Srho * C.T * Qu
    return dict(normal=n, known=known, unknown=unknown, S=S, inv=inv, Smfk=Smfk, u_inv=u_inv, u_mfk=u_mfk,
                u_q=u_q, r_q=r_q, r_mfk=r_mfk, r_qu=r_qu)


def frac(x):
    x = sp.Rational(x)
    return Fraction(int(x.p), int(x.q))


def c_float(x) -> str:
    q = frac(x)
    if q.denominator == 1:
        return f"{q.numerator}.f"
    return f"{q.numerator}.f / {q.denominator}.f"


def emit(path: Path):
    rows = [normal_data(n) for n in NORMALS]
    L = []
    L.append("/* GENERATED by gen_mbbc.py -- do not edit. */")
    L.append("/* Moment-based open-boundary tables for the 26 outer normals (see gen_mbbc.py).")
    L.append(" * Plain C aggregate data, readable from C, C++ and CUDA device code. */")
    L.append("#ifndef LBM_MBBC_TABLES_TYPE_H")
    L.append("#define LBM_MBBC_TABLES_TYPE_H")
    L.append("")
    L.append("#define LBM_MBBC_NORMALS 26")
    L.append("#define LBM_MBBC_MAX_UNKNOWN 19")
    L.append("")
    L.append("typedef struct LbmMbbcTable {")
    L.append("    int code;                 /* (nx+5)*100 + (ny+5)*10 + (nz+5) */")
    L.append("    int nk, nu;               /* known / unknown population counts */")
    L.append("    int face;                 /* 1: face, velocity from the face closed form */")
    L.append("    signed char known[27];")
    L.append("    signed char unknown[LBM_MBBC_MAX_UNKNOWN];")
    L.append("    signed char moment[LBM_MBBC_MAX_UNKNOWN];       /* selected moment (0..22) per equation */")
    L.append("    signed char smfk[LBM_MBBC_MAX_UNKNOWN][27];     /* moment weight of each known population */")
    L.append("    float inv[LBM_MBBC_MAX_UNKNOWN][LBM_MBBC_MAX_UNKNOWN];  /* (S Mfu)^-1 */")
    L.append("    float rhoQ;               /* restoreRho: s = rhoQ + rhoQu . u */")
    L.append("    float rhoQu[3];")
    L.append("    float rhoMfk[27];         /*             rho = (rhoMfk . f_k) / s */")
    L.append("    float uInv[3][3];         /* restoreUxUyUz (edges, corners) */")
    L.append("    float uMfk[3][27];")
    L.append("    float uQ[3];")
    L.append("} LbmMbbcTable;")
    L.append("")
    L.append("#endif")
    L.append("")
    L.append("/* host data; define LBM_MBBC_TYPES_ONLY to include the type alone */")
    L.append("#if !defined(LBM_MBBC_TYPES_ONLY) && !defined(LBM_MBBC_TABLES_DATA_H)")
    L.append("#define LBM_MBBC_TABLES_DATA_H")
    L.append("")
    L.append("/* coefficients are correctly rounded num.f / den.f of the exact rationals */")
    L.append("static const LbmMbbcTable kLbmMbbc[LBM_MBBC_NORMALS] = {")
    for r in rows:
        n = r["normal"]
        code = (n[0] + 5) * 100 + (n[1] + 5) * 10 + (n[2] + 5)
        nk, nu = len(r["known"]), len(r["unknown"])
        face = int(sum(abs(x) for x in n) == 1)
        known = r["known"] + [0] * (27 - nk)
        unknown = r["unknown"] + [0] * (19 - nu)
        moment = r["S"] + [0] * (19 - nu)
        smfk = [[int(r["Smfk"][i, k]) if i < nu and k < nk else 0 for k in range(27)] for i in range(19)]
        inv = [[c_float(r["inv"][i, j]) if i < nu and j < nu else "0.f" for j in range(19)] for i in range(19)]
        rmfk = [c_float(r["r_mfk"][0, k]) if k < nk else "0.f" for k in range(27)]
        rqu = [c_float(r["r_qu"][0, a]) for a in range(3)]
        uinv = [[c_float(r["u_inv"][i, j]) for j in range(3)] for i in range(3)]
        umfk = [[c_float(r["u_mfk"][i, k]) if k < nk else "0.f" for k in range(27)] for i in range(3)]
        uq = [c_float(r["u_q"][i, 0]) for i in range(3)]
        L.append("    {%d, %d, %d, %d," % (code, nk, nu, face))
        L.append("     {" + ", ".join(map(str, known)) + "},")
        L.append("     {" + ", ".join(map(str, unknown)) + "},")
        L.append("     {" + ", ".join(map(str, moment)) + "},")
        L.append("     {" + ", ".join("{" + ", ".join(map(str, row)) + "}" for row in smfk) + "},")
        L.append("     {" + ", ".join("{" + ", ".join(row) + "}" for row in inv) + "},")
        L.append("     %s, {%s}," % (c_float(r["r_q"]), ", ".join(rqu)))
        L.append("     {" + ", ".join(rmfk) + "},")
        L.append("     {" + ", ".join("{" + ", ".join(row) + "}" for row in uinv) + "},")
        L.append("     {" + ", ".join("{" + ", ".join(row) + "}" for row in umfk) + "},")
        L.append("     {" + ", ".join(uq) + "}},")
    L.append("};")
    L.append("")
    L.append("#endif")
    path.write_text("\n".join(L) + "\n")


if __name__ == "__main__":
    emit(Path(__file__).resolve().parent / "mbbc_tables.h")
    print("wrote mbbc_tables.h")
