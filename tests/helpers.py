"""Shared test helpers: tolerances and comparisons."""
import numpy as np

# FP32 field parity bar for the collide-stream path (relative L2 of
# dRho, ux, uy, uz against the oracle after N steps).
FIELD_REL_L2 = 1e-5


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def load_golden(name: str):
    from pathlib import Path
    path = Path(__file__).resolve().parent / "golden" / name
    rows = [l.split(";") for l in path.read_text().splitlines() if l and not l.startswith("#")]
    return np.array([[float(a), float(b)] for a, b in rows])


def field_errors(got: np.ndarray, ref: np.ndarray):
    """(rel L2 of dRho, rel L2 of the velocity vector field) for [4][n] macro arrays."""
    e_rho = rel_l2(got[0], ref[0])
    e_u = rel_l2(got[1:4].reshape(-1), ref[1:4].reshape(-1))
    return e_rho, e_u


def density_velocity_errors(got: np.ndarray, ref: np.ndarray):
    """(rel L2 of rho = 1 + dRho, rel L2 of the velocity vector field, max
    |delta dRho|) for [4][n] macro arrays.  For states near rest density the
    dRho field itself is tiny and its relative error only measures rounding."""
    e_rho = rel_l2(1.0 + got[0].astype(np.float64), 1.0 + ref[0].astype(np.float64))
    e_u = rel_l2(got[1:4].reshape(-1), ref[1:4].reshape(-1))
    return e_rho, e_u, float(np.max(np.abs(got[0] - ref[0]))) if got.shape[1] else 0.0


def plan_ijk(plan, level: int = 0):
    """(i, j, k) of every cell, decoded from the compressed rows
    (getCompressedIJK, include/cellFunctions.h:51-72)."""
    sh = plan.array("shifter", level)
    ri, rj, rk = plan.array("row_i", level), plan.array("row_j", level), plan.array("row_k", level)
    idx = np.arange(len(sh))
    head = np.where(sh >= 0, idx, idx + sh)
    row = sh[head]
    off = idx - head
    return ri[row] + off, rj[row], rk[row]
