"""Procedural triangle soups and binary STL I/O for static bodies.

The generated surfaces stand in for the reference's CAD STLs: an axis
aligned box (exact voxelization checks), an icosphere (flow around a sphere)
and a 4-blade rotor.  All coordinates are in millimetres, triangles are
float32 [n][9] arrays (ax ay az bx by bz cx cy cz) with outward normals.
"""
from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from . import _abi as A


def box(lo, hi) -> np.ndarray:
    """Closed axis-aligned box, 12 triangles."""
    x0, y0, z0 = (float(v) for v in lo)
    x1, y1, z1 = (float(v) for v in hi)
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=np.float64)
    faces = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
             (3, 7, 6), (3, 6, 2), (0, 4, 7), (0, 7, 3), (1, 2, 6), (1, 6, 5)]
    return np.array([np.concatenate([v[a], v[b], v[c]]) for a, b, c in faces], dtype=np.float32)


def icosphere(subdivisions: int, radius: float, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Geodesic sphere: an icosahedron whose faces are split into 4
    `subdivisions` times, vertices projected onto the sphere
    (20 * 4**subdivisions triangles)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nxt = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nxt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nxt
    v = np.array(verts) * float(radius) + np.asarray(center, dtype=np.float64)
    return np.array([np.concatenate([v[a], v[b], v[c]]) for a, b, c in faces], dtype=np.float32)


def rotor(blades: int = 4, hub_radius: float = 8.0, tip_radius: float = 40.0, pitch_deg: float = 30.0,
          chord: float = 12.0, thickness: float = 2.0, hub_length: float = 16.0, center=(0.0, 0.0, 0.0),
          segments: int = 64, radial_cells: int = 8, seed: int = 0) -> np.ndarray:
    """Axial rotor about z through `center`: a closed hub cylinder and
    `blades` closed flat blades (chord x thickness plates from just outside
    the hub to the tip, pitched by `pitch_deg` about their radial axis),
    spaced evenly in angle from a seeded phase.  The solids touch nowhere,
    so ray parity gives their union.  Faces are subdivided radially into
    `radial_cells` strips."""
    rng = np.random.default_rng(seed)
    phase = float(rng.uniform(0.0, 2.0 * np.pi / blades))
    c = np.asarray(center, dtype=np.float64)
    tris = []
    # hub: closed cylinder
    h0, h1 = -0.5 * hub_length, 0.5 * hub_length
    ang = np.linspace(0.0, 2.0 * np.pi, segments, endpoint=False)
    ring = np.stack([hub_radius * np.cos(ang), hub_radius * np.sin(ang)], axis=1)
    for q in range(segments):
        a, b = ring[q], ring[(q + 1) % segments]
        p00, p01 = np.array([a[0], a[1], h0]), np.array([b[0], b[1], h0])
        p10, p11 = np.array([a[0], a[1], h1]), np.array([b[0], b[1], h1])
        tris += [(p00, p01, p11), (p00, p11, p10)]
        tris += [(np.array([0, 0, h0]), p01, p00), (np.array([0, 0, h1]), p10, p11)]
    # blades: boxes in local (radial r, chord s, thickness t) coordinates
    r0 = hub_radius * 1.03
    pitch = np.deg2rad(pitch_deg)
    for bidx in range(blades):
        th = phase + 2.0 * np.pi * bidx / blades
        er = np.array([np.cos(th), np.sin(th), 0.0])
        et = np.array([-np.sin(th), np.cos(th), 0.0])
        ez = np.array([0.0, 0.0, 1.0])
        es = np.cos(pitch) * et + np.sin(pitch) * ez      # chord direction
        en = -np.sin(pitch) * et + np.cos(pitch) * ez     # thickness direction

        def P(r, sc, tn):
            return r * er + sc * es + tn * en

        rs = np.linspace(r0, tip_radius, radial_cells + 1)
        hs, ht = 0.5 * chord, 0.5 * thickness
        for q in range(radial_cells):
            ra, rb = rs[q], rs[q + 1]
            for (s0, t0), (s1, t1) in (((-hs, -ht), (hs, -ht)), ((hs, -ht), (hs, ht)),
                                       ((hs, ht), (-hs, ht)), ((-hs, ht), (-hs, -ht))):
                a0, a1, b0, b1 = P(ra, s0, t0), P(ra, s1, t1), P(rb, s0, t0), P(rb, s1, t1)
                tris += [(a0, b0, b1), (a0, b1, a1)]
        for r_end, sign in ((r0, -1.0), (tip_radius, 1.0)):
            p = [P(r_end, -hs, -ht), P(r_end, hs, -ht), P(r_end, hs, ht), P(r_end, -hs, ht)]
            if sign > 0:
                tris += [(p[0], p[1], p[2]), (p[0], p[2], p[3])]
            else:
                tris += [(p[0], p[2], p[1]), (p[0], p[3], p[2])]
    out = np.array([np.concatenate([a + c, b + c, d + c]) for a, b, d in tris], dtype=np.float32)
    return out


def set_rotors(case: A.LbmCase, rotors) -> A.LbmCase:
    """Attach forcing rotors: a list of (triangles, dict(axis=0|1|2,
    origin=(x, y, z), radians_per_second=w)).  Arrays are kept alive on the case."""
    if len(rotors) > A.LBM_MAX_ROTORS:
        raise ValueError("too many rotors")
    keep = []
    case.rotor_count = len(rotors)
    for r, (tris, spec) in enumerate(rotors):
        arr = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        keep.append(arr)
        rt = case.rotor[r]
        rt.triangles = arr.ctypes.data_as(C.POINTER(C.c_float))
        rt.triangle_count = len(arr)
        rt.axis = spec.get("axis", 2)
        o = spec.get("origin", (0.0, 0.0, 0.0))
        for a in range(3):
            rt.origin[a] = o[a]
        rt.radians_per_second = spec.get("radians_per_second", 0.0)
    case._rotors = keep
    return case


def cylinder(radius: float, z0: float, z1: float, center=(0.0, 0.0), segments: int = 128) -> np.ndarray:
    """Closed cylinder along z with flat end caps (outward normals)."""
    cx, cy = float(center[0]), float(center[1])
    a = np.linspace(0.0, 2.0 * np.pi, segments, endpoint=False)
    p = np.stack([cx + radius * np.cos(a), cy + radius * np.sin(a)], axis=1)
    tris = []
    for q in range(segments):
        (x0, y0), (x1, y1) = p[q], p[(q + 1) % segments]
        tris += [((x0, y0, z0), (x1, y1, z0), (x1, y1, z1)), ((x0, y0, z0), (x1, y1, z1), (x0, y0, z1)),
                 ((cx, cy, z0), (x1, y1, z0), (x0, y0, z0)), ((cx, cy, z1), (x0, y0, z1), (x1, y1, z1))]
    return np.array([np.concatenate(t) for t in np.array(tris, dtype=np.float64)], dtype=np.float32)


def bored_block(half: float, radius: float, z0: float, z1: float, center=(0.0, 0.0), segments: int = 128,
                phase_deg: float = 0.0) -> np.ndarray:
    """Closed solid: the square prism |x|, |y| <= half (about `center`) along z
    with a cylindrical bore of `radius` whose `segments` polygon vertices sit
    at phase_deg + 360 q / segments degrees (the fixed outer wall of a
    Taylor-Couette cell, or a pipe in a square block).  The outer boundary
    follows each bore vertex's ray out to the square, with the square's
    corners inserted where they fall between two rays."""
    cx, cy = float(center[0]), float(center[1])
    a = np.radians(phase_deg) + np.linspace(0.0, 2.0 * np.pi, segments, endpoint=False)
    c, s = np.cos(a), np.sin(a)
    inner = np.stack([cx + radius * c, cy + radius * s], axis=1)
    scale = half / np.maximum(np.abs(c), np.abs(s))   # ray from the axis to the square
    outer = np.stack([cx + scale * c, cy + scale * s], axis=1)
    tris = []
    for q in range(segments):
        r = (q + 1) % segments
        i0, i1 = inner[q], inner[r]
        # outer path from ray q to ray q+1: a square corner strictly between
        # the two rays is a vertex of it
        path = [outer[q]]
        a0, a1 = a[q], a[q] + 2.0 * np.pi / segments
        for k in range(-1, 9):
            ac = np.pi / 4.0 + k * np.pi / 2.0
            if a0 + 1e-12 < ac < a1 - 1e-12:
                path.append(np.array([cx + half * np.sign(np.cos(ac)), cy + half * np.sign(np.sin(ac))]))
        path.append(outer[r])
        # bore (normal towards the axis)
        tris += [((*i0, z0), (*i1, z1), (*i1, z0)), ((*i0, z0), (*i0, z1), (*i1, z1))]
        for o0, o1 in zip(path[:-1], path[1:]):
            # outer sides
            tris += [((*o0, z0), (*o1, z0), (*o1, z1)), ((*o0, z0), (*o1, z1), (*o0, z1))]
        # end caps: the strip between the bore edge and the outer path, fanned from i0
        tris += [((*i0, z0), (*i1, z0), (*path[-1], z0)), ((*i0, z1), (*path[-1], z1), (*i1, z1))]
        for o0, o1 in zip(path[:-1], path[1:]):
            tris += [((*i0, z0), (*o1, z0), (*o0, z0)), ((*i0, z1), (*o0, z1), (*o1, z1))]
    return np.array([np.concatenate(t) for t in np.array(tris, dtype=np.float64)], dtype=np.float32)


def write_binary_stl(path, tris: np.ndarray) -> None:
    tris = np.asarray(tris, dtype=np.float32).reshape(-1, 9)
    with open(path, "wb") as fh:
        fh.write(b"lbm3_b200 generated".ljust(80, b" "))
        fh.write(struct.pack("<I", len(tris)))
        for t in tris:
            a, b, c = t[0:3], t[3:6], t[6:9]
            n = np.cross(b - a, c - a)
            ln = np.linalg.norm(n)
            n = n / ln if ln > 0 else n
            fh.write(struct.pack("<3f", *n))
            fh.write(t.astype("<f4").tobytes())
            fh.write(b"\0\0")


def read_binary_stl(path) -> np.ndarray:
    """Binary STL reader (readSTL, include/STLFunctions.h:317-462); degenerate
    triangles are kept here and dropped by the grid builder."""
    data = Path(path).read_bytes()
    (n,) = struct.unpack_from("<I", data, 80)
    rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]), count=n,
                        offset=84)
    return np.ascontiguousarray(rec["v"], dtype=np.float32)


def set_bodies(case: A.LbmCase, bodies) -> A.LbmCase:
    """Attach static bodies to a case.  `bodies` is a list of triangle arrays
    or (triangles, motion_dict) pairs; the body index is its wallID.  The
    arrays are kept alive on the case object."""
    if len(bodies) > A.LBM_MAX_BODIES:
        raise ValueError("too many bodies")
    keep = []
    case.body_count = len(bodies)
    for b, item in enumerate(bodies):
        tris, motion = (item, {}) if not isinstance(item, tuple) else item
        arr = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        keep.append(arr)
        body = case.body[b]
        body.triangles = arr.ctypes.data_as(C.POINTER(C.c_float))
        body.triangle_count = len(arr)
        body.motion = motion.get("motion", A.LBM_WALL_STATIC)
        body.axis = motion.get("axis", 2)
        o = motion.get("origin", (0.0, 0.0, 0.0))
        for a in range(3):
            body.origin[a] = o[a]
        body.radians_per_second = motion.get("radians_per_second", 0.0)
    case._bodies = keep
    return case
