"""Continuous-batching simulation server over the C ABI.

Requests (a case and a step count) arrive over time.  A request is admitted
as soon as a slot is free and its device footprint (the plan's
grid_memory_bytes) fits the remaining HBM budget; admitted domains keep their
populations and tables resident and advance together with update_batch, one
stream each, in chunks of steps, so that work of requests that arrived at
different times overlaps on the GPU.  A finished domain reads its result,
frees its memory and its slot, and the next waiting request is admitted.

Each result is the one the request gets when run alone: batched stepping is
bit-identical to stepping a domain by itself.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .grids import Grids, Plan, update_batch


@dataclass
class Request:
    rid: int
    case: A.LbmCase
    steps: int
    arrival: float = 0.0        # seconds after the server starts
    wall_id: int = 0            # body whose force is the result (-1: kinetic energy)
    footprint: int = 0          # device bytes, if known at submission (else planned at admission)
    updates: int = 0            # fluid cell updates per step, with footprint


@dataclass
class Result:
    rid: int
    steps: int
    updates: int                # fluid cell updates the request needed
    admitted: float
    finished: float
    arrival: float
    force: np.ndarray | None = None
    macro: np.ndarray | None = None

    @property
    def time_to_result(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Active:
    req: Request
    grids: Grids
    stream: object
    remaining: int
    footprint: int
    admitted: float
    updates: int


@dataclass
class Server:
    """`hbm_budget` bytes of device memory for resident domains, at most
    `max_slots` of them, stepped in chunks of up to `chunk_steps`."""
    hbm_budget: int
    max_slots: int = 16
    chunk_steps: int = 100
    keep_fields: bool = False
    results: list = field(default_factory=list)

    def run(self, requests) -> list:
        import torch
        pending = sorted(requests, key=lambda r: r.arrival)
        active: list[_Active] = []
        used = 0
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            # admission: arrived, a free slot, and the footprint fits
            while pending and pending[0].arrival <= now and len(active) < self.max_slots:
                req = pending[0]
                if req.footprint > 0:
                    footprint, updates = req.footprint, req.updates * req.steps
                else:
                    plan = Plan(req.case)
                    footprint = int(plan.info().grid_memory_bytes)
                    updates = int(plan.fluid_updates_per_iteration) * req.steps
                    plan.close()
                if footprint > self.hbm_budget:
                    raise ValueError(f"request {req.rid} needs {footprint} bytes, more than the whole budget")
                if used + footprint > self.hbm_budget:
                    break
                pending.pop(0)
                g = Grids(req.case)
                stream = torch.cuda.Stream()
                g.set_stream(stream.cuda_stream)
                active.append(_Active(req, g, stream, req.steps, footprint, time.perf_counter() - t0, updates))
                used += footprint
            if not active:
                # idle until the next arrival
                time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                continue
            chunk = min(self.chunk_steps, min(a.remaining for a in active))
            update_batch([a.grids for a in active], chunk)
            for a in active:
                a.remaining -= chunk
            done = [a for a in active if a.remaining == 0]
            for a in done:
                g = a.grids
                g.synchronize()
                res = Result(a.req.rid, a.req.steps, a.updates, a.admitted, 0.0, a.req.arrival)
                if a.req.wall_id >= 0:
                    res.force = g.wall_force(a.req.wall_id)
                if self.keep_fields:
                    res.macro = g.macro()
                res.finished = time.perf_counter() - t0
                g.close()
                used -= a.footprint
                self.results.append(res)
            active = [a for a in active if a.remaining > 0]
        return self.results


def summarize(results, wall_seconds: float) -> dict:
    """p50/p99 time-to-result and aggregate MLUPS of a served stream."""
    ttr = np.array([r.time_to_result for r in results])
    updates = sum(r.updates for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(ttr, 50)),
            "p99_s": float(np.percentile(ttr, 99)), "mlups": updates / wall_seconds / 1e6}


def channel_request(rid: int, edge: int, rng, steps: int, storage: int = A.LBM_STORE_F16,
                    u_in: float = 0.04, arrival: float = 0.0) -> Request:
    """A request of the serving stream: a 2e x e x e channel (velocity inlet,
    non-reflective outlet, velocity sides) around a seeded obstacle, an
    ellipsoid with semi-axes 0.1-0.3 e or an icosphere, at a Reynolds number
    uniform in 20-200 on the obstacle's largest extent."""
    from .cases import open_channel
    from .geometry import icosphere, set_bodies
    e = float(edge)
    if rng.random() < 0.5:
        axes = rng.uniform(0.1, 0.3, size=3) * e
    else:
        axes = np.full(3, rng.uniform(0.1, 0.3) * e)
    tris = icosphere(3, 1.0).reshape(-1, 3, 3) * axes + np.array([0.6 * e, 0.5 * e, 0.5 * e])
    reynolds = rng.uniform(20.0, 200.0)
    nu = u_in * 2.0 * float(axes.max()) / reynolds
    c = open_channel(2 * edge, edge, edge, u_in=u_in, nu_lattice=nu, storage=storage)
    set_bodies(c, [tris.reshape(-1, 9).astype(np.float32)])
    c.track_wall_force = 1
    return Request(rid, c, steps, arrival)
