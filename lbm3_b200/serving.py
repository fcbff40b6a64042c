"""Continuous-batching simulation server over the C ABI.

Requests (a case and a step count) arrive over time.  A request is admitted
as soon as a slot is free and its device footprint (the plan's
grid_memory_bytes, every device array the build allocates) fits the
remaining HBM budget.  Its grids are then built on a builder thread (host
voxelization and tables, upload, initial condition) while the domains
already resident keep stepping; once built, a domain joins the active set.
Active domains keep their populations and tables resident and advance in
chunks of steps.  Single-level domains without rotors advance in a packed
batch per storage type: one persistent collide-stream launch over the packed
block table of all of them, one open-boundary and one periodic launch per
step, replayed as a CUDA graph (PackedBatch); the batch is rebuilt whenever
a domain joins or leaves.  A domain that joins at the other esotwist parity
than the batch steps once on its own first (as a batch of one).  Other domains (several levels,
rotors, FP64) advance with update_batch on their own streams.  A finished
domain reads its result, frees its memory and its slot, and the next
waiting request is admitted.

Each result is the one the request gets when served alone: a packable
domain always steps through the packed kernel (alone it is a batch of one),
whose per-item work does not depend on the other members, so its fields are
bit-identical alone and in the mix; against lbm_update_all_grids, whose
kernel takes the level descriptor as a parameter, they agree to FP32
rounding.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .grids import Grids, PackedBatch, Plan, update_batch


@dataclass
class Request:
    rid: int
    case: A.LbmCase
    steps: int
    arrival: float = 0.0        # seconds after the server starts
    wall_id: int = 0            # body whose force is the result; -1: the kinetic energy instead
    footprint: int = 0          # device bytes, if known at submission (else planned at admission)
    updates: int = 0            # fluid cell updates per step, with footprint
    energy_ref: tuple = (1.0, 1000.0)  # (u_ref m/s, domain length mm) normalising the kinetic energy


@dataclass
class Result:
    rid: int
    steps: int
    updates: int                # fluid cell updates the request needed
    admitted: float
    finished: float
    arrival: float
    force: np.ndarray | None = None
    energy: float | None = None
    macro: np.ndarray | None = None

    @property
    def time_to_result(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Active:
    req: Request
    grids: Grids | None
    stream: object
    remaining: int
    footprint: int
    admitted: float
    updates: int
    build: object = None        # future of the grid build while it runs
    packable: bool = False      # single level, no rotors, FP32 / FP16 / BF16

    @property
    def parity(self) -> int:
        return (self.req.steps - self.remaining) & 1


def _packable(g: Grids) -> bool:
    c = g.case
    return g.level_count() == 1 and c.rotor_count == 0 and c.storage != A.LBM_STORE_F64


def _footprint(req: Request):
    if req.footprint > 0:
        return req.footprint, req.updates * req.steps
    plan = Plan(req.case)
    try:
        return int(plan.info().grid_memory_bytes), int(plan.fluid_updates_per_iteration) * req.steps
    finally:
        plan.close()


@dataclass
class Server:
    """`hbm_budget` bytes of device memory for resident domains, at most
    `max_slots` of them, stepped in chunks of up to `chunk_steps`; grids are
    built by `builders` host threads."""
    hbm_budget: int
    max_slots: int = 16
    chunk_steps: int = 100
    keep_fields: bool = False
    builders: int = 2
    pack: bool = True           # packed batches (False: every domain on its own stream)
    results: list = field(default_factory=list)
    _batches: dict = field(default_factory=dict)   # storage -> (member rids, PackedBatch)

    def _close_batches(self, rids=None):
        """Close the packed batches holding any of `rids` (all with None)."""
        for st in list(self._batches):
            key, b = self._batches[st]
            if rids is None or any(r in key for r in rids):
                b.close()
                del self._batches[st]

    def _advance(self, ready, chunk):
        groups, loose = {}, []
        for a in ready:
            (groups.setdefault(a.req.case.storage, []) if self.pack and a.packable else loose).append(a)
        for st, members in groups.items():
            # a lone domain is a batch of one: the same kernel alone or in the mix
            key = tuple(a.req.rid for a in members)
            if st not in self._batches or self._batches[st][0] != key:
                self._close_batches([r for r in (self._batches.get(st) or ((), None))[0]])
                self._batches[st] = (key, PackedBatch([a.grids for a in members]))
            self._batches[st][1].update(chunk)
        if loose:
            update_batch([a.grids for a in loose], chunk)

    def run(self, requests) -> list:
        import torch
        pending = sorted(requests, key=lambda r: r.arrival)
        device = torch.cuda.current_device()
        active: list[_Active] = []
        used = 0
        pool = ThreadPoolExecutor(max_workers=max(1, self.builders))

        def build(case):
            torch.cuda.set_device(device)
            return Grids(case)

        t0 = time.perf_counter()
        try:
            while pending or active:
                now = time.perf_counter() - t0
                # admission: arrived, a free slot, and the footprint fits
                while pending and pending[0].arrival <= now and len(active) < self.max_slots:
                    req = pending[0]
                    footprint, updates = _footprint(req)
                    if footprint > self.hbm_budget:
                        raise ValueError(f"request {req.rid} needs {footprint} bytes, more than the whole budget")
                    if used + footprint > self.hbm_budget:
                        break
                    pending.pop(0)
                    active.append(_Active(req, None, None, req.steps, footprint, time.perf_counter() - t0,
                                          updates, pool.submit(build, req.case)))
                    used += footprint
                # domains whose build finished join the stepping set
                for a in active:
                    if a.build is not None and a.build.done():
                        a.grids = a.build.result()
                        a.build = None
                        a.stream = torch.cuda.Stream()
                        a.grids.set_stream(a.stream.cuda_stream)
                        a.packable = _packable(a.grids)
                        # join the packed batch of its storage type at the batch's parity
                        mates = [b for b in active if b is not a and b.grids is not None and b.packable
                                 and b.req.case.storage == a.req.case.storage and b.remaining > 0]
                        if self.pack and a.packable and mates and mates[0].parity != a.parity:
                            with PackedBatch([a.grids]) as own:
                                own.update(1)
                            a.remaining -= 1
                ready = [a for a in active if a.grids is not None and a.remaining > 0]
                finished = any(a.grids is not None and a.remaining == 0 for a in active)
                if not ready and not finished:
                    # idle until the next arrival or build completion
                    wait = 0.002 if active else max(0.0, pending[0].arrival - (time.perf_counter() - t0))
                    time.sleep(min(0.01, wait))
                    continue
                if ready:
                    chunk = min(self.chunk_steps, min(a.remaining for a in ready))
                    self._advance(ready, chunk)
                    for a in ready:
                        a.remaining -= chunk
                done = [a for a in active if a.grids is not None and a.remaining == 0]
                if done:
                    self._close_batches([a.req.rid for a in done])
                for a in done:
                    g = a.grids
                    g.synchronize()
                    res = Result(a.req.rid, a.req.steps, a.updates, a.admitted, 0.0, a.req.arrival)
                    if a.req.wall_id >= 0:
                        res.force = g.wall_force(a.req.wall_id)
                    else:
                        res.energy = g.kinetic_energy(*a.req.energy_ref)
                    if self.keep_fields:
                        res.macro = g.macro()
                    res.finished = time.perf_counter() - t0
                    g.close()
                    a.grids = None
                    used -= a.footprint
                    self.results.append(res)
                active = [a for a in active if a.remaining > 0]
        finally:
            # on an error, release everything admitted so far
            self._close_batches()
            for a in active:
                if a.build is not None:
                    try:
                        a.grids = a.build.result()
                    except Exception:
                        a.grids = None
                if a.grids is not None:
                    a.grids.close()
            pool.shutdown(wait=True)
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
