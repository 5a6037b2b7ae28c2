"""Continuous-batching segment server for nucleation-style trajectory requests.

The reference's hybrid-MC nucleation move (Source/mod_nucleation.f90:300-570)
runs a segment of MD steps, analyses the largest solid-glycine cluster
(Source/mod_cluster.f90:15-83) and continues or rolls back.  This server
runs many such segments at once on one GPU:

* requests (a seeded glycine/water system, a step count, optionally the id
  of an earlier request to continue) queue FIFO;
* admission: up to ``max_active`` replicas run at once, and a request is
  admitted only while the estimated device memory of everything resident
  (running + parked) stays within ``hbm_budget`` bytes; parked states are
  evicted least-recently-used when room is needed;
* every chunk of ``chunk_steps`` steps advances all running replicas with one
  graph launch per step (``Batch``); requests that arrived meanwhile are
  admitted at the next chunk boundary (continuous batching);
* a finished segment ends with the largest-cluster analysis on the device;
  its state (positions, velocities, neighbour list, RNG step counter) stays
  resident so a continuation request resumes it without a host round trip.

Results do not depend on what else is in the batch (replicas never exchange
data and every force sum is in fixed point), which ``tests`` check.
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np

from . import mixed as M
from .batch import Batch, Tuner, set_margin
from .nonbond import Context, get_greatest_cluster

BYTES_PER_ATOM = 1200      # resident state + lists + records, measured order of magnitude
FIXED_BYTES = 8 << 20      # per-replica constant overhead (contexts, staging, reductions)


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float            # seconds (server clock)
    sysdata: object           # SofiaSystem
    nsteps: int
    continues: int | None = None  # rid of a finished request whose state to resume


@dataclasses.dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    nsteps: int
    atoms: int
    cluster_size: int
    energies: dict | None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def service(self) -> float:
        return self.finished - self.admitted


class _Replica:
    def __init__(self, req: Request, ctx: Context, system: M.System, now: float):
        self.req = req
        self.ctx = ctx
        self.system = system
        self.remaining = req.nsteps
        self.admitted = now
        s = req.sysdata
        self.ptta = s.xyz[:10 * s.n_gly].astype(np.float64).copy()
        self.greatest = 0
        self.last_used = now


def estimate_bytes(n_atoms: int) -> int:
    return FIXED_BYTES + BYTES_PER_ATOM * int(n_atoms)


class Server:
    def __init__(self, device: int = 0, max_active: int = 64, hbm_budget: int = 32 << 30,
                 chunk_steps: int = 100, precision: int = M.MIXED, tune: bool = False,
                 cut: float = 10.0, skin: float = 2.0, dt: float = 2.0,
                 temperature: float = 300.0, gamma: float = 0.001,
                 cluster=(9.0, 5.0, 11), warm_in: int = 50):
        self.device = device
        self.ctx = Context(device)
        self.max_active = max_active
        self.hbm_budget = hbm_budget
        self.chunk_steps = chunk_steps
        self.precision = precision
        self.cut, self.skin, self.dt = cut, skin, dt
        self.temperature, self.gamma = temperature, gamma
        self.mrcut, self.denscut, self.densmin = cluster
        self.warm_in = warm_in
        self.tuner = Tuner() if tune else None
        self.queue: collections.deque[Request] = collections.deque()
        self.active: list[_Replica] = []
        self.parked: collections.OrderedDict[int, _Replica] = collections.OrderedDict()
        self.results: list[Result] = []
        self.batch = None
        self.batch_members: tuple = ()
        self.t0 = time.perf_counter()
        self.atom_steps = 0
        self.replica_steps = 0

    # -- clock and memory -------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def resident_bytes(self) -> int:
        return sum(estimate_bytes(r.req.sysdata.np_atoms) for r in self.active) + \
            sum(estimate_bytes(r.req.sysdata.np_atoms) for r in self.parked.values())

    # -- admission ----------------------------------------------------------
    def submit(self, req: Request):
        self.queue.append(req)

    def _new_replica(self, req: Request) -> _Replica:
        s = req.sysdata
        ctx = Context(self.device)
        m = M.System(ctx, s, cut=self.cut, skin=self.skin, precision=self.precision)
        if self.tuner is not None:
            set_margin(m, self.tuner.margin_for(ctx, s, cut=self.cut, skin=self.skin,
                                                precision=self.precision))
        m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
        if self.warm_in:
            # damped warm-in from a lattice start (part of the request's service time)
            m.md_setup(s, dt=1.0, temperature=self.temperature, gamma=0.02,
                       seed=7 * (req.rid + 1))
            m.md_run(self.warm_in)
        m.md_setup(s, dt=self.dt, temperature=self.temperature, gamma=self.gamma,
                   seed=1000003 * (req.rid + 1))
        return _Replica(req, ctx, m, self.now())

    def _admit(self):
        while self.queue and len(self.active) < self.max_active:
            req = self.queue[0]
            if req.continues is not None and req.continues in self.parked:
                rep = self.parked.pop(req.continues)
                rep.req = dataclasses.replace(req, sysdata=rep.req.sysdata)
                rep.remaining = req.nsteps
                rep.admitted = self.now()
                self.queue.popleft()
                self.active.append(rep)
                continue
            need = estimate_bytes(req.sysdata.np_atoms)
            while self.resident_bytes() + need > self.hbm_budget and self.parked:
                _, old = self.parked.popitem(last=False)  # evict least recently used
                old.system.close()
                old.ctx.close()
            if self.resident_bytes() + need > self.hbm_budget:
                break  # wait for running replicas to finish
            self.queue.popleft()
            self.active.append(self._new_replica(req))

    # -- one chunk ----------------------------------------------------------
    def step_chunk(self) -> int:
        self._admit()
        if not self.active:
            return 0
        members = tuple(id(r) for r in self.active)
        if members != self.batch_members:
            if self.batch is not None:
                self.batch.close()
            self.batch = Batch(self.ctx, [r.system for r in self.active])
            self.batch_members = members
        k = min(self.chunk_steps, min(r.remaining for r in self.active))
        want_e = any(r.remaining == k for r in self.active)
        energies = self.batch.run(k, energy_every=k if want_e else 0)
        for r in self.active:
            r.remaining -= k
            self.atom_steps += k * r.req.sysdata.np_atoms
            self.replica_steps += k
        done = [i for i, r in enumerate(self.active) if r.remaining == 0]
        for i in reversed(done):
            r = self.active.pop(i)
            size = self._cluster(r)
            now = self.now()
            self.results.append(Result(r.req.rid, r.req.arrival, r.admitted, now, r.req.nsteps,
                                       r.req.sysdata.np_atoms, size,
                                       energies[i] if energies else None))
            r.last_used = now
            self.parked[r.req.rid] = r
        return k

    def _cluster(self, r: _Replica) -> int:
        s = r.req.sysdata
        if s.n_gly == 0:
            return 0
        x, _, _ = r.system.get_state()
        L = float(s.box)
        xw = np.mod(x, L).astype(np.float32)
        xw[xw <= 0] += np.float32(L)
        pos = s.position_aos()
        pos[:, :3] = xw
        gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
        size, g, _, _ = get_greatest_cluster(r.ctx, pos, gid, s.n_gly, 10, s.box, self.mrcut,
                                             self.denscut, self.densmin, r.ptta, r.greatest)
        r.greatest = g
        return size

    def drain(self):
        while self.queue or self.active:
            if self.step_chunk() == 0 and not self.active:
                break

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for r in self.active + list(self.parked.values()):
            r.system.close()
            r.ctx.close()
        self.active.clear()
        self.parked.clear()


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def run_stream(server: Server, requests: list[Request]) -> dict:
    """Feed requests at their arrival times (server clock) and serve to completion."""
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    server.t0 = time.perf_counter()
    while pending or server.queue or server.active:
        now = server.now()
        while pending and pending[0].arrival <= now:
            server.submit(pending.popleft())
        if not server.active and not server.queue and pending:
            time.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
            continue
        server.step_chunk()
    wall = server.now()
    lat = np.array([r.latency for r in server.results])
    svc = np.array([r.service for r in server.results])
    return {"requests": len(server.results), "wall_s": wall,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "service_p50_s": float(np.percentile(svc, 50)),
            "service_p99_s": float(np.percentile(svc, 99)),
            "replica_steps_per_s": server.replica_steps / wall,
            "atom_steps_per_s": server.atom_steps / wall}
