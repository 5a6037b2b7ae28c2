"""Continuous-batching segment server for nucleation-style trajectory requests.

The reference's hybrid-MC nucleation move (Source/mod_nucleation.f90:300-570)
runs a segment of MD steps, analyses the largest solid-glycine cluster
(Source/mod_cluster.f90:15-83) and continues or rolls back.  This server
runs many such segments at once on one GPU:

* requests (a seeded glycine/water system, a step count, optionally the id
  of an earlier request to continue) queue FIFO;
* admission: up to ``max_active`` replicas run at once, and a request is
  admitted only while the device memory of everything resident (running +
  parked) stays within ``hbm_budget`` bytes.  Resident systems count what they
  actually hold (``System.device_bytes``, which grows with their lists); a new
  request is charged the largest bytes-per-atom seen so far until it exists.
  Parked states are evicted least-recently-used when room is needed;
* all running replicas advance together in one ``Batch`` (every kernel of a
  step once for all of them, captured segment graphs); requests that arrive
  meanwhile join at the next chunk boundary and finished ones leave, by
  changing the batch's members without a graph recapture (continuous
  batching);
* a new replica's damped warm-in from its lattice start runs inside the batch
  (1 fs steps, strong friction) instead of blocking the running replicas;
* a finished segment ends with the largest-cluster analysis on the device-
  resident positions (no host copy of them); its state (positions,
  velocities, neighbour list, RNG step counter, the analysis's reference
  positions) stays resident so a continuation request resumes it.

Results do not depend on what else is in the batch (replicas never exchange
data and every force sum is in fixed point), which ``tests`` check.
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np

from . import mixed as M
from .batch import Batch, Tuner, apply_shape
from .nonbond import Context

BYTES_PER_ATOM = 1200      # charge per atom of a request before any system exists
FIXED_BYTES = 8 << 20      # per-replica constant overhead (context, staging, reductions)
# largest-cluster criterion of the reference's run input (mrcut, denscut, densmin):
# input_files/input:41
REFERENCE_CLUSTER = (9.0, 6.0, 11)


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
        """Segment latency: arrival to the end of the segment's cluster analysis."""
        return self.finished - self.arrival

    @property
    def service(self) -> float:
        return self.finished - self.admitted


class _Replica:
    def __init__(self, req: Request, ctx: Context, system: M.System, now: float, warm: int):
        self.req = req
        self.ctx = ctx
        self.system = system
        self.warm = warm            # warm-in steps left (run before the segment's steps)
        self.remaining = req.nsteps
        self.admitted = now
        self.greatest = 0
        self.last_used = now
        self.bytes = system.device_bytes()

    def to_event(self) -> int:
        return self.warm if self.warm > 0 else self.remaining


def estimate_bytes(n_atoms: int, bytes_per_atom: float = BYTES_PER_ATOM) -> int:
    return FIXED_BYTES + int(bytes_per_atom * int(n_atoms))


class Server:
    def __init__(self, device: int = 0, max_active: int = 64, hbm_budget: int = 32 << 30,
                 chunk_steps: int = 100, precision: int = M.MIXED, tune: bool = False,
                 cut: float = 10.0, skin: float = 2.0, dt: float = 2.0,
                 temperature: float = 300.0, gamma: float = 0.001,
                 cluster=REFERENCE_CLUSTER, warm_in: int = 50, segment_graph: int = 50):
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
        self.segment_graph = segment_graph
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
        self.bytes_per_atom = float(BYTES_PER_ATOM)
        self.recaptures = 0

    # -- clock and memory -------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def resident_bytes(self) -> int:
        return sum(FIXED_BYTES + r.bytes for r in self.active) + \
            sum(FIXED_BYTES + r.bytes for r in self.parked.values())

    # -- admission ----------------------------------------------------------
    def submit(self, req: Request):
        self.queue.append(req)

    def _new_replica(self, req: Request) -> _Replica:
        s = req.sysdata
        ctx = Context(self.device)
        m = M.System(ctx, s, cut=self.cut, skin=self.skin, precision=self.precision)
        if self.tuner is not None:
            apply_shape(m, self.tuner.shape_for(ctx, s, cut=self.cut, skin=self.skin,
                                                precision=self.precision))
        m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
        if self.warm_in:
            # damped warm-in from a lattice start, run inside the batch (part of the
            # request's service time)
            m.md_setup(s, dt=1.0, temperature=self.temperature, gamma=0.02,
                       seed=7 * (req.rid + 1))
        else:
            self._production(m, req)
        rep = _Replica(req, ctx, m, self.now(), self.warm_in)
        self.bytes_per_atom = max(self.bytes_per_atom, rep.bytes / s.np_atoms)
        return rep

    def _production(self, m: M.System, req: Request):
        m.md_setup(req.sysdata, dt=self.dt, temperature=self.temperature, gamma=self.gamma,
                   seed=1000003 * (req.rid + 1))

    def _admit(self):
        while self.queue and len(self.active) < self.max_active:
            req = self.queue[0]
            if req.continues is not None and req.continues in self.parked:
                rep = self.parked.pop(req.continues)
                rep.req = dataclasses.replace(req, sysdata=rep.req.sysdata)
                rep.remaining = req.nsteps
                rep.warm = 0
                rep.admitted = self.now()
                self.queue.popleft()
                self.active.append(rep)
                continue
            need = estimate_bytes(req.sysdata.np_atoms, self.bytes_per_atom)
            while self.resident_bytes() + need > self.hbm_budget and self.parked:
                _, old = self.parked.popitem(last=False)  # evict least recently used
                old.system.close()
                old.ctx.close()
            if self.resident_bytes() + need > self.hbm_budget and self.active:
                break  # wait for running replicas to finish (a lone request always runs)
            self.queue.popleft()
            self.active.append(self._new_replica(req))

    # -- one chunk ----------------------------------------------------------
    def _sync_batch(self):
        members = tuple(id(r) for r in self.active)
        if members == self.batch_members:
            return
        systems = [r.system for r in self.active]
        if self.batch is None:
            self.batch = Batch(self.ctx, systems)
            self.batch.set_segment(self.segment_graph)
            self.recaptures += 1
        else:
            self.batch.set_systems(systems)
        self.batch_members = members

    def step_chunk(self) -> int:
        self._admit()
        if not self.active:
            return 0
        self._sync_batch()
        k = min(self.chunk_steps, min(r.to_event() for r in self.active))
        want_e = any(r.warm == 0 and r.remaining == k for r in self.active)
        energies = self.batch.run(k, energy_every=k if want_e else 0)
        finished = []
        for i, r in enumerate(self.active):
            r.bytes = r.system.device_bytes()  # lists may have grown
            self.bytes_per_atom = max(self.bytes_per_atom, r.bytes / r.req.sysdata.np_atoms)
            self.atom_steps += k * r.req.sysdata.np_atoms
            self.replica_steps += k
            if r.warm > 0:
                r.warm -= k
                if r.warm == 0:
                    self._production(r.system, r.req)
                continue
            r.remaining -= k
            if r.remaining == 0:
                finished.append(i)
        for i in reversed(finished):
            r = self.active.pop(i)
            size = self._cluster(r)
            now = self.now()
            self.results.append(Result(r.req.rid, r.req.arrival, r.admitted, now, r.req.nsteps,
                                       r.req.sysdata.np_atoms, size,
                                       energies[i] if energies else None))
            r.last_used = now
            r.bytes = r.system.device_bytes()
            self.parked[r.req.rid] = r
        return k

    def _cluster(self, r: _Replica) -> int:
        s = r.req.sysdata
        if s.n_gly == 0:
            return 0
        size, g = r.system.greatest_cluster(s.n_gly, self.mrcut, self.denscut, self.densmin,
                                            greatest=r.greatest)
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
            "segment_latency_p50_s": float(np.percentile(lat, 50)),
            "segment_latency_p99_s": float(np.percentile(lat, 99)),
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "service_p50_s": float(np.percentile(svc, 50)),
            "service_p99_s": float(np.percentile(svc, 99)),
            "replica_steps_per_s": server.replica_steps / wall,
            "atom_steps_per_s": server.atom_steps / wall}
