"""Batches of independent replicas and the per-size-class autotuner.

A ``Batch`` groups device-resident systems and advances all of them together
(``sofia_batch_md_run``): each kernel of a step runs once for every replica,
and steps run as captured graphs of ``seg`` steps.  Members can change between
runs (``set_systems``) without a graph recapture.  Replicas never exchange data, so each replica's
trajectory is bit-identical to the same replica run alone.

``autotune`` times short MD segments of one replica per candidate shape --
the cluster geometry (the xy column width relative to the cube side of 8
atoms, i.e. how tall the 8-atom clusters are) and the prune margin of the
inner list -- and keeps the fastest for the replica's size class; ``Tuner``
caches the choice per class, so every replica of that class uses it (in a
batch every replica keeps its own shape: the batched kernels read each
replica's geometry from the device table).
"""
from __future__ import annotations

import ctypes as C
import multiprocessing as mp
import time

import numpy as np

from ._lib import SOFIA_MD_NE, MD_ENERGY_NAMES
from . import mixed as M
from .nonbond import Context
from .system import random_replica

SIZE_CLASSES = [(0, 6000), (6000, 12000), (12000, 24000), (24000, 48000), (48000, 1 << 30)]
MARGINS = (0.3, 0.5, 0.8, 1.2)
ASPECTS = (0.8, 1.0, 1.25)


def size_class(n: int) -> int:
    for k, (lo, hi) in enumerate(SIZE_CLASSES):
        if lo <= n < hi:
            return k
    return len(SIZE_CLASSES) - 1


class Batch:
    def __init__(self, ctx: Context, systems: list):
        self.ctx = ctx
        self.systems = list(systems)
        arr = (C.c_void_p * len(self.systems))(*[s.handle.value for s in self.systems])
        h = C.c_void_p()
        ctx.check(ctx._lib.sofia_batch_create(ctx.handle, arr, len(self.systems), C.byref(h)))
        self.handle = h
        ctx.adopt(self)

    close_rank = 0  # a batch is destroyed before the systems it steps

    def run(self, nsteps: int, energy_every: int = 0):
        e = np.zeros((len(self.systems), SOFIA_MD_NE))
        self.ctx.check(self.ctx._lib.sofia_batch_md_run(self.handle, int(nsteps),
                                                        int(energy_every), e.ctypes.data))
        if energy_every <= 0:
            return None
        return [dict(zip(MD_ENERGY_NAMES, row.tolist())) for row in e]

    def set_systems(self, systems: list):
        """New members for the next run (continuous batching, no graph recapture)."""
        arr = (C.c_void_p * len(systems))(*[s.handle.value for s in systems])
        self.ctx.check(self.ctx._lib.sofia_batch_set_systems(self.handle, arr, len(systems)))
        self.systems = list(systems)

    def set_segment(self, steps: int):
        """Steps per captured graph (default 100)."""
        self.ctx.check(self.ctx._lib.sofia_batch_set_segment(self.handle, int(steps)))

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.sofia_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_margin(system: M.System, margin: float):
    system.ctx.check(system.ctx._lib.sofia_system_set_margin(system.handle, float(margin)))


def set_cluster_shape(system: M.System, aspect: float):
    system.ctx.check(system.ctx._lib.sofia_system_set_cluster_shape(system.handle,
                                                                   float(aspect)))


def apply_shape(system: M.System, shape):
    """shape = (aspect, margin) as chosen by the tuner."""
    set_cluster_shape(system, shape[0])
    set_margin(system, shape[1])


def autotune(ctx: Context, sysdata, aspects=ASPECTS, margins=(0.35, 0.45, 0.6), steps: int = 40,
             cut: float = 10.0, skin: float = 2.0, precision: int = M.MIXED):
    """Fastest (cluster aspect, prune margin) for this replica: short Langevin
    segments timed with CUDA events, every candidate from the same 300 K state
    (damped relaxation from the lattice start, then strong-coupling 2 fs steps,
    as the benchmarks prepare their systems)."""
    import torch
    stream = torch.cuda.ExternalStream(ctx._lib.sofia_stream(ctx.handle))
    base = M.System(ctx, sysdata, cut=cut, skin=skin, precision=precision)
    base.set_state(sysdata.xyz.astype(np.float64), sysdata.velocity.astype(np.float64))
    base.md_setup(sysdata, dt=1.0, gamma=0.02, seed=1)
    base.md_run(100)
    base.md_setup(sysdata, dt=2.0, gamma=0.02, seed=3)
    base.md_run(200)
    x, v, _ = base.get_state()
    base.close()
    times = {}
    for a in aspects:
        for mg in margins:
            m = M.System(ctx, sysdata, cut=cut, skin=skin, precision=precision)
            try:
                set_cluster_shape(m, a)
            except Exception:
                m.close()
                continue  # the box is too small for that column grid
            set_margin(m, mg)
            m.set_state(x, v)
            m.md_setup(sysdata, dt=2.0, gamma=0.001, seed=2)
            m.md_run(10)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            m.md_run(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            times[(a, mg)] = e0.elapsed_time(e1) / steps
            m.close()
    best = min(times, key=times.get)
    return best, times


def autotune_margin(ctx: Context, sysdata, margins=MARGINS, steps: int = 60, cut: float = 10.0,
                    skin: float = 2.0, precision: int = M.MIXED) -> tuple[float, dict]:
    """Fastest prune margin for this replica (short Langevin segments, CUDA events)."""
    import torch
    stream = torch.cuda.ExternalStream(ctx._lib.sofia_stream(ctx.handle))
    times = {}
    for mg in margins:
        m = M.System(ctx, sysdata, cut=cut, skin=skin, precision=precision)
        set_margin(m, mg)
        m.set_state(sysdata.xyz.astype(np.float64), sysdata.velocity.astype(np.float64))
        m.md_setup(sysdata, dt=1.0, gamma=0.02, seed=1)
        m.md_run(20)
        m.md_setup(sysdata, dt=2.0, gamma=0.001, seed=2)
        m.md_run(5)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.md_run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        times[mg] = e0.elapsed_time(e1) / steps
        m.close()
    best = min(times, key=times.get)
    return best, times


class Tuner:
    """Per-size-class (cluster aspect, prune margin) choices, filled lazily by
    ``autotune`` on the first replica of each class."""

    def __init__(self):
        self.choice: dict[int, tuple] = {}
        self.timings: dict[int, dict] = {}

    def shape_for(self, ctx: Context, sysdata, **kw) -> tuple:
        k = size_class(sysdata.np_atoms)
        if k not in self.choice:
            best, t = autotune(ctx, sysdata, **kw)
            self.choice[k] = best
            self.timings[k] = t
        return self.choice[k]

    def margin_for(self, ctx: Context, sysdata, **kw) -> float:
        return self.shape_for(ctx, sysdata, **kw)[1]


def _gen(args):
    seed, n_min, n_max, nucleus = args
    rng = np.random.default_rng(seed)
    return random_replica(rng, n_min, n_max, seed=seed, nucleus=nucleus)


def make_replicas(n: int, seed: int = 4000, n_min: int = 3000, n_max: int = 30000,
                  processes: int = 8, nucleus_every: int = 0, nucleus: int = 60):
    """Seeded replicas of N ~ U[n_min, n_max] atoms (generated in a spawn pool).
    Every ``nucleus_every``-th replica (0 = none) starts with a compact crystalline
    glycine nucleus of up to ``nucleus`` molecules (5.5 A fcc)."""
    args = [(seed + k, n_min, n_max,
             nucleus if nucleus_every and k % nucleus_every == 0 else 0) for k in range(n)]
    if processes <= 1 or n <= 2:
        return [_gen(a) for a in args]
    with mp.get_context("spawn").Pool(processes) as pool:
        return pool.map(_gen, args)


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
