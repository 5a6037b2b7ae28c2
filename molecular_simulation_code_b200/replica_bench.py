"""Throughput and latency of batched replicas and of the segment server.

batch:  64 seeded replicas, N ~ U[3,000, 30,000] atoms, glycine 5-20 % of
        molecules, own cubic box at 1.0 g/cm^3; 100-step segments (one graph
        launch per kernel and step for all replicas); cluster shape and prune
        margin autotuned per size class (--tune); mixed and FP64 atom-steps/s.
serve:  Poisson request stream (default 200 requests/s), systems of
        N ~ U[2,000, 60,000] atoms, U[500, 5,000] steps (times --steps-scale),
        every 4th with a crystalline glycine nucleus, up to 64 concurrent
        replicas, largest-cluster analysis on the device at the end of every
        segment; p50/p99 segment latency and replica-steps/s, mixed and FP64.

Prints one JSON line per mode:
    python -m molecular_simulation_code_b200.replica_bench --mode batch|serve
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def bench_batch(args):
    import torch

    from . import mixed as M
    from .batch import Batch, Tuner, apply_shape, make_replicas, size_class
    from .nonbond import Context

    reps = make_replicas(args.replicas, seed=args.seed, n_min=3000, n_max=30000,
                         processes=args.procs)
    master = Context(0)
    out = {"mode": "batch", "replicas": len(reps),
           "atoms_total": int(sum(r.np_atoms for r in reps)),
           "atoms_min": int(min(r.np_atoms for r in reps)),
           "atoms_max": int(max(r.np_atoms for r in reps)), "segment_steps": args.segment}
    tuner = Tuner()
    if args.tune:
        for r in reps:
            tuner.shape_for(master, r, steps=30)
        out["tuned_shape_per_class"] = {str(k): {"aspect": v[0], "margin": v[1]}
                                        for k, v in tuner.choice.items()}
    stream = torch.cuda.ExternalStream(master._lib.sofia_stream(master.handle))
    for name, prec in (("mixed", M.MIXED), ("fp64", M.FP64)):
        ctxs = [Context(0) for _ in reps]
        systems = []
        for c, r in zip(ctxs, reps):
            m = M.System(c, r, precision=prec)
            if args.tune:
                apply_shape(m, tuner.choice[size_class(r.np_atoms)])
            m.set_state(r.xyz.astype(np.float64), r.velocity.astype(np.float64))
            m.md_setup(r, dt=1.0, gamma=0.02, seed=7)
            systems.append(m)
        # the same preparation as the single-system benchmark: damped relaxation from
        # the lattice start (100 x 1 fs), 300 K equilibration with strong coupling
        # (400 x 2 fs), then the production coupling (gamma = 1/ps)
        stages = ((1.0, 0.02, 100, 7), (2.0, 0.02, 400, 8), (2.0, 0.001, args.segment, 9))
        for k, (dt, gamma, nsteps, seed) in enumerate(stages):
            for m, r in zip(systems, reps):
                m.md_setup(r, dt=dt, gamma=gamma, seed=seed)
            b = Batch(master, systems)
            b.set_segment(args.segment)  # steps per captured segment graph
            b.run(nsteps)  # the last stage is the warm-up segment (captures the graphs)
            if k < len(stages) - 1:
                b.close()
        torch.cuda.synchronize()
        st0 = [m.stats() for m in systems]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(f"batch_timed_{name}")  # lets ncu select the timed steps
        e0.record(stream)
        for _ in range(args.segments):
            en = b.run(args.segment, energy_every=args.segment)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        steps = args.segments * args.segment
        st1 = [m.stats() for m in systems]
        rsteps = len(reps) * steps
        out[name] = {"atom_steps_per_s": out["atoms_total"] * steps / t,
                     "replica_steps_per_s": rsteps / t,
                     "ms_per_batch_step": 1e3 * t / steps,
                     "temperature_K_mean": float(np.mean([e["temperature"] for e in en])),
                     "list_builds_per_replica_step":
                         sum(b1["builds"] - b0["builds"] for b0, b1 in zip(st0, st1)) / rsteps,
                     "prunes_per_replica_step":
                         sum(b1["prunes"] - b0["prunes"] for b0, b1 in zip(st0, st1)) / rsteps}
        b.close()
        for m in systems:
            m.close()
        for c in ctxs:
            c.close()
    out["mixed_over_fp64"] = out["mixed"]["atom_steps_per_s"] / out["fp64"]["atom_steps_per_s"]
    return out


def bench_serve(args):
    from . import mixed as M
    from .batch import make_replicas
    from .serve import Request, Server, poisson_arrivals, run_stream

    rng = np.random.default_rng(args.seed)
    systems = make_replicas(args.requests, seed=args.seed + 1, n_min=2000, n_max=60000,
                            processes=args.procs, nucleus_every=args.nucleus_every)
    arrivals = poisson_arrivals(args.rate, args.requests, seed=args.seed + 2)
    steps = (rng.integers(500, 5001, size=args.requests) * args.steps_scale).astype(int)
    steps = np.maximum(steps // args.chunk, 1) * args.chunk
    out = {"mode": "serve", "requests": args.requests, "rate_per_s": args.rate,
           "steps_scale": args.steps_scale, "max_active": args.max_active,
           "atoms_range": [int(min(s.np_atoms for s in systems)),
                           int(max(s.np_atoms for s in systems))]}
    for name, prec in (("mixed", M.MIXED), ("fp64", M.FP64)):
        srv = Server(max_active=args.max_active, hbm_budget=int(args.budget_gb * (1 << 30)),
                     chunk_steps=args.chunk, precision=prec)
        reqs = [Request(k, float(arrivals[k]), systems[k], int(steps[k]))
                for k in range(args.requests)]
        stats = run_stream(srv, reqs)
        per_step = np.array([r.service / r.nsteps for r in srv.results])
        stats["per_step_service_p50_ms"] = float(np.percentile(per_step, 50) * 1e3)
        stats["per_step_service_p99_ms"] = float(np.percentile(per_step, 99) * 1e3)
        stats["segment_latency_p99_over_p50"] = (stats["segment_latency_p99_s"] /
                                                 stats["segment_latency_p50_s"])
        seeded = [r for r in srv.results if args.nucleus_every and r.rid % args.nucleus_every == 0]
        stats["cluster_sizes_seeded"] = sorted(int(r.cluster_size) for r in seeded)
        stats["cluster_sizes_top5_other"] = sorted(int(r.cluster_size) for r in srv.results
                                                   if r not in seeded)[-5:]
        stats["batch_graph_captures"] = srv.recaptures
        stats["cluster_criterion"] = {"mrcut_A": srv.mrcut, "denscut_A": srv.denscut,
                                      "densmin": srv.densmin}
        out[name] = stats
        srv.close()
    out["mixed_over_fp64_replica_steps"] = (out["mixed"]["replica_steps_per_s"] /
                                            out["fp64"]["replica_steps_per_s"])
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=["batch", "serve"], default="batch")
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--segment", type=int, default=100)
    ap.add_argument("--segments", type=int, default=3)
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--requests", type=int, default=128)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--steps-scale", type=float, default=1.0)
    ap.add_argument("--nucleus-every", type=int, default=4,
                    help="every k-th request starts with a crystalline glycine nucleus")
    ap.add_argument("--chunk", type=int, default=100)
    ap.add_argument("--max-active", type=int, default=64)
    ap.add_argument("--budget-gb", type=float, default=64.0)
    ap.add_argument("--seed", type=int, default=5000)
    ap.add_argument("--procs", type=int, default=min(16, os.cpu_count() or 1))
    args = ap.parse_args(argv)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    t0 = time.time()
    out = bench_batch(args) if args.mode == "batch" else bench_serve(args)
    out["wall_s"] = time.time() - t0
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
