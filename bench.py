#!/usr/bin/env python
"""Throughput of the Sofia nonbonded hot path on B200 (atom-steps/s).

Workload (default): the 275,000-atom glycine/water system (3,500 glycine +
80,000 SPC/E water, 1.0 g/cm^3, L = 14.1 nm), rc = 10 A, skin 2 A, DSF
alpha = 0.2 A^-1, seeded synthetic coordinates, 2 fs steps, Langevin 300 K
with gamma = 1/ps, SHAKE on X-H bonds and rigid water.

value: device-resident MD atom-steps/s of the mixed path (FP64 positions,
FP32 pair arithmetic, 64-bit fixed-point forces): each step is velocity
Verlet + Langevin + SHAKE + bonded/1-4 terms + the nonbonded hot path
(displacement check, list rebuild/prune on trigger, LJ + DSF forces), the
steps captured as one CUDA graph, energies on the last step of the timed
segment; max over ranks (replicas only, no exchange).
e2e: the reference-facing drop-in call (sofia_force_nonbond_mixed) with
pinned host buffers: positions in, real*4 forces and energies out, every
step, on a ballistic trajectory.
Also reported: the plain FP64 variants (same MD in FP64, and the FP64
reference-semantics path), the nonbonded-only hot path, the roofline of the
pair kernel against a measured FP32 CUDA-core peak, and the CPU baseline
(oracle port, all host cores).

``--impl reference`` times the CPU restatement of the reference path
(oracle port, OpenMP over all host cores) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 2.0            # fs
RELAX_STEPS = 100   # untimed damped steps from the lattice start
EQUIL_STEPS = 400   # untimed 2 fs steps with strong Langevin coupling: brings the lattice start to 300 K
CUT = 10.0          # A
SKIN = 2.0          # A
ALPHA = 0.2         # 1/A
FLOP_PER_PAIR = 82  # algorithmic FLOP per unique pair within rc + skin


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gly3500_wat80000_275k")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--only-hot", action="store_true",
                    help="time only the nonbonded hot path (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the rows of the other configurations (9k, 90k, batch, serving)")
    ap.add_argument("--serve-requests", type=int, default=48)
    return ap.parse_args()


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as td
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, ws


def allreduce_max(v: float, ws: int, device=None) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as td
    t = torch.tensor([v], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as td
        td.barrier()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for k, n in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def count_pairs_within(s, rv: float) -> int:
    """Unique non-excluded atom pairs within rv (minimum image)."""
    from scipy.spatial import cKDTree
    L = float(s.box)
    x = np.mod(s.xyz.astype(np.float64), L)
    tree = cKDTree(x, boxsize=L)
    total = int(tree.count_neighbors(tree, rv) - s.np_atoms) // 2
    # excluded pairs (1-2/1-3/1-4) within rv are not listed
    cols = np.arange(12)[None, :] < s.num3bond[:, None]
    ii, ll = np.nonzero(cols)
    jj = s.specbond[ii, ll] - 1
    d = x[jj] - x[ii]
    d -= L * np.round(d / L)
    excl = int((np.einsum("ij,ij->i", d, d) < rv * rv).sum())
    return total - excl // 2


def measure_fp32_peak() -> float:
    """FP32 CUDA-core TFLOP/s from cuBLAS SGEMM with TF32 disabled (8192^3)."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def measured_hbm():
    """HBM copy bandwidth of this pool's B200s (GB/s) and where it came from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool)"


def read_profile_traffic():
    """Per-launch DRAM bytes of the pair kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_pair_mixed_275k.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def build_system(args, rank):
    from molecular_simulation_code_b200.system import make_workload
    return make_workload(args.workload, seed=1000 * 3 + rank)


def cpu_baseline(s, rebuild_interval: float):
    """Oracle port (OpenMP, all host threads): one list build + force evaluations,
    per-step cost = force + build / rebuild_interval."""
    from oracle import oracle as O
    p = O.params(ALPHA, s.box, CUT, CUT, SKIN)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    t0 = time.perf_counter()
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 1024, fast=True)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    nf = 2
    for _ in range(nf):
        O.force_dsf(p, pos, s.q, lj, s.ntypes, nl, nn, na, fast=True)
    t_force = (time.perf_counter() - t0) / nf
    per_step = t_force + t_build / max(rebuild_interval, 1.0)
    return {"value": s.np_atoms / per_step, "unit": "atom-steps/s", "cores": os.cpu_count(),
            "kind": "port",
            "sample": f"275k-atom workload: 1 reference list build ({t_build:.2f} s) + {nf} FP64 "
                      f"force evaluations ({t_force:.2f} s each); per step = force + build/"
                      f"{rebuild_interval:.1f} (the GPU run's rebuild interval)"}


def run_reference(args, rank, ws):
    """CPU restatement of the reference path (neighbor_wrapper on trigger +
    lj_cut_coul_dsf_nonewton), all host threads, same workload and metric."""
    from oracle import oracle as O
    if rank != 0:
        return
    s = build_system(args, 0)
    p = O.params(ALPHA, s.box, CUT, CUT, SKIN)
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    x0 = s.xyz.astype(np.float64)
    v = s.velocity.astype(np.float64)
    n = s.np_atoms
    pos = s.position_aos()
    # bounded sample: each step evaluates a prefix of the atom rows if a full step
    # would make the run longer than about three minutes
    t0 = time.perf_counter()
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 1024, fast=True)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.force_dsf(p, pos, s.q, lj, s.ntypes, nl, nn, na, fast=True)
    t_force = time.perf_counter() - t0
    budget = 180.0
    nsteps = args.steps + args.warmup
    frac = min(1.0, budget / (nsteps * (t_force + t_build / 10.0)))
    rows = max(1024, int(n * frac))
    import ctypes as C
    L = O.lib(fast=True)
    xref = x0.copy()
    half2 = (0.5 * SKIN) ** 2
    Lb = float(s.box)
    elapsed = 0.0
    builds = 0
    for k in range(nsteps):
        x = x0 + v * DT * (k + 1)
        posk = pos.copy()
        posk[:, :3] = np.mod(x, Lb).astype(np.float32)
        posk[:, :3][posk[:, :3] <= 0] += np.float32(Lb)
        t0 = time.perf_counter()
        d = x - xref
        d -= Lb * np.round(d / Lb)
        if (np.einsum("ij,ij->i", d, d) > half2).any():
            nl, nn, na = O.neighbor_wrapper(p, posk, s.specbond, s.num3bond, na, fast=True)
            xref = x.copy()
            builds += 1 if k >= args.warmup else 0
        ff = np.zeros(rows * 3, np.float32)
        pot = C.c_double()
        ec = C.c_double()
        L.orc_force_dsf_nonewton(C.byref(p), rows, posk, np.ascontiguousarray(s.q), lj[0], lj[1],
                                 lj[2], lj[3], s.ntypes, nl, nn, na, ff, C.byref(pot),
                                 C.byref(ec), np.zeros(3), None, 0)
        dt_ = time.perf_counter() - t0
        if k >= args.warmup:
            elapsed += dt_
    value = rows * args.steps / elapsed
    out = {"impl": "reference", "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.workload, "atoms": n, "rc_A": CUT, "skin_A": SKIN},
           "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": os.cpu_count(),
                            "kind": "port",
                            "sample": f"{rows} of {n} atom rows per step, {args.steps} steps, "
                                      f"{builds} list rebuilds (half-skin trigger)"},
           "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def md_rate(ctx, M, s, precision, nsteps, seed=11):
    """Device-resident MD atom-steps/s of one system: damped relaxation and 300 K
    equilibration (untimed), then nsteps in captured graphs with CUDA events."""
    import torch
    stream = torch.cuda.ExternalStream(ctx._lib.sofia_stream(ctx.handle))
    m = M.System(ctx, s, alpha=ALPHA, cut=CUT, skin=SKIN, precision=precision)
    m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    m.md_setup(s, dt=1.0, temperature=300.0, gamma=0.02, seed=seed)
    m.md_run(RELAX_STEPS)
    m.md_setup(s, dt=DT, temperature=300.0, gamma=0.02, seed=seed + 1)
    m.md_run(EQUIL_STEPS)
    m.md_setup(s, dt=DT, temperature=300.0, gamma=0.001, seed=seed + 2)
    m.md_run(10)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    en = m.md_run(nsteps, energy_every=nsteps, use_graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    x, v, _ = m.get_state()
    m.close()
    return {"atom_steps_per_s": s.np_atoms * nsteps / t, "ms_per_step": 1e3 * t / nsteps,
            "ns_per_day": DT * 1e-6 * nsteps / t * 86400.0, "steps": nsteps,
            "temperature_K": en["temperature"]}, x, v


def cpu_md_sample(s, nsteps):
    """Oracle port (OpenMP, all host threads) on a ballistic trajectory: neighbour
    rebuild on the half-skin trigger plus the FP64 force every step."""
    import ctypes as C
    from oracle import oracle as O
    p = O.params(ALPHA, s.box, CUT, CUT, SKIN)
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    x0 = s.xyz.astype(np.float64)
    v = s.velocity.astype(np.float64)
    pos = s.position_aos()
    Lb = float(s.box)
    L = O.lib(fast=True)
    xref = None
    nl = nn = None
    na = 1024
    half2 = (0.5 * SKIN) ** 2
    builds = 0
    t0 = time.perf_counter()
    for k in range(nsteps):
        x = x0 + v * DT * (k + 1)
        posk = pos.copy()
        posk[:, :3] = np.mod(x, Lb).astype(np.float32)
        posk[:, :3][posk[:, :3] <= 0] += np.float32(Lb)
        if xref is None:
            rebuild = True
        else:
            d = x - xref
            d -= Lb * np.round(d / Lb)
            rebuild = bool((np.einsum("ij,ij->i", d, d) > half2).any())
        if rebuild:
            nl, nn, na = O.neighbor_wrapper(p, posk, s.specbond, s.num3bond, na, fast=True)
            xref = x.copy()
            builds += 1
        ff = np.zeros(s.np_atoms * 3, np.float32)
        pot = C.c_double()
        ec = C.c_double()
        L.orc_force_dsf_nonewton(C.byref(p), s.np_atoms, posk, np.ascontiguousarray(s.q), lj[0],
                                 lj[1], lj[2], lj[3], s.ntypes, nl, nn, na, ff, C.byref(pot),
                                 C.byref(ec), np.zeros(3), None, 0)
    t = time.perf_counter() - t0
    return {"value": s.np_atoms * nsteps / t, "unit": "atom-steps/s", "cores": os.cpu_count(),
            "kind": "port", "steps": nsteps, "list_rebuilds": builds,
            "sample": f"{s.np_atoms} atoms, {nsteps} steps: reference list build on the half-skin "
                      "trigger + FP64 force every step, ballistic trajectory"}


def row_hash(nl, nn, na, chunk=4096):
    """Order-independent hash of each neighbour row (sum of a 64-bit mix of its ids),
    computed over blocks of rows to bound the host memory."""
    n = nn.shape[0]
    rows = nl.reshape(n, na)
    out = np.zeros(n, np.uint64)
    cols = np.arange(na)[None, :]
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        h = rows[a:b].astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        h ^= h >> np.uint64(29)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h[cols >= nn[a:b, None]] = 0
        out[a:b] = h.sum(axis=1, dtype=np.uint64)
    return out


def extra_rows(args, ctx, budget_s=420.0):
    """The other configurations' rows (9k, 90k, 64-replica batch, serving), each
    bounded in time; the MD rows use the same step and timing as ``value``."""
    import torch

    from molecular_simulation_code_b200 import mixed as M
    from molecular_simulation_code_b200 import nonbond as nb
    from molecular_simulation_code_b200.system import make_workload
    t_start = time.time()
    out = {}
    # config 1: 9,000 atoms
    s9 = make_workload("gly150_wat2500_9k", seed=1000)
    r_mixed, _, _ = md_rate(ctx, M, s9, M.MIXED, 1000)
    r_fp64, _, _ = md_rate(ctx, M, s9, M.FP64, 1000)
    cpu = cpu_md_sample(s9, 1000)
    out["cfg1_9k"] = {"atoms": s9.np_atoms, "mixed": r_mixed, "fp64": r_fp64,
                      "mixed_over_fp64": r_mixed["atom_steps_per_s"] / r_fp64["atom_steps_per_s"],
                      "cpu_reference_1000_steps": cpu,
                      "gpu_mixed_over_cpu": r_mixed["atom_steps_per_s"] / cpu["value"]}
    # config 2: 90,000 atoms
    s90 = make_workload("gly1500_wat25000_90k", seed=2000)
    r_mixed, x, v = md_rate(ctx, M, s90, M.MIXED, 500)
    r_fp64, _, _ = md_rate(ctx, M, s90, M.FP64, 500)
    row = {"atoms": s90.np_atoms, "mixed": r_mixed, "fp64": r_fp64,
           "mixed_over_fp64": r_mixed["atom_steps_per_s"] / r_fp64["atom_steps_per_s"]}
    # force error on snapshots of a Langevin trajectory
    run = M.System(ctx, s90, alpha=ALPHA, cut=CUT, skin=SKIN)
    run.set_state(x, v)
    run.md_setup(s90, dt=DT, temperature=300.0, gamma=0.001, seed=31)
    probe = M.System(ctx, s90, alpha=ALPHA, cut=CUT, skin=SKIN)
    rms, mx = [], []
    for _ in range(5):
        run.md_run(200)
        xs, _, _ = run.get_state()
        probe.set_state(xs)
        probe.compute(M.FP64, rebuild=True, energy=False, virial=False)
        f64 = probe.get_state()[2]
        probe.compute(M.MIXED, rebuild=True, energy=False, virial=False)
        f32 = probe.get_state()[2]
        rms.append(M.force_rms_rel(f32, f64))
        mx.append(M.force_max_rel(f32, f64))
    row["force_error_vs_fp64"] = {"snapshots": 5, "rms_rel_max": max(rms),
                                  "max_rel_max": max(mx), "bar_rms": 1e-6}
    # neighbour rows of the reference-semantics GPU build vs the oracle, as sets
    from oracle import oracle as O
    xs, vs, _ = run.get_state()
    pos = s90.position_aos().copy()
    Lb = float(s90.box)
    w = np.mod(xs, Lb).astype(np.float32)
    w[w <= 0] += np.float32(Lb)
    pos[:, :3] = w
    p = nb.DsfParams(alpha=ALPHA, box=s90.box, cut_coul=CUT, rcut=CUT, neighbor_pad=SKIN)
    gnl, gnn, gna = nb.neighbor_wrapper(ctx, pos, s90.specbond, s90.num3bond, p, 1024)
    op = O.params(ALPHA, s90.box, CUT, CUT, SKIN)
    # the strict-IEEE oracle (the parity checker), not the contracting timing build
    onl, onn, ona = O.neighbor_wrapper(op, pos, s90.specbond, s90.num3bond, 1024)
    same = bool(np.array_equal(gnn, onn) and
                np.array_equal(row_hash(gnl, gnn, gna), row_hash(onl, onn, ona)))
    row["neighbor_sets_bit_exact"] = {"equal": same, "entries": int(onn.sum())}
    run.close()
    probe.close()
    # NVE drift: the reference scheme and the RATTLE + LJ-shift variant
    from molecular_simulation_code_b200.validate import nve_drift
    drift = {}
    for name, rattle, shift in (("reference_scheme", False, False),
                                ("rattle_ljshift", True, True)):
        drift[name] = nve_drift(M, ctx, s90, xs, vs, dt=DT, precision=M.MIXED, rattle=rattle,
                                lj_shift=shift, shake_tol=1e-10, ps=20.0, cut=CUT, skin=SKIN)
    row["nve_drift_20ps"] = drift
    out["cfg2_90k"] = row
    # config 4: 64 replicas in one batch
    if time.time() - t_start < budget_s:
        from molecular_simulation_code_b200.replica_bench import bench_batch
        a = argparse.Namespace(replicas=64, seed=5000, procs=min(16, os.cpu_count() or 1),
                               tune=False, segment=100, segments=3)
        out["cfg4_batch64"] = bench_batch(a)
        out["cfg4_batch64"]["pair_launches_per_batch_step"] = 1
    # config 5: serving
    if time.time() - t_start < budget_s:
        from molecular_simulation_code_b200.replica_bench import bench_serve
        a = argparse.Namespace(requests=args.serve_requests, rate=200.0, steps_scale=1.0,
                               chunk=100, max_active=64, budget_gb=96.0, seed=7000,
                               procs=min(16, os.cpu_count() or 1), nucleus_every=4)
        out["cfg5_serve"] = bench_serve(a)
    out["wall_s"] = time.time() - t_start
    return out


def run_ours(args, rank, ws):
    import torch

    from molecular_simulation_code_b200 import mixed as M
    from molecular_simulation_code_b200 import nonbond as nb

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    s = build_system(args, rank)
    n = s.np_atoms
    fp32_peak = measure_fp32_peak() if rank == 0 else 0.0
    ctx = nb.Context(dev)
    stream = torch.cuda.ExternalStream(ctx._lib.sofia_stream(ctx.handle))
    sysm = M.System(ctx, s, alpha=ALPHA, cut=CUT, skin=SKIN, precision=M.MIXED)
    x0 = s.xyz.astype(np.float64)
    v0 = s.velocity.astype(np.float64)
    sysm.set_state(x0, v0)

    def md_loop(precision, nsteps, warm):
        """Device-resident MD: relax (untimed), warm up, then time nsteps in one graph segment."""
        m = M.System(ctx, s, alpha=ALPHA, cut=CUT, skin=SKIN, precision=precision)
        m.set_state(x0, v0)
        m.md_setup(s, dt=1.0, temperature=300.0, gamma=0.02, seed=11)
        m.md_run(RELAX_STEPS)  # lattice start: short strongly damped relaxation
        m.md_setup(s, dt=DT, temperature=300.0, gamma=0.02, seed=13)
        m.md_run(EQUIL_STEPS)  # release the lattice energy into the bath (tau = 50 fs)
        m.md_setup(s, dt=DT, temperature=300.0, gamma=0.001, seed=12)
        m.md_run(max(warm, 1))
        b0 = m.stats()
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("md_timed")  # lets ncu select the timed MD steps
        e0.record(stream)
        en = m.md_run(nsteps, energy_every=nsteps, use_graph=True)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        barrier(ws)
        b1 = m.stats()
        t = e0.elapsed_time(e1) / 1e3
        m.close()
        return t, en, b1["builds"] - b0["builds"], b1["prunes"] - b0["prunes"], \
            b1["launches"] - b0["launches"]

    def timed_loop(precision, nsteps, warm):
        sysm.set_state(x0, v0)
        for _ in range(warm):
            sysm.drift(DT)
            sysm.compute(precision, energy=True, virial=False)
        b0 = sysm.stats()
        sysm.timers(True)
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps):
            sysm.drift(DT)
            sysm.compute(precision, energy=True, virial=False)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        t = e0.elapsed_time(e1) / 1e3
        tm = sysm.timers(False)
        b1 = sysm.stats()
        return t, tm, b1["builds"] - b0["builds"], b1["launches"] - b0["launches"], b1

    if args.only_hot:
        t_hot, tm, builds, launches, st = timed_loop(M.MIXED, args.steps, args.warmup)
        print(json.dumps({"mode": "hot path only", "atom_steps_per_s": n * args.steps / t_hot,
                          "pair_ms": tm["pair_ms"] / max(tm["pairs"], 1), "list": st}),
              flush=True)
        return
    with Clocks(dev) as clk:
        t_md, md_en, md_builds, md_prunes, md_launches = md_loop(M.MIXED, args.steps,
                                                                 args.warmup)
    t_max = allreduce_max(t_md, ws, device=torch.device("cuda", dev))
    value = n * ws * args.steps / t_max
    t_md64 = None
    if not args.no_fp64:
        t_md64, _, _, _, _ = md_loop(M.FP64, args.steps, args.warmup)
        t_md64 = allreduce_max(t_md64, ws, device=torch.device("cuda", dev))

    # nonbonded hot path only (ballistic drift between evaluations), with kernel timers
    t_hot, tm, builds, launches, st = timed_loop(M.MIXED, args.steps, args.warmup)
    t_hot = allreduce_max(t_hot, ws, device=torch.device("cuda", dev))

    # plain FP64 twin of the same kernel and list
    t_fp64 = None
    if not args.no_fp64:
        t_fp64, tm64, _, _, _ = timed_loop(M.FP64, args.steps, args.warmup)
        t_fp64 = allreduce_max(t_fp64, ws, device=torch.device("cuda", dev))

    # FP64 reference-semantics path (27-cell full list + FP64 pair kernel)
    t_ref = None
    if not args.no_fp64:
        p = nb.DsfParams(alpha=ALPHA, box=s.box, cut_coul=CUT, rcut=CUT, neighbor_pad=SKIN)
        lj = [torch.from_numpy(a).cuda() for a in (s.lj1, s.lj2, s.lj3, s.lj4)]
        qd = torch.from_numpy(s.q).cuda()
        sbd = torch.from_numpy(np.ascontiguousarray(s.specbond)).cuda()
        n3d = torch.from_numpy(s.num3bond).cuda()
        posd = torch.from_numpy(s.position_aos()).cuda()
        L = float(s.box)
        half2 = (0.5 * SKIN) ** 2
        na = 1024
        xref = x0.copy()
        frames = []
        for k in range(args.steps + args.warmup):
            x = x0 + v0 * DT * (k + 1)
            rb = False
            d = x - xref
            d -= L * np.round(d / L)
            if k == 0 or (np.einsum("ij,ij->i", d, d) > half2).any():
                rb = True
                xref = x.copy()
            xw = np.mod(x, L).astype(np.float32)
            xw[xw <= 0] += np.float32(L)
            frames.append((xw, rb))
        ff = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        tot = 0.0
        for k, (xw, rb) in enumerate(frames):
            posd[:, :3] = torch.from_numpy(xw).cuda()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if rb:
                _, _, na = nb.neighbor_wrapper(ctx, posd, sbd, n3d, p, na, want_host=False)
            nb.lj_cut_coul_dsf_nonewton(ctx, posd, qd, lj, s.ntypes, None, None, na, p, ff=ff)
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= args.warmup:
                tot += e0.elapsed_time(e1) / 1e3
        t_ref = allreduce_max(tot, ws, device=torch.device("cuda", dev))
        del lj, qd, sbd, n3d, posd, ff

    # e2e: drop-in call with pinned host positions in and real*4 forces out each step
    nf = args.steps + args.warmup
    frames = torch.empty((nf, n, 4), dtype=torch.float32, pin_memory=True)
    tbits = torch.from_numpy(s.types.view(np.float32).copy())
    for k in range(nf):
        frames[k, :, :3] = torch.from_numpy((x0 + v0 * DT * (k + 1)).astype(np.float32))
        frames[k, :, 3] = tbits
    ffh = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    drop = M.System(ctx, s, alpha=ALPHA, cut=CUT, skin=SKIN, precision=M.MIXED)
    for k in range(args.warmup):
        drop.forces_dropin(frames[k], ff=ffh)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.warmup, nf):
        drop.forces_dropin(frames[k], ff=ffh)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = allreduce_max(e0.elapsed_time(e1) / 1e3, ws, device=torch.device("cuda", dev))
    drop.close()

    if rank != 0:
        return
    P_rv = count_pairs_within(s, CUT + SKIN)
    pair_ms = tm["pair_ms"] / max(tm["pairs"], 1)
    achieved = FLOP_PER_PAIR * P_rv / (pair_ms / 1e3) / 1e12
    rebuild_interval = args.steps / max(md_builds, 1)
    cpu = None if args.no_cpu_baseline else cpu_baseline(s, rebuild_interval)
    clocks = clk.summary()
    # the list build: algorithmic bytes per rebuild (positions and types read, sorted
    # records written, cell ids, 4 B list index per pair within rc + skin) over the
    # measured build time, against the measured HBM copy bandwidth
    build_ms = tm["build_ms"] / max(tm["builds"], 1)
    b_nb = n * (24 + 4) + n * 28 + n * 4 + 4 * P_rv
    hbm_peak, peak_src = measured_hbm()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    fp32_spec = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    extras = None
    if not args.no_extras and ws == 1:
        extras = extra_rows(args, ctx)
    out = {
        "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "atoms_per_gpu": n, "rc_A": CUT, "skin_A": SKIN,
                   "prune_margin_A": 0.4,
                   "dt_fs": DT, "precision": "mixed FP32 pair / FP64 positions / int64 forces",
                   "parallelism": f"replicas x{ws} (no exchange)",
                   "l2": "inputs larger than L2 (cluster-pair list "
                         f"{st['entries'] * 12 / 1e9:.2f} GB)",
                   "step": "2 fs MD step: velocity Verlet + Langevin 300 K + SHAKE + bonded/1-4 + "
                           "nonbonded LJ/DSF (list rebuild/prune on device triggers), CUDA graph"},
        "md": {"energies_last_step": md_en, "list_rebuilds": md_builds, "prunes": md_prunes,
               "ns_per_day": DT * 1e-6 * args.steps / t_max * 86400.0},
        "fp64": {"md_atom_steps_per_s": (n * ws * args.steps / t_md64) if t_md64 else None,
                 "mixed_over_fp64_md": (t_md64 / t_max) if t_md64 else None,
                 "hot_path_cluster_atom_steps_per_s": (n * ws * args.steps / t_fp64) if t_fp64 else None,
                 "hot_path_reference_list_atom_steps_per_s": (n * ws * args.steps / t_ref) if t_ref else None,
                 "hot_path_mixed_over_fp64_cluster": (t_fp64 / t_hot) if t_fp64 else None,
                 "hot_path_mixed_over_fp64_reference_list": (t_ref / t_hot) if t_ref else None},
        "hot_path": {"atom_steps_per_s": n * ws * args.steps / t_hot,
                     "step": "2 fs ballistic update + displacement check + rebuild/prune on "
                             "trigger + LJ/DSF forces and energies"},
        # d2h: real*4 forces, 5 energy words and the 16 list-status words
        "e2e": {"value": n * ws * args.steps / t_e2e, "unit": "atom-steps/s",
                "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 12 * n + 40 + 64},
        "gpu_launches": md_launches,
        "list": {"rebuilds": builds, "clusters": st["clusters"], "entries": st["entries"],
                 "pruned_entries": st["inner_entries"], "prunes": st["prunes"],
                 "build_ms": tm["build_ms"] / max(tm["builds"], 1)},
        "roofline": {"bound": "fp32", "kernel": "k_pair<float,EN=1,VIR=0>",
                     "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak if fp32_peak else None,
                     "traffic": read_profile_traffic(),
                     "pair_ms": pair_ms, "pairs_P_rv": P_rv,
                     "flop_per_pair": FLOP_PER_PAIR,
                     "peak_source": "measured cuBLAS SGEMM 8192^3, TF32 off, on this GPU"},
        "roofline_build": {"bound": "hbm", "kernels": "k_wrap_bin .. k_search (one rebuild)",
                           "build_ms": build_ms, "algorithmic_bytes": b_nb,
                           "achieved": b_nb / (build_ms / 1e3) / 1e9 if build_ms else None,
                           "peak": hbm_peak, "unit": "GB/s",
                           "frac": (b_nb / (build_ms / 1e3) / 1e9 / hbm_peak) if build_ms else None,
                           "peak_source": peak_src,
                           "list_bytes_written": st["entries"] * 12},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "configs": extras,
    }
    out["roofline"]["peak_fp32_spec"] = fp32_spec
    out["roofline"]["frac_of_fp32_spec"] = achieved / fp32_spec
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, ws = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, ws)
        else:
            run_ours(args, rank, ws)
    finally:
        if ws > 1:
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
