"""Accuracy and stability measurements of the production path.

Measures, on a seeded glycine/water system (default 90,000 atoms: 1,500
glycine + 25,000 water):

* mixed (FP32 pair / fixed-point) vs plain FP64 forces on N snapshots taken
  every ``--every`` steps of a Langevin trajectory: force RMS relative error
  sqrt(sum|df|^2 / sum|f|^2) and max relative error max|df| / max|f|;
* NVE energy drift over ``--nve-ps`` picoseconds for both precisions, as the
  slope of a least-squares line through the total energy, in kT/ns/atom.

``--drift-study`` instead runs the NVE drift of several integration variants
from one equilibrated state (time step, SHAKE tolerance, the RATTLE velocity
stage, the LJ energy shift at the cut-off, mixed or FP64 pair arithmetic) and
reports each slope with two error estimates: the least-squares standard error
(independent residuals) and the spread of the slopes of five consecutive
blocks (correlated residuals).

Prints one JSON line.  Usage:
    python -m molecular_simulation_code_b200.validate [--workload NAME]
    python -m molecular_simulation_code_b200.validate --drift-study [--nve-ps PS]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="gly1500_wat25000_90k")
    ap.add_argument("--snapshots", type=int, default=20)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--equil", type=int, default=1000)
    ap.add_argument("--nve-ps", type=float, default=10.0)
    ap.add_argument("--dt", type=float, default=2.0)
    ap.add_argument("--cut", type=float, default=10.0)
    ap.add_argument("--skin", type=float, default=2.0)
    ap.add_argument("--drift-study", action="store_true")
    ap.add_argument("--variants", default="all",
                    help="comma-separated variant names of the drift study (default all)")
    args = ap.parse_args(argv)
    if args.drift_study:
        return drift_study(args)

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from molecular_simulation_code_b200 import mixed as M
    from molecular_simulation_code_b200 import nonbond as nb
    from molecular_simulation_code_b200.system import make_workload

    t0 = time.time()
    s = make_workload(args.workload, seed=2000)
    n = s.np_atoms
    ctx = nb.Context(0)
    run = M.System(ctx, s, cut=args.cut, skin=args.skin, precision=M.MIXED)
    run.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    run.md_setup(s, dt=1.0, temperature=300.0, gamma=0.02, seed=21)
    run.md_run(100)
    run.md_setup(s, dt=args.dt, temperature=300.0, gamma=0.001, seed=22)
    run.md_run(args.equil)
    probe = M.System(ctx, s, cut=args.cut, skin=args.skin, precision=M.MIXED)
    rms, mx = [], []
    for k in range(args.snapshots):
        run.md_run(args.every)
        x, v, _ = run.get_state()
        probe.set_state(x)
        probe.compute(M.FP64, rebuild=True, energy=False)
        _, _, f64 = probe.get_state()
        probe.compute(M.MIXED, rebuild=True, energy=False)
        _, _, f32 = probe.get_state()
        rms.append(M.force_rms_rel(f32, f64))
        mx.append(M.force_max_rel(f32, f64))
    x_last, v_last, _ = run.get_state()

    # NVE drift for both precisions from the last snapshot
    kT = 0.001987204181 * 300.0
    nsteps = int(round(args.nve_ps * 1000.0 / args.dt))
    chunk = 50
    drift = {}
    for name, prec in (("mixed", M.MIXED), ("fp64", M.FP64)):
        sysn = M.System(ctx, s, cut=args.cut, skin=args.skin, precision=prec)
        sysn.set_state(x_last, v_last)
        sysn.md_setup(s, dt=args.dt, gamma=0.0, seed=1, shake_maxiter=100, shake_tol=1e-10)
        ts, es = [], []
        for k in range(nsteps // chunk):
            e = sysn.md_run(chunk, energy_every=chunk)
            ts.append((k + 1) * chunk * args.dt * 1e-6)  # ns
            es.append(e["total"])
        ts = np.array(ts)
        es = np.array(es)
        coef = np.polyfit(ts, es, 1)
        slope = float(coef[0])  # kcal/mol/ns
        resid = es - np.polyval(coef, ts)
        # standard error of the least-squares slope (independent residuals)
        se = float(np.sqrt((resid ** 2).sum() / max(len(ts) - 2, 1) / ((ts - ts.mean()) ** 2).sum()))
        drift[name] = {"kT_per_ns_per_atom": slope / kT / n,
                       "stderr_kT_per_ns_per_atom": se / kT / n,
                       "energy_rms_fluct_kcal": float(np.std(resid)),
                       "ps": args.nve_ps, "last_temperature_K": e["temperature"]}
        sysn.close()
    out = {"workload": args.workload, "atoms": n, "snapshots": args.snapshots,
           "force_rms_rel": {"max": max(rms), "mean": float(np.mean(rms))},
           "force_max_rel": {"max": max(mx), "mean": float(np.mean(mx))},
           "nve_drift": drift,
           "wall_s": time.time() - t0}
    print(json.dumps(out), flush=True)
    return out


# name -> (dt fs, precision, rattle, lj_shift, shake_tol)
VARIANTS = {
    "ref_2fs": (2.0, "mixed", False, False, 1e-10),
    "ref_2fs_tol1e-4": (2.0, "mixed", False, False, 1e-4),
    "rattle_2fs": (2.0, "mixed", True, False, 1e-10),
    "ljshift_2fs": (2.0, "mixed", False, True, 1e-10),
    "both_2fs": (2.0, "mixed", True, True, 1e-10),
    "both_1fs": (1.0, "mixed", True, True, 1e-10),
    "both_0.5fs": (0.5, "mixed", True, True, 1e-10),
    "both_2fs_fp64": (2.0, "fp64", True, True, 1e-10),
}


def nve_drift(M, ctx, s, x, v, *, dt, precision, rattle, lj_shift, shake_tol, ps, cut, skin,
              sample_fs=100.0):
    """NVE run from (x, v): total energy every ``sample_fs``; returns the drift fit."""
    n = s.np_atoms
    kT = 0.001987204181 * 300.0
    sysn = M.System(ctx, s, cut=cut, skin=skin, precision=precision)
    sysn.set_state(x, v)
    sysn.md_setup(s, dt=dt, gamma=0.0, seed=1, shake_maxiter=200, shake_tol=shake_tol,
                  rattle=rattle, lj_shift=lj_shift)
    chunk = max(1, int(round(sample_fs / dt)))
    nsteps = int(round(ps * 1000.0 / dt))
    ts, es, comps = [], [], []
    names = ("lj", "coul", "kinetic", "bond", "angle", "coul14", "lj14", "improper")
    e = None
    t0 = time.time()
    for k in range(nsteps // chunk):
        e = sysn.md_run(chunk, energy_every=chunk)
        ts.append((k + 1) * chunk * dt * 1e-6)  # ns
        es.append(e["total"])
        comps.append([e[c] for c in names])
    wall = time.time() - t0
    ts, es = np.array(ts), np.array(es)
    comps = np.array(comps)
    coef = np.polyfit(ts, es, 1)
    resid = es - np.polyval(coef, ts)
    se = float(np.sqrt((resid ** 2).sum() / max(len(ts) - 2, 1) / ((ts - ts.mean()) ** 2).sum()))
    blocks = [np.polyfit(tb, eb, 1)[0] for tb, eb in zip(np.array_split(ts, 5),
                                                          np.array_split(es, 5))]
    st = sysn.stats()
    sysn.close()
    scale = 1.0 / kT / n
    parts = {c: float(np.polyfit(ts, comps[:, i], 1)[0]) * scale for i, c in enumerate(names)}
    return {"kT_per_ns_per_atom": float(coef[0]) * scale,
            "component_slopes_kT_per_ns_per_atom": parts,
            "stderr_lsq": se * scale,
            "stderr_blocks": float(np.std(blocks, ddof=1) / np.sqrt(len(blocks))) * scale,
            "energy_rms_fluct_kcal": float(np.std(resid)),
            "ps": ps, "dt_fs": dt, "last_temperature_K": e["temperature"],
            "shake_maxiter_hits": st["shake_maxiter_hits"], "wall_s": wall}


def drift_study(args):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from molecular_simulation_code_b200 import mixed as M
    from molecular_simulation_code_b200 import nonbond as nb
    from molecular_simulation_code_b200.system import make_workload

    t0 = time.time()
    s = make_workload(args.workload, seed=2000)
    ctx = nb.Context(0)
    run = M.System(ctx, s, cut=args.cut, skin=args.skin, precision=M.MIXED)
    run.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    run.md_setup(s, dt=1.0, temperature=300.0, gamma=0.02, seed=21)
    run.md_run(100)
    run.md_setup(s, dt=2.0, temperature=300.0, gamma=0.02, seed=22)
    run.md_run(1000)
    run.md_setup(s, dt=2.0, temperature=300.0, gamma=0.001, seed=23)
    run.md_run(args.equil)
    x, v, _ = run.get_state()
    run.close()
    names = list(VARIANTS) if args.variants == "all" else args.variants.split(",")
    out = {"workload": args.workload, "atoms": s.np_atoms, "equil_steps": args.equil,
           "variants": {}}
    for name in names:
        dt, prec, rattle, shift, tol = VARIANTS[name]
        out["variants"][name] = nve_drift(
            M, ctx, s, x, v, dt=dt, precision=M.MIXED if prec == "mixed" else M.FP64,
            rattle=rattle, lj_shift=shift, shake_tol=tol, ps=args.nve_ps, cut=args.cut,
            skin=args.skin)
        print(name, json.dumps(out["variants"][name]), file=sys.stderr, flush=True)
    out["wall_s"] = time.time() - t0
    print(json.dumps(out), flush=True)
    ctx.close()
    return out


if __name__ == "__main__":
    main()
