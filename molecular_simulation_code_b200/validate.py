"""Accuracy and stability measurements of the production path.

Measures, on a seeded glycine/water system (default 90,000 atoms: 1,500
glycine + 25,000 water):

* mixed (FP32 pair / fixed-point) vs plain FP64 forces on N snapshots taken
  every ``--every`` steps of a Langevin trajectory: force RMS relative error
  sqrt(sum|df|^2 / sum|f|^2) and max relative error max|df| / max|f|;
* NVE energy drift over ``--nve-ps`` picoseconds for both precisions, as the
  slope of a least-squares line through the total energy, in kT/ns/atom.

Prints one JSON line.  Usage:
    python -m molecular_simulation_code_b200.validate [--workload NAME]
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
    args = ap.parse_args(argv)

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


if __name__ == "__main__":
    main()
