"""GPU tests of the device-resident MD step (residency kernels around the hot path)."""
import numpy as np
import pytest

from molecular_simulation_code_b200 import mixed as M
from molecular_simulation_code_b200.system import make_system

pytestmark = pytest.mark.gpu


def _system(ctx, s, precision=M.MIXED, **md):
    sysm = M.System(ctx, s, cut=8.0, skin=2.0, precision=precision)
    sysm.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    sysm.md_setup(s, **md)
    return sysm


@pytest.fixture(scope="module")
def small():
    return make_system(20, 900, 21)


def _constraint_err(s, x):
    L = float(s.box)
    worst = 0.0
    for g, b in zip(s.shake, s.shake_bond):
        num, a = int(g[0]), g[1:] - 1
        pairs = {1: [(0, 1)], 3: [(0, 1), (0, 2)], 4: [(0, 1), (0, 2), (0, 3)],
                 -3: [(0, 1), (0, 2), (1, 2)]}[num]
        for k, (u, w) in enumerate(pairs):
            d = x[a[u]] - x[a[w]]
            d -= L * np.round(d / L)
            worst = max(worst, abs(np.linalg.norm(d) - b[k]))
    return worst


def test_md_deterministic_and_graph_equals_eager(ctx, small):
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.01, seed=7)
    a.md_run(30, use_graph=True)
    xa, va, fa = a.get_state()
    b = _system(ctx, s, dt=1.0, gamma=0.01, seed=7)
    b.md_run(30, use_graph=False)
    xb, vb, fb = b.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and np.array_equal(fa, fb)
    c = _system(ctx, s, dt=1.0, gamma=0.01, seed=8)
    c.md_run(30)
    xc, _, _ = c.get_state()
    assert not np.array_equal(xa, xc)  # another noise stream
    for o in (a, b, c):
        o.close()


def test_stats_before_first_build(ctx, small):
    """A system queried before its first list build reports no clusters, even when
    its buffers reuse device memory full of another run's data, and the query
    leaves no CUDA error behind for the next call."""
    import torch
    junk = torch.full((64 << 20,), 0x7fffffff, dtype=torch.int32, device="cuda")
    del junk
    torch.cuda.empty_cache()
    a = _system(ctx, small, dt=1.0, gamma=0.01, seed=3)
    st = a.stats()
    assert st["clusters"] == 0 and st["entries"] == 0 and st["inner_entries"] == 0
    a.md_run(3, use_graph=True)
    st = a.stats()
    assert 0 < st["clusters"] <= st["max_clusters"] and st["entries"] > 0
    a.close()


def test_segment_graphs_with_energies_equal_eager(ctx, small):
    """Segment graphs chain each step's closing half-kick into the next step's
    kick and drift; with energies every 7th step (segments with and without an
    energy step, single-step graphs between them) the state and the energies
    equal the eager step-by-step path's bit for bit."""
    s = small
    a = _system(ctx, s, dt=2.0, gamma=0.01, seed=6)
    ea = [a.md_run(37, energy_every=7, use_graph=True) for _ in range(2)]
    b = _system(ctx, s, dt=2.0, gamma=0.01, seed=6)
    eb = [b.md_run(37, energy_every=7, use_graph=False) for _ in range(2)]
    xa, va, fa = a.get_state()
    xb, vb, fb = b.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and np.array_equal(fa, fb)
    assert ea == eb
    a.close()
    b.close()


def test_graph_conditional_build_and_prune_equal_eager(ctx, small):
    """Long enough for several list rebuilds and prunes: the captured step (build
    and prune as conditional graph nodes) takes exactly the eager path's steps."""
    s = small
    a = _system(ctx, s, dt=2.0, gamma=0.01, seed=5)
    a0 = a.stats()
    a.md_run(150, use_graph=True)
    a1 = a.stats()
    b = _system(ctx, s, dt=2.0, gamma=0.01, seed=5)
    b.md_run(150, use_graph=False)
    b1 = b.stats()
    assert a1["builds"] - a0["builds"] >= 2 and a1["prunes"] - a0["prunes"] >= 2
    assert (a1["builds"], a1["prunes"]) == (b1["builds"], b1["prunes"])
    xa, va, _ = a.get_state()
    xb, vb, _ = b.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    a.close()
    b.close()


def test_md_improper_term_matches_reference_entry(ctx, small):
    """The device MD's improper energy equals sofia_improper_harmonic on the same
    positions, and switching the term off removes it.  The reference entry takes
    real*4 positions, so the two evaluate at positions that differ by the float
    rounding (hence rel 1e-4).  The comparison with the oracle on positions exact
    in real*4 (energy at 1e-10, forces at the oracle's real*4 storage) is in
    test_gpu_residency_parity.py."""
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.0, seed=1)
    e = a.md_run(1, energy_every=1)
    x, _, _ = a.get_state()
    from molecular_simulation_code_b200.nonbond import DsfParams, improper_harmonic
    pos = s.position_aos().copy()
    pos[:, :3] = x.astype(np.float32)
    p = DsfParams(alpha=0.2, box=s.box, cut_coul=8.0, rcut=8.0, neighbor_pad=2.0)
    _, e_ref, _ = improper_harmonic(ctx, pos, s.impropers, s.impro_coeff, p)
    assert e["improper"] == pytest.approx(e_ref, rel=1e-4, abs=1e-6)
    b = _system(ctx, s, dt=1.0, gamma=0.0, seed=1, terms=15)
    assert b.md_run(1, energy_every=1)["improper"] == 0.0
    a.close()
    b.close()


def test_md_shake_keeps_constraints(ctx, small):
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.02, seed=3, shake_maxiter=200, shake_tol=1e-10)
    a.md_run(50)
    x, _, _ = a.get_state()
    assert _constraint_err(s, x) < 1e-5
    a.close()


def test_md_langevin_thermalises_and_stays_finite(ctx, small):
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.05, seed=5, temperature=300.0)
    e = None
    for _ in range(8):
        e = a.md_run(50, energy_every=50)
    assert np.isfinite(e["total"])
    assert 200.0 < e["temperature"] < 420.0, e
    x, v, f = a.get_state()
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    a.close()


def test_md_nve_conserves_energy_short(ctx, small):
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.05, seed=9, shake_maxiter=100, shake_tol=1e-10)
    a.md_run(300)  # relax the lattice start under the thermostat
    a.md_setup(s, dt=1.0, gamma=0.0, seed=9, shake_maxiter=100, shake_tol=1e-10)
    es = [a.md_run(20, energy_every=20)["total"] for _ in range(10)]
    ke = a.md_run(1, energy_every=1)["kinetic"]
    spread = max(es) - min(es)
    assert spread < 0.01 * ke, (es, ke)
    a.close()


def test_md_fp64_and_mixed_trajectories_stay_close(ctx, small):
    s = small
    a = _system(ctx, s, dt=1.0, gamma=0.0, seed=1)
    b = _system(ctx, s, precision=M.FP64, dt=1.0, gamma=0.0, seed=1)
    a.md_run(10)
    b.md_run(10)
    xa, _, _ = a.get_state()
    xb, _, _ = b.get_state()
    assert np.abs(xa - xb).max() < 1e-3
    a.close()
    b.close()


def _velocity_constraint_residual(s, x, v):
    """max |(v_p - v_q) . r_pq| / |r_pq| over all SHAKE constraints, relative to rms |v|."""
    L = float(s.box)
    worst = 0.0
    for g in s.shake:
        num, a = int(g[0]), g[1:] - 1
        pairs = {1: [(0, 1)], 3: [(0, 1), (0, 2)], 4: [(0, 1), (0, 2), (0, 3)],
                 -3: [(0, 1), (0, 2), (1, 2)]}[num]
        for u, w in pairs:
            d = x[a[u]] - x[a[w]]
            d -= L * np.round(d / L)
            worst = max(worst, abs(np.dot(v[a[u]] - v[a[w]], d)) / np.linalg.norm(d))
    return worst / np.sqrt((v * v).sum(axis=1).mean())


def test_md_rattle_changes_only_full_step_velocities(ctx, small):
    """The RATTLE stage projects the full-step velocities onto the constraints
    and leaves the positions of the SHAKE step unchanged (to rounding of the
    fixed-point force it compensates).  Both runs start from the same relaxed
    state: from the lattice start the first steps are violent collisions that
    amplify the rounding-level differences by orders of magnitude within a few
    steps.  An uncompensated velocity projection would move positions by about
    1e-3 A per step, so 1e-7 A after 10 steps separates the two cases by four
    orders of magnitude."""
    s = small
    w = _system(ctx, s, dt=1.0, gamma=0.02, seed=3)
    w.md_run(100)
    x0, v0, _ = w.get_state()
    w.close()
    kw = dict(dt=2.0, gamma=0.0, seed=1, shake_maxiter=200, shake_tol=1e-12)
    a = M.System(ctx, s, cut=8.0, skin=2.0)
    a.set_state(x0, v0)
    a.md_setup(s, **kw)
    b = M.System(ctx, s, cut=8.0, skin=2.0)
    b.set_state(x0, v0)
    b.md_setup(s, rattle=True, **kw)
    a.md_run(10)
    b.md_run(10)
    xa, va, _ = a.get_state()
    xb, vb, _ = b.get_state()
    assert np.abs(xa - xb).max() < 1e-7, np.abs(xa - xb).max()
    assert _velocity_constraint_residual(s, xb, vb) < 1e-9
    assert _velocity_constraint_residual(s, xa, va) > 1e-6
    a.close()
    b.close()


def test_md_nve_drift_slope_bounded(ctx):
    """NVE energy drift of the 9,000-atom system over 4 ps after a Langevin
    warm-up (0.5 fs steps, RATTLE velocity stage, LJ energy shift, SHAKE to
    1e-10): the least-squares slope of the total energy stays within
    0.02 kT/ns/atom (the 90k-atom 100 ps runs give |slope| <= 3e-4 at 2 fs with
    the same options), which a broken force or integrator exceeds by orders of
    magnitude."""
    s = make_system(150, 2500, 1)
    m = M.System(ctx, s, cut=10.0, skin=2.0)
    m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    m.md_setup(s, dt=1.0, gamma=0.02, seed=3)
    m.md_run(500)
    m.md_setup(s, dt=2.0, gamma=0.01, seed=4)
    m.md_run(1000)
    m.md_setup(s, dt=0.5, gamma=0.0, seed=5, shake_maxiter=200, shake_tol=1e-10, rattle=True,
               lj_shift=True)
    ts, es = [], []
    for k in range(40):
        e = m.md_run(200, energy_every=200)
        ts.append((k + 1) * 200 * 0.5e-6)  # ns
        es.append(e["total"])
    kT = 0.001987204181 * 300.0
    slope = np.polyfit(np.array(ts), np.array(es), 1)[0] / kT / s.np_atoms
    print("9k NVE drift (kT/ns/atom):", slope, "T:", e["temperature"])
    assert abs(slope) < 0.02, slope
    assert 250.0 < e["temperature"] < 360.0
    m.close()
