"""GPU tests: replica batches and the continuous-batching segment server.

Bar: a replica's trajectory is bit-identical alone and inside a batch (and
across segment boundaries), so each served result is the same alone and in
the mix (tolerance: exact).
"""
import numpy as np
import pytest

from molecular_simulation_code_b200 import mixed as M
from molecular_simulation_code_b200 import nonbond as nb
from molecular_simulation_code_b200.batch import (Batch, autotune, autotune_margin,
                                                  set_cluster_shape, set_margin)
from molecular_simulation_code_b200.serve import Request, Server, estimate_bytes, run_stream
from molecular_simulation_code_b200.system import make_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def replicas():
    return [make_system(6, 700, 31), make_system(12, 1100, 32), make_system(4, 600, 33)]


def _prep(ctx, s, seed):
    m = M.System(ctx, s, cut=8.0, skin=2.0)
    m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    m.md_setup(s, dt=1.0, gamma=0.01, seed=seed)
    return m


def test_batch_equals_alone(ctx, replicas):
    alone = []
    for k, s in enumerate(replicas):
        c = nb.Context(0)
        m = _prep(c, s, 100 + k)
        m.md_run(40)
        alone.append(m.get_state()[0])
        m.close()
        c.close()
    ctxs = [nb.Context(0) for _ in replicas]
    systems = [_prep(c, s, 100 + k) for k, (c, s) in enumerate(zip(ctxs, replicas))]
    b = Batch(ctx, systems)
    b.run(15)
    e = b.run(25, energy_every=25)
    assert len(e) == len(replicas) and all(np.isfinite(r["total"]) for r in e)
    for k, m in enumerate(systems):
        assert np.array_equal(m.get_state()[0], alone[k]), f"replica {k} differs"
    b.close()
    for m in systems:
        m.close()
    for c in ctxs:
        c.close()


def _alone(s, seed, nsteps, **md):
    c = nb.Context(0)
    m = M.System(c, s, cut=8.0, skin=2.0)
    m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    m.md_setup(s, dt=1.0, gamma=0.01, seed=seed, **md)
    e = m.md_run(nsteps, energy_every=nsteps)
    x, v, _ = m.get_state()
    m.close()
    c.close()
    return x, v, e


def test_batch_segment_graphs_equal_alone(ctx, replicas):
    """Captured multi-step segments (10 steps per graph) and single-step launches
    give each replica exactly its lone trajectory and last-step energies."""
    ref = [_alone(s, 300 + k, 37) for k, s in enumerate(replicas)]
    ctxs = [nb.Context(0) for _ in replicas]
    systems = [_prep(c, s, 300 + k) for k, (c, s) in enumerate(zip(ctxs, replicas))]
    b = Batch(ctx, systems)
    b.set_segment(10)
    e = b.run(37, energy_every=37)  # 3 segment graphs + 7 single steps
    for k, m in enumerate(systems):
        x, v, _ = m.get_state()
        assert np.array_equal(x, ref[k][0]) and np.array_equal(v, ref[k][1]), k
        assert e[k] == ref[k][2], k
    b.close()
    for m in systems:
        m.close()
    for c in ctxs:
        c.close()


def test_batch_membership_change_keeps_trajectories(ctx, replicas):
    """Continuous batching: members leave and join between runs (no recapture);
    every replica still follows its lone trajectory."""
    ref = [_alone(s, 400 + k, 30) for k, s in enumerate(replicas)]
    ctxs = [nb.Context(0) for _ in replicas]
    systems = [_prep(c, s, 400 + k) for k, (c, s) in enumerate(zip(ctxs, replicas))]
    b = Batch(ctx, systems[:2])
    b.set_segment(5)
    b.run(10)                       # replicas 0, 1: 10 steps
    b.set_systems(systems[1:])      # 0 leaves, 2 joins
    b.run(20)                       # replica 1: 30 steps, replica 2: 20
    b.set_systems([systems[0], systems[2]])
    b.run(10)                       # replica 0: 20, replica 2: 30
    b.set_systems([systems[0]])
    b.run(10)                       # replica 0: 30
    for k, m in enumerate(systems):
        assert np.array_equal(m.get_state()[0], ref[k][0]), k
    b.close()
    for m in systems:
        m.close()
    for c in ctxs:
        c.close()


def test_segments_compose(ctx, replicas):
    s = replicas[0]
    a = _prep(ctx, s, 5)
    a.md_run(30)
    a.md_run(30)
    b = _prep(ctx, s, 5)
    b.md_run(60)
    assert np.array_equal(a.get_state()[0], b.get_state()[0])
    a.close()
    b.close()


def test_autotune_returns_a_candidate(ctx, replicas):
    best, times = autotune_margin(ctx, replicas[1], margins=(0.4, 0.8), steps=10, cut=8.0)
    assert best in (0.4, 0.8) and all(t > 0 for t in times.values())
    best, times = autotune(ctx, replicas[1], aspects=(0.8, 1.0), margins=(0.5,), steps=10,
                           cut=8.0)
    assert best in times and best[1] == 0.5 and all(t > 0 for t in times.values())
    m = M.System(ctx, replicas[1], cut=8.0, skin=2.0)
    with pytest.raises(Exception):
        set_margin(m, 5.0)  # larger than the skin
    m.close()


def test_server_serves_and_continues(replicas):
    srv = Server(max_active=2, hbm_budget=1 << 30, chunk_steps=20, cut=8.0,
                 dt=1.0, gamma=0.01, warm_in=0)
    reqs = [Request(k, 0.0, s, 40) for k, s in enumerate(replicas)]
    reqs.append(Request(10, 0.0, replicas[0], 20, continues=0))
    stats = run_stream(srv, reqs)
    assert stats["requests"] == 4
    got = {r.rid: r for r in srv.results}
    assert set(got) == {0, 1, 2, 10}
    assert all(r.cluster_size >= 0 and r.latency > 0 for r in srv.results)
    # the continuation resumed replica 0: its state equals 60 steps run alone
    cont = srv.parked[10]
    x_served = cont.system.get_state()[0]
    srv.close()
    c = nb.Context(0)
    m = M.System(c, replicas[0], cut=8.0, skin=2.0)
    m.set_state(replicas[0].xyz.astype(np.float64), replicas[0].velocity.astype(np.float64))
    m.md_setup(replicas[0], dt=1.0, gamma=0.01, seed=1000003 * 1)
    m.md_run(60)
    assert np.array_equal(m.get_state()[0], x_served)
    m.close()
    c.close()


def test_resident_cluster_analysis_equals_host_path(ctx):
    """get_greatestCluster on the device-resident positions equals the host-fed
    call on the same (wrapped real*4) positions; a seeded crystalline nucleus
    takes the analysis's real branch (solid molecules, greatest label > 0)."""
    from molecular_simulation_code_b200.nonbond import get_greatest_cluster
    s = make_system(60, 1500, 5, nucleus=40)
    m = M.System(ctx, s, cut=8.0, skin=2.0)
    m.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    m.md_setup(s, dt=1.0, gamma=0.02, seed=9)
    m.md_run(20)
    x, _, _ = m.get_state()
    L = float(s.box)
    w = (x - L * np.floor(x / L)).astype(np.float32)
    w[w <= 0] += np.float32(L)
    pos = s.position_aos().copy()
    pos[:, :3] = w
    gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
    mrcut, denscut, densmin = 9.0, 6.0, 11
    ptta_h = s.xyz[:10 * s.n_gly].astype(np.float64).copy()
    ptta_d = ptta_h.copy()
    size_h, g_h, dens, _ = get_greatest_cluster(ctx, pos, gid, s.n_gly, 10, s.box, mrcut, denscut,
                                                densmin, ptta_h, 0)
    size_d, g_d = m.greatest_cluster(s.n_gly, mrcut, denscut, densmin, greatest=0, ptta=ptta_d)
    assert (size_d, g_d) == (size_h, g_h)
    assert np.array_equal(ptta_d, ptta_h)
    assert (np.asarray(dens) >= densmin).sum() > 0 and g_h > 0 and size_h > 0
    # the system's own device copy of ptta (set from the current positions)
    size_r, g_r = m.greatest_cluster(s.n_gly, mrcut, denscut, densmin, greatest=0)
    assert size_r > 0 and g_r > 0
    assert m.device_bytes() > 0
    m.close()


def test_server_warm_in_inside_batch_and_nucleus(replicas):
    """Warm-in runs inside the batch (admission does not step the replica), every
    request finishes with the device cluster analysis, and a nucleus-seeded request
    reports a non-trivial cluster; the batch graphs are captured once."""
    nuc = make_system(60, 1500, 5, nucleus=40)
    srv = Server(max_active=3, hbm_budget=1 << 30, chunk_steps=20, cut=8.0, dt=1.0,
                 gamma=0.01, warm_in=10, segment_graph=10)
    reqs = [Request(0, 0.0, nuc, 40), Request(1, 0.0, replicas[1], 60),
            Request(2, 0.01, replicas[2], 20)]
    stats = run_stream(srv, reqs)
    assert stats["requests"] == 3 and srv.recaptures == 1
    got = {r.rid: r for r in srv.results}
    assert got[0].cluster_size > 0
    assert all(r.latency >= r.service > 0 for r in srv.results)
    srv.close()


def test_cluster_shape_keeps_forces_and_coverage(ctx):
    """Taller or flatter clusters (the tuner's geometry knob) change the list, not the
    physics: FP64 forces and energies agree within 1e-10 relative, and the pruned list
    still holds every pair within rc."""
    from scipy.spatial import cKDTree
    s = make_system(150, 2500, 1)
    ref = None
    for aspect in (1.0, 0.8, 1.25):
        m = M.System(ctx, s, cut=10.0, skin=2.0, precision=M.FP64)
        if aspect != 1.0:
            set_cluster_shape(m, aspect)
        m.set_state(s.xyz.astype(np.float64))
        e = m.compute(M.FP64, rebuild=True)
        f = m.get_state()[2]
        pairs, _ = m.list_pairs(1)
        n = s.np_atoms
        keys = np.unique(np.minimum(pairs[:, 0], pairs[:, 1]).astype(np.int64) * n +
                         np.maximum(pairs[:, 0], pairs[:, 1]))
        L = float(s.box)
        xw = np.mod(s.xyz.astype(np.float64), L)
        pr = cKDTree(xw, boxsize=L).query_pairs(10.0, output_type="ndarray").astype(np.int64)
        need = pr.min(axis=1) * n + pr.max(axis=1)
        excl = {min(i, int(j) - 1) * n + max(i, int(j) - 1)
                for i in range(n) for j in s.specbond[i, :s.num3bond[i]] if j > 0}
        need = np.setdiff1d(need, np.array(sorted(excl), np.int64))
        assert np.isin(need, keys).all(), aspect
        if ref is None:
            ref = (e, f)
        else:
            assert M.force_max_rel(f, ref[1]) <= 1e-10, aspect
            assert abs(e[0] - ref[0][0]) <= 1e-10 * abs(ref[0][0])
            assert abs(e[1] - ref[0][1]) <= 1e-10 * abs(ref[0][1])
        m.close()
