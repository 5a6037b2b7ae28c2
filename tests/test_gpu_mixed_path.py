"""GPU tests of the production cluster-pair path (mixed FP32/fixed-point and FP64).

Bars (stated here and in the design notes):
  * FP64 cluster kernel vs the oracle's FP64 list forces: 1e-10 relative
    (max |df| / max |f|) and 1e-10 relative on potential and e_coul;
  * mixed vs FP64: force RMS relative error <= 1e-6 (sqrt(sum|df|^2/sum|f|^2));
  * mixed forces are bit-identical run to run and under relabelling of atoms.
"""
import numpy as np
import pytest

from helpers import small_system
from molecular_simulation_code_b200 import mixed as M
from molecular_simulation_code_b200.system import make_system
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _oracle_forces(s, cut, pad, alpha=0.2, n2=False):
    p = O.params(alpha, s.box, cut, cut, pad)
    pos = s.position_aos()
    if n2:
        nl, nn = O.neighbor_n2(p, pos, s.specbond, s.num3bond, 2048)
        na = 2048
    else:
        nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 1024)
    _, ff64, pot, ec, vir = O.force_dsf(p, pos, s.q, (s.lj1, s.lj2, s.lj3, s.lj4), s.ntypes,
                                        nl, nn, na)
    return ff64, pot, ec, vir


@pytest.fixture(scope="module")
def sys9k():
    return make_system(150, 2500, 1)


def test_fp64_cluster_matches_oracle(ctx, sys9k):
    s = sys9k
    sysm = M.System(ctx, s, cut=10.0, skin=2.0, precision=M.FP64)
    sysm.set_state(s.xyz.astype(np.float64))
    e = sysm.compute(M.FP64, rebuild=True)
    _, _, f = sysm.get_state()
    ff64, pot, ec, vir = _oracle_forces(s, 10.0, 2.0)
    assert abs(e[0] - pot) <= 1e-10 * abs(pot)
    assert abs(e[1] - ec) <= 1e-10 * abs(ec)
    assert M.force_max_rel(f, ff64) <= 1e-10
    assert np.abs(e[2:] - vir).max() <= 1e-9 * np.abs(vir).max()
    sysm.close()


def test_mixed_error_vs_fp64(ctx, sys9k):
    s = sys9k
    sysm = M.System(ctx, s, cut=10.0, skin=2.0)
    sysm.set_state(s.xyz.astype(np.float64))
    e64 = sysm.compute(M.FP64, rebuild=True)
    _, _, f64 = sysm.get_state()
    e32 = sysm.compute(M.MIXED)
    _, _, f32 = sysm.get_state()
    rms = M.force_rms_rel(f32, f64)
    print("force rms rel", rms, "max rel", M.force_max_rel(f32, f64))
    assert rms <= 1e-6
    assert abs(e32[0] - e64[0]) <= 1e-5 * abs(e64[0]) + 1e-3
    assert abs(e32[1] - e64[1]) <= 1e-5 * abs(e64[1])
    sysm.close()


def test_mixed_bit_reproducible_and_label_independent(ctx, sys9k):
    s = sys9k
    sysm = M.System(ctx, s, cut=10.0, skin=2.0)
    x = s.xyz.astype(np.float64)
    sysm.set_state(x)
    ea = sysm.compute(rebuild=True)
    _, _, fa = sysm.get_state()
    eb = sysm.compute(rebuild=True)
    _, _, fb = sysm.get_state()
    assert np.array_equal(fa, fb) and np.array_equal(ea, eb)
    sysm.close()
    # relabel the atoms (permute every per-atom array and the exclusion ids)
    perm = np.random.default_rng(5).permutation(s.np_atoms)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(s.np_atoms)
    import copy
    t = copy.copy(s)
    t.xyz = s.xyz[perm]
    t.types = s.types[perm]
    t.q = s.q[perm]
    sb = s.specbond[perm].copy()
    nz = sb > 0
    sb[nz] = inv[sb[nz] - 1] + 1
    t.specbond = sb
    t.num3bond = s.num3bond[perm]
    sysp = M.System(ctx, t, cut=10.0, skin=2.0)
    sysp.set_state(t.xyz.astype(np.float64))
    ep = sysp.compute(rebuild=True)
    _, _, fp = sysp.get_state()
    assert np.array_equal(fp, fa[perm])
    assert ep[0] == pytest.approx(ea[0], rel=1e-12) and ep[1] == pytest.approx(ea[1], rel=1e-12)
    sysp.close()


def test_dropin_host_buffers_equal_resident(ctx):
    s = small_system(20, 1200, 4)
    sysm = M.System(ctx, s, cut=8.0, skin=2.0)
    pos = s.position_aos()
    ff, pot, ec, vir = sysm.forces_dropin(pos)
    sysm.set_state(pos[:, :3].astype(np.float64))
    e = sysm.compute(rebuild=True)
    _, _, f = sysm.get_state()
    assert np.array_equal(ff, f.astype(np.float32))
    assert pot == e[0] and ec == e[1]
    sysm.close()


def test_dropin_graph_equals_host_driven_sequence(ctx):
    """After the first call the drop-in runs as one captured graph (rebuild and
    prune decided on the device); with timers on it stays host-driven.  Over a
    drifting trajectory with rebuilds both give identical forces and energies."""
    s = small_system(20, 1200, 4)
    a = M.System(ctx, s, cut=8.0, skin=2.0)
    b = M.System(ctx, s, cut=8.0, skin=2.0)
    b.timers(True)
    pos = s.position_aos().copy()
    v = s.velocity.astype(np.float32) * np.float32(40.0)  # ~0.5 A per call for fast atoms
    for k in range(25):
        fa, pa, ea, _ = a.forces_dropin(pos)
        fb, pb, eb, _ = b.forces_dropin(pos)
        assert np.array_equal(fa, fb) and pa == pb and ea == eb, k
        pos[:, :3] += v
    sa, sb = a.stats(), b.stats()
    assert sa["builds"] == sb["builds"] and sa["builds"] >= 3
    assert sa["prunes"] == sb["prunes"]
    a.close()
    b.close()


def test_rebuild_trigger_and_wrapped_positions(ctx):
    s = small_system(20, 1200, 4)
    sysm = M.System(ctx, s, cut=8.0, skin=2.0)
    pos = s.position_aos()
    f0, p0, e0, _ = sysm.forces_dropin(pos)
    b0 = sysm.stats()["builds"]
    # wrapping atoms by a box length changes nothing and does not rebuild
    w = pos.copy()
    L = np.float32(s.box)
    sel = w[:, 0] > L / 2
    w[sel, 0] = w[sel, 0] - L
    f1, p1, e1, _ = sysm.forces_dropin(w)
    assert sysm.stats()["builds"] == b0
    assert M.force_max_rel(f1, f0) < 1e-5
    # small moves (< skin/2) reuse the list; forces match a fresh build
    rng = np.random.default_rng(2)
    m = pos.copy()
    m[:, :3] += rng.uniform(-0.5, 0.5, (s.np_atoms, 3)).astype(np.float32) * 0.9 / np.sqrt(3)
    f2, p2, _, _ = sysm.forces_dropin(m)
    assert sysm.stats()["builds"] == b0
    fresh = M.System(ctx, s, cut=8.0, skin=2.0)
    f3, p3, _, _ = fresh.forces_dropin(m)
    assert M.force_max_rel(f2, f3) < 1e-5
    assert p2 == pytest.approx(p3, rel=1e-6)
    # a move beyond skin/2 rebuilds
    m[0, :3] += np.float32(1.5)
    sysm.forces_dropin(m)
    assert sysm.stats()["builds"] == b0 + 1
    sysm.close()
    fresh.close()


def test_small_box_images(ctx):
    """L ~ 27 A with rc = 10 A: every pair within rc counted once (minimum image)."""
    s = make_system(20, 600, 8)
    assert float(s.box) < 30.0
    sysm = M.System(ctx, s, cut=10.0, skin=2.0, precision=M.FP64)
    sysm.set_state(s.xyz.astype(np.float64))
    e = sysm.compute(M.FP64, rebuild=True)
    _, _, f = sysm.get_state()
    ff64, pot, ec, _ = _oracle_forces(s, 10.0, 2.0, n2=True)
    assert M.force_max_rel(f, ff64) <= 1e-10
    assert abs(e[0] - pot) <= 1e-10 * abs(pot) and abs(e[1] - ec) <= 1e-10 * abs(ec)
    sysm.close()


def _pairs_within(x, box, r):
    """All unordered atom pairs within r (minimum image) as sorted int64 keys i*N + j, i < j."""
    from scipy.spatial import cKDTree
    L = float(box)
    xw = np.mod(np.asarray(x, np.float64), L)
    xw[xw >= L] = 0.0
    pr = cKDTree(xw, boxsize=L).query_pairs(r, output_type="ndarray").astype(np.int64)
    n = x.shape[0]
    return np.unique(pr.min(axis=1) * n + pr.max(axis=1))


def _list_keys(pairs, n):
    a, b = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64)
    return np.minimum(a, b) * n + np.maximum(a, b)


def _excluded_keys(s):
    n = s.np_atoms
    ks = []
    for i in range(n):
        for l in range(int(s.num3bond[i])):
            j = int(s.specbond[i, l]) - 1
            if j >= 0:
                ks.append(min(i, j) * n + max(i, j))
    return np.unique(np.array(ks, np.int64))


def test_list_covers_every_pair_within_rlist(ctx):
    """The cluster lists, expanded into atom pairs, hold every non-excluded pair
    once: the outer list every pair within rc + skin at its build positions, the
    pruned list every pair within rc + margin at its prune positions and every
    pair within rc at the current positions, after a rebuild and along a
    drifting trajectory with several prunes and rebuilds."""
    s = make_system(150, 2500, 1)
    n = s.np_atoms
    from molecular_simulation_code_b200.batch import set_margin
    cut, skin, margin = 10.0, 2.0, 0.4
    sysm = M.System(ctx, s, cut=cut, skin=skin, precision=M.MIXED)
    set_margin(sysm, margin)
    sysm.set_state(s.xyz.astype(np.float64), s.velocity.astype(np.float64))
    sysm.md_setup(s, dt=2.0, temperature=300.0, gamma=0.01, seed=4)
    sysm.compute(M.MIXED, rebuild=True, energy=False, virial=False)
    excl = _excluded_keys(s)
    st0 = sysm.stats()
    checks = 0
    for seg in range(6):
        x, _, _ = sysm.get_state()
        outer, xo = sysm.list_pairs(0)
        inner, xi = sysm.list_pairs(1)
        ko, ki = _list_keys(outer, n), _list_keys(inner, n)
        # each pair at most once, never an excluded (1-2, 1-3, 1-4) or self pair
        assert np.unique(ko).size == ko.size and np.unique(ki).size == ki.size
        assert not np.isin(ko, excl).any() and not np.isin(ki, excl).any()
        assert (outer[:, 0] != outer[:, 1]).all()
        assert np.isin(ki, ko).all()  # the pruned list is a subset of the outer list
        need_o = np.setdiff1d(_pairs_within(xo, s.box, cut + skin), excl)
        need_i = np.setdiff1d(_pairs_within(xi, s.box, cut + margin), excl)
        need_c = np.setdiff1d(_pairs_within(x, s.box, cut), excl)
        assert np.isin(need_o, ko).all(), np.setdiff1d(need_o, ko)[:5]
        assert np.isin(need_i, ki).all(), np.setdiff1d(need_i, ki)[:5]
        assert np.isin(need_c, ki).all(), np.setdiff1d(need_c, ki)[:5]
        checks += 1
        sysm.md_run(40)
    st = sysm.stats()
    assert checks == 6
    assert st["prunes"] - st0["prunes"] >= 3 and st["builds"] - st0["builds"] >= 1, (st0, st)
    sysm.close()
