"""CPU tests of the oracle itself: the restatement is self-consistent.

The reference ships no golden vectors (parity unpinned), so the oracle is
pinned by independent cross-checks: the cell-list build against the O(N^2)
build, the list-based forces (+1-4 pairs) against the O(N^2) kernel with its
in-loop exclusion weights (Source/mod_force_nonbond.f90:409-502), Newton's
third law, finite differences of the energy, and hand-checked structural
facts of the stencil and sort.
"""
import math

import numpy as np
import pytest

from helpers import pair_set, rel_err, small_system
from oracle import oracle as O


def _p(s, cut=7.0, pad=1.5, alpha=0.2):
    return O.params(alpha, s.box, cut, cut, pad)


def test_constants_precision_archaeology():
    p = O.params(0.22, 77.61, 12.0, 12.0, 1.5)
    assert p.EWALD_P == float(np.float32(0.3275911))
    assert p.MY_PIS == float(np.float32(1.77245385090551602729))
    assert p.MY_PIS != math.sqrt(math.pi)
    assert p.coulpre == float(np.float32(332.06371))
    # e_shift/f_shift from the defining formulas (get_started.f90:112-116)
    cc = 12.0
    erfcc = math.erfc(0.22 * cc)
    erfcd = math.exp(-(0.22 * 0.22 * cc * cc))
    fs = -(erfcc / 144.0 + 2.0 / p.MY_PIS * 0.22 * erfcd / cc)
    assert p.f_shift == pytest.approx(fs, rel=1e-15)
    assert p.e_shift == pytest.approx(erfcc / cc - fs * cc, rel=1e-15)
    assert p.rv2 == float(np.float32(13.5)) ** 2


def test_stencil_structure():
    for nd in (3, 4, 5):
        nt = nd ** 3
        c = O.stencil(nt, nd).reshape(nt, 27)
        assert np.array_equal(c[:, 0], np.arange(nt))
        for ic in range(nt):
            assert len(set(c[ic].tolist())) == 27
        # symmetric neighbourhood
        for ic in range(nt):
            for jc in c[ic]:
                assert ic in c[jc]


def test_bin_sort_is_lifo_cell_order():
    s = small_system()
    p = _p(s)
    pos = s.position_aos()
    tt, ttb, st, en, ab = O.bin_sort(p, pos)
    assert np.array_equal(np.sort(ttb), np.arange(1, s.np_atoms + 1))
    assert np.array_equal(tt[ttb - 1], np.arange(1, s.np_atoms + 1))
    assert np.all(np.diff(ab) >= 0)
    for c in range(len(st)):
        members = ttb[st[c] - 1:en[c]]
        assert np.all(np.diff(members) < 0)  # head-of-chain order: descending input index


def test_cell_list_equals_n2_list_for_small_box():
    s = small_system()
    p = _p(s)
    pos = s.position_aos()
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512)
    nl2, nn2 = O.neighbor_n2(p, pos, s.specbond, s.num3bond, na)
    assert pair_set(nl, nn, na) == pair_set(nl2, nn2, na)


def test_cell_list_misses_skin_pairs_when_cells_are_cut_sized():
    """With rn sized from the cutoff (not cutoff+skin) the 27-cell stencil misses
    pairs with rn < r < rv in non-adjacent cells, as the reference does."""
    s = small_system(20, 1200, 9)
    p = O.params(0.2, s.box, 8.0, 8.0, 3.0)
    _, _, nd = O.cell_grid(p)
    assert nd >= 4
    pos = s.position_aos()
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 1024)
    nl2, nn2 = O.neighbor_n2(p, pos, s.specbond, s.num3bond, na)
    a = pair_set(nl, nn, na)
    b = pair_set(nl2, nn2, na)
    assert a < b
    # every missed pair lies beyond the cutoff (forces at build time are complete)
    x = pos[:, :3].astype(np.float64)
    L = float(s.box)
    for i, j in list(b - a)[:2000]:
        d = x[i - 1] - x[j - 1]
        d -= L * np.round(d / L)
        assert np.linalg.norm(d) > 8.0


def test_list_forces_plus_14_equal_n2_forces():
    s = small_system()
    p = _p(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512)
    ff, ff64, pot, ec, vir = O.force_dsf(p, pos, s.q, lj, s.ntypes, nl, nn, na)
    ffh, ed, ec14, p14 = O.dihedral_opls_dsf(p, pos, s.q, s.ntypes, s.lj14, s.dihedrals,
                                             s.dihed_coeff)
    f2, pot2, ec2 = O.force_dsf_n2(p, pos, s.q, lj, s.ntypes, s.specbond, s.num1bond,
                                   s.num2bond, s.num3bond)
    # ffh is real*4 (rounded after every dihedral) and 1-4 displacements are real*4 differences
    assert rel_err(ff64 + ffh, f2) < 5e-7
    # 1-4 prefactor coulpre*q*q is a real*4 product there (mod_force_dihed.f90:1010)
    assert pot + p14 == pytest.approx(pot2, rel=1e-7)
    assert ec + ec14 == pytest.approx(ec2, rel=1e-7)
    assert np.abs(ff64.sum(axis=0)).max() < 1e-9 * np.abs(ff64).max() * s.np_atoms
    assert np.array_equal(ff, ff64.astype(np.float32))


def test_force_is_minus_energy_gradient():
    s = small_system(2, 100, 11)
    p = _p(s, cut=6.0, pad=2.0)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512)
    _, ff64, _, _, _ = O.force_dsf(p, pos, s.q, lj, s.ntypes, nl, nn, na)
    # LJ is truncated, not shifted (mod_force_nonbond.f90:155): skip atoms with a
    # neighbour within 0.004 A of the cutoff, where the energy jumps
    x = pos[:, :3].astype(np.float64)
    L = float(s.box)
    ok = []
    for i in range(s.np_atoms):
        d = x[i] - x
        d -= L * np.round(d / L)
        r = np.linalg.norm(d, axis=1)
        if not np.any(np.abs(r - 6.0) < 0.004):
            ok.append(i)
    rng = np.random.default_rng(0)
    for i in rng.choice(ok, 5, replace=False):
        for c in range(3):
            h = 1e-3
            e = []
            for sgn in (1, -1):
                q = pos.copy()
                q[i, c] = np.float32(q[i, c] + sgn * h)
                _, _, pp, ee, _ = O.force_dsf(p, q, s.q, lj, s.ntypes, nl, nn, na)
                e.append(pp + ee)
            hh = float(np.float32(pos[i, c] + h)) - float(np.float32(pos[i, c] - h))
            fd = -(e[0] - e[1]) / hh
            assert ff64[i, c] == pytest.approx(fd, rel=2e-2, abs=2e-2)


def test_thread_count_does_not_change_results():
    s = small_system()
    p = _p(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    a = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512, nthreads=1)
    b = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512, nthreads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    fa = O.force_dsf(p, pos, s.q, lj, s.ntypes, *a, nthreads=1)
    fb = O.force_dsf(p, pos, s.q, lj, s.ntypes, *a, nthreads=4)
    assert np.array_equal(fa[0], fb[0]) and fa[2] == fb[2] and fa[3] == fb[3]


def test_e_self_formula():
    s = small_system()
    p = _p(s)
    e = O.e_self(p, s.q)
    ref = -sum((0.5 * p.e_shift + p.alpha / p.MY_PIS) * float(q) * float(q) * p.coulpre
               for q in s.q)
    assert e == pytest.approx(ref, rel=1e-12)


def test_gewald_bisection():
    g = O.calculate_gewald(12.0)
    assert math.erfc(g * 12.0) / 12.0 == pytest.approx(float(np.float32(1e-6)), rel=1e-6)


def test_shake_satisfies_constraints():
    s = small_system(4, 40, 13)
    x = s.xyz.astype(np.float64)
    v = s.velocity.astype(np.float64)
    f = np.random.default_rng(1).normal(0, 5.0, x.shape)
    m = s.mass_type[s.types - 1]
    dt, k2a = 2.0, float(np.float32(0.0004184))
    fn, st = O.shake(x, v, f, m, float(s.box), s.shake, s.shake_bond, dt, k2a,
                     tolerance=1e-10, maxiter=200)
    assert st == 0
    xs = x + dt * v + dt * dt * k2a * fn / m[:, None]
    L = float(s.box)
    for g, b in zip(s.shake, s.shake_bond):
        num, a = g[0], g[1:] - 1
        pairs = {1: [(0, 1)], 3: [(0, 1), (0, 2)], 4: [(0, 1), (0, 2), (0, 3)],
                 -3: [(0, 1), (0, 2), (1, 2)]}[int(num)]
        for k, (u, w) in enumerate(pairs):
            d = xs[a[u]] - xs[a[w]]
            d -= L * np.round(d / L)
            assert np.linalg.norm(d) == pytest.approx(b[k], abs=1e-6)


def _cluster_positions(seed=1, n_gly=27, spacing=5.0):
    from molecular_simulation_code_b200.system import make_system
    s = make_system(n_gly, 600, seed)
    pos = s.position_aos()
    L = float(s.box)
    g = pos[:10 * n_gly, :3].reshape(n_gly, 10, 3).astype(np.float64)
    g = g - L * np.round((g - g[:, :1, :]) / L)  # unwrap each molecule about its atom 1
    g = g - g.mean(axis=1, keepdims=True)
    k = round(n_gly ** (1 / 3))
    sites = np.array([(i, j, l) for i in range(k) for j in range(k) for l in range(k)])
    centres = 5.0 + sites * spacing
    pos[:10 * n_gly, :3] = (g + centres[:, None, :]).reshape(-1, 3).astype(np.float32)
    return s, pos


def test_cluster_known_answer_simple_cubic():
    """27 glycines on a 3x3x3 simple-cubic block at 5 A spacing, denscut 6 A:
    interior/face/edge/corner molecules have 6/5/4/3 neighbours."""
    s, pos = _cluster_positions()
    gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
    box = s.box
    ibox = np.float32(1.0 / np.float64(box))
    vol = np.float32(np.float32(box * box) * box)
    # the atom with global id n_gly*10 is never refreshed (mod_build_ptta.f90:127):
    # start it at its true position so every centre is exact
    ptta = pos[:270, :3].astype(np.float64)
    # densmin 4: corners (3 neighbours) are non-solid surface molecules
    size, g, dens, bel = O.greatest_cluster(pos, gid, 27, 10, box, ibox, vol, 9.0, 6.0, 4, ptta)
    counts = sorted(dens.tolist())
    assert counts == [3] * 8 + [4] * 12 + [5] * 6 + [6]
    assert g == 1 and size == 27  # 19 solid + 8 corner surface molecules
    size, g, dens, bel = O.greatest_cluster(pos, gid, 27, 10, box, ibox, vol, 9.0, 6.0, 7, ptta,
                                            greatest_in=9)
    assert size == 0 and g == 9  # no solid molecule; caller's label matches nothing
    size, g, dens, bel = O.greatest_cluster(pos, gid, 27, 10, box, ibox, vol, 9.0, 6.0, 7, ptta,
                                            greatest_in=0)
    assert size == 27 and g == 0  # label 0 matches every unclustered molecule


def test_cluster_stale_last_atom_quirk():
    """build_ptta_wrap_cluster2 never refreshes the atom with id == n_gly*10."""
    s, pos = _cluster_positions()
    gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
    box = s.box
    ibox = np.float32(1.0 / np.float64(box))
    vol = np.float32(np.float32(box * box) * box)
    ptta = np.full((270, 3), 1.0)
    O.greatest_cluster(pos, gid, 27, 10, box, ibox, vol, 9.0, 6.0, 4, ptta)
    assert np.all(np.isclose(ptta[:269], pos[:269, :3], atol=1e-4) |
                  np.isclose(np.abs(ptta[:269] - pos[:269, :3]), float(box), atol=1e-3))
    assert not np.allclose(ptta[269], pos[269, :3], atol=1e-3)


def _long_fp64(p, pos, q, lj, ntypes, nl, nn, na, g, cut):
    """Independent FP64 real-space Ewald + LJ with the exact erfc, over the list."""
    from scipy.special import erfc
    x = pos[:, :3].astype(np.float64)
    t = pos[:, 3].view(np.int32) - 1
    L = float(p.box)
    n = x.shape[0]
    ii = np.repeat(np.arange(n), nn)
    jj = np.concatenate([nl[i * na:i * na + nn[i]] for i in range(n)]) - 1
    d = x[ii] - x[jj]
    d -= L * np.round(d / L)
    r2 = (d * d).sum(axis=1)
    r = np.sqrt(r2)
    off = t[ii] * ntypes + t[jj]
    dr6i = np.where(r2 > cut * cut, 0.0, 1.0 / r2 ** 3)
    flj = dr6i * (lj[0][off] * dr6i - lj[1][off])
    elj = dr6i * (dr6i * lj[2][off] - lj[3][off])
    pref = np.where(r2 > cut * cut, 0.0, float(p.coulpre) * q[ii].astype(np.float64) * q[jj] / r)
    ec = pref * erfc(g * r)
    fc = pref * (erfc(g * r) + 2.0 / math.sqrt(math.pi) * g * r * np.exp(-(g * r) ** 2))
    fr = (fc + flj) / r2
    f = np.zeros((n, 3))
    np.add.at(f, ii, d * fr[:, None])
    return f, 0.5 * elj.sum(), 0.5 * ec.sum(), 0.5 * np.abs(ec).sum()


def test_long_range_real_space_vs_exact_fp64():
    """The real*4 restatement with the A&S 7.1.26 erfc (|error| <= 1.5e-7) against
    an FP64 evaluation with the exact erfc: real*4-level agreement."""
    s = small_system()
    p = _p(s, cut=7.0, pad=1.5)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    g = O.calculate_gewald(7.0)
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512)
    ff, ff64, pot, ec, vir = O.force_long(p, pos, s.q, lj, s.ntypes, nl, nn, na, g)
    f_ref, pot_ref, ec_ref, ec_abs = _long_fp64(p, pos, s.q, lj, s.ntypes, nl, nn, na, g, 7.0)
    assert pot == pytest.approx(pot_ref, rel=1e-5)
    # e_coul cancels strongly; bound its error by the sum of |pair terms|
    assert abs(ec - ec_ref) <= 1e-5 * ec_abs
    assert rel_err(ff64, f_ref) < 1e-5
    assert np.array_equal(ff, ff64.astype(np.float32))
    # the full list holds each pair twice: the net force vanishes to rounding
    assert np.abs(ff64.sum(axis=0)).max() < 1e-4 * np.abs(ff64).max()


def test_long_range_thread_count_invariant():
    s = small_system()
    p = _p(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    g = O.calculate_gewald(7.0)
    a = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 512)
    fa = O.force_long(p, pos, s.q, lj, s.ntypes, *a, g, nthreads=1)
    fb = O.force_long(p, pos, s.q, lj, s.ntypes, *a, g, nthreads=4)
    assert np.array_equal(fa[0], fb[0]) and fa[2] == fb[2] and fa[3] == fb[3]


def test_product_gewald_equals_oracle():
    from molecular_simulation_code_b200.nonbond import calculate_gewald
    for c in (8.0, 9.5, 10.0, 12.0):
        assert calculate_gewald(c) == O.calculate_gewald(c)


def test_improper_energy_gradient_and_rest_angle():
    """improper_harmonic_lammps14 restatement: zero energy at omega0, forces equal
    minus the finite-difference gradient of the energy, zero net force."""
    from molecular_simulation_code_b200.system import improper_omega
    s = small_system(4, 30, 9)
    p = _p(s)
    pos = s.position_aos()
    il = s.impropers
    om = improper_omega(pos[:, :3], float(s.box), il[:, :4] - 1)
    coeff = np.array([[1.1, 0.0]])
    _, e_rest, _ = O.improper_harmonic(p, pos, il[:1], np.array([[1.1, om[0]]]))
    assert abs(e_rest) < 1e-9
    rng = np.random.default_rng(2)
    pos2 = pos.copy()
    pos2[:40, :3] += rng.normal(0, 0.15, (40, 3)).astype(np.float32)
    f, e, vir = O.improper_harmonic(p, pos2, il, coeff)
    assert e > 0 and np.isfinite(vir).all()
    assert np.abs(f.sum(axis=0)).max() < 1e-4
    for i in (0, 1, 3, 4, 13):
        for c in range(3):
            h = 2e-3
            ee = []
            for sgn in (1, -1):
                q = pos2.copy()
                q[i, c] = np.float32(q[i, c] + sgn * h)
                ee.append(O.improper_harmonic(p, q, il, coeff)[1])
            hh = float(np.float32(pos2[i, c] + h)) - float(np.float32(pos2[i, c] - h))
            assert f[i, c] == pytest.approx(-(ee[0] - ee[1]) / hh, rel=2e-2, abs=2e-3)
