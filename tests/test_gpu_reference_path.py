"""GPU parity of the reference-semantics path against the oracle (C restatement).

Bar: bit-exact neighbour sets and rows, bit-exact integer cell sort and cluster
sizes; FP64 accumulators within 1e-10 relative; real*4 outputs within a few
real*4 ulps (the reference rounds its FP64 sums to real*4 at the end).
"""
import numpy as np
import pytest

from helpers import pair_set, ref_params, rel_err, rows, small_system
from molecular_simulation_code_b200 import nonbond as nb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _orc_params(p):
    return O.params(p.alpha, p.box, p.cut_coul, p.rcut, p.neighbor_pad)


def test_dsf_constants_match_oracle():
    s = small_system()
    p = ref_params(s)
    op = _orc_params(p)
    assert p.e_shift == op.e_shift and p.f_shift == op.f_shift
    assert p.rv2 == op.rv2 and float(p.ibox) == op.ibox


def test_cell_sort_exact(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    tt, ttb, st, en, ab, ps = nb.cell_sort(ctx, pos, p)
    ott, ottb, ost, oen, oab = O.bin_sort(_orc_params(p), pos)
    assert np.array_equal(tt, ott)
    assert np.array_equal(ttb, ottb)
    assert np.array_equal(st, ost)
    assert np.array_equal(en, oen)
    assert np.array_equal(ab, oab)
    assert np.array_equal(ps.view(np.int32), pos[ottb - 1].view(np.int32))


@pytest.mark.parametrize("cut,pad", [(7.0, 1.5), (5.0, 2.0), (10.0, 1.5)])
def test_neighbor_list_sets_bit_exact(ctx, cut, pad):
    s = small_system()
    p = ref_params(s, cut=cut, pad=pad)
    pos = s.position_aos()
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, neigh_alloc=64)
    onl, onn, ona = O.neighbor_wrapper(_orc_params(p), pos, s.specbond, s.num3bond, 64)
    assert na == ona
    assert np.array_equal(nn, onn)
    assert pair_set(nl, nn, na) == pair_set(onl, onn, ona)


def test_neighbor_rows_exact_on_sorted_input(ctx):
    """On reference-sorted arrays the rows equal the reference's, entry by entry."""
    s = small_system()
    p = ref_params(s)
    op = _orc_params(p)
    pos = s.position_aos()
    tt, ttb, st, en, ab = O.bin_sort(op, pos)
    ps = np.ascontiguousarray(pos[ttb - 1])
    sb = np.zeros_like(s.specbond)
    for snew in range(s.np_atoms):
        o = ttb[snew] - 1
        k = s.num3bond[o]
        sb[snew, :k] = tt[s.specbond[o, :k] - 1]
    n3 = np.ascontiguousarray(s.num3bond[ttb - 1])
    _, nt, nd = O.cell_grid(op)
    cnum = O.stencil(nt, nd)
    onl, onn, mx = O.build_neighbor_sorted(op, ps, ab, st, en, cnum, sb, n3, 512)
    nl, nn, na = nb.neighbor_wrapper(ctx, ps, sb, n3, p, neigh_alloc=512)
    assert mx <= 512 and na == 512
    assert rows(nl, nn, na) == rows(onl, onn, 512)


def test_neighbor_redo_loop_grows(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, neigh_alloc=16)
    assert na % 16 == 0 and na >= nn.max()
    assert na == int(nn.max() * 1.2) + (-int(nn.max() * 1.2)) % 16


def test_neighbor_small_box_duplicates_like_reference(ctx):
    """ncellD = 2: the reference stencil visits cells twice; rows match it exactly."""
    s = small_system(2, 60, 5)
    p = ref_params(s, cut=5.0, pad=1.0)
    _, _, nd = nb.cell_grid(p.box, p.cut_coul, p.rcut)
    assert nd == 2
    op = _orc_params(p)
    pos = s.position_aos()
    tt, ttb, st, en, ab = O.bin_sort(op, pos)
    ps = np.ascontiguousarray(pos[ttb - 1])
    sb = np.zeros_like(s.specbond)
    for snew in range(s.np_atoms):
        o = ttb[snew] - 1
        sb[snew, :s.num3bond[o]] = tt[s.specbond[o, :s.num3bond[o]] - 1]
    n3 = np.ascontiguousarray(s.num3bond[ttb - 1])
    _, nt, _ = O.cell_grid(op)
    onl, onn, mx = O.build_neighbor_sorted(op, ps, ab, st, en, O.stencil(nt, nd), sb, n3, 2048)
    nl, nn, na = nb.neighbor_wrapper(ctx, ps, sb, n3, p, neigh_alloc=2048)
    assert rows(nl, nn, na) == rows(onl, onn, 2048)


def test_force_fp64_matches_oracle(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    onl, onn, ona = O.neighbor_wrapper(_orc_params(p), pos, s.specbond, s.num3bond, 512)
    off, off64, opot, oec, ovir = O.force_dsf(_orc_params(p), pos, s.q, lj, s.ntypes, onl, onn,
                                              ona)
    ff, pot, ec, vir = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, onl, onn, ona, p)
    assert abs(pot - opot) <= FP64_TOL * abs(opot)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert rel_err(vir, ovir) <= FP64_TOL
    # ff is the real*4 rounding of FP64 sums: allow one real*4 ulp of the largest force
    ulp = np.spacing(np.abs(off).max())
    assert np.abs(ff - off).max() <= 2 * ulp


@pytest.mark.parametrize("cut,pad", [(7.0, 1.5), (5.0, 2.0)])
def test_force_long_matches_oracle(ctx, cut, pad):
    """Real-space Ewald (real*4 pair arithmetic): FP64 sums within 1e-10, real*4
    forces within two ulps of the largest force."""
    s = small_system()
    p = ref_params(s, cut=cut, pad=pad)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    g = nb.calculate_gewald(cut)
    onl, onn, ona = O.neighbor_wrapper(_orc_params(p), pos, s.specbond, s.num3bond, 512)
    off, _, opot, oec, ovir = O.force_long(_orc_params(p), pos, s.q, lj, s.ntypes, onl, onn,
                                           ona, g)
    ff, pot, ec, vir = nb.lj_cut_coul_long_nonewton(ctx, pos, s.q, lj, s.ntypes, onl, onn, ona,
                                                    p, g)
    assert abs(pot - opot) <= FP64_TOL * abs(opot)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert rel_err(vir, ovir) <= FP64_TOL
    assert np.abs(ff - off).max() <= 2 * np.spacing(np.abs(off).max())
    # resident list path gives the same result
    _, _, na2 = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 512, want_host=False)
    ff2, pot2, ec2, _ = nb.lj_cut_coul_long_nonewton(ctx, pos, s.q, lj, s.ntypes, None, None,
                                                     na2, p, g)
    assert abs(pot2 - opot) <= FP64_TOL * abs(opot) and abs(ec2 - oec) <= FP64_TOL * abs(oec)
    with pytest.raises(RuntimeError):
        nb.lj_cut_coul_long_nonewton(ctx, pos, s.q, lj, s.ntypes, onl, onn, ona, p, 0.0)


def test_force_resident_list_equals_host_list(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 512)
    ff1, pot1, ec1, _ = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, nl, nn, na, p)
    _, _, na2 = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 512, want_host=False)
    ff2, pot2, ec2, _ = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, None, None, na2,
                                                    p)
    assert np.array_equal(ff1, ff2) and pot1 == pot2 and ec1 == ec2


def test_force_run_to_run_bit_identical(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 512)
    a = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, nl, nn, na, p)
    b = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, nl, nn, na, p)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1] and a[2] == b[2]


def test_pair14_matches_oracle(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    dc = np.array([[0.3, -0.2, 0.15, 0.05], [0.0, 0.0, 0.1556, 0.0]])
    offh, oed, oec, op14 = O.dihedral_opls_dsf(_orc_params(p), pos, s.q, s.ntypes, s.lj14,
                                               s.dihedrals, dc)
    ffh, ed, ec, p14 = nb.dihedral_opls_dsf(ctx, pos, s.q, s.ntypes, s.lj14, s.dihedrals, dc, p)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert abs(p14 - op14) <= FP64_TOL * max(abs(op14), 1e-30)
    assert abs(ed - oed) <= 1e-9 * max(abs(oed), 1.0)
    # the reference rounds ffh to real*4 after every dihedral; the device rounds once
    assert rel_err(ffh, offh) <= 1e-6


def test_sort_permutations_match_reference(ctx):
    """sort_posit_charge / sort_specbond_numbond / sort_*list on the device equal
    their numpy restatements, with tt/ttb from the oracle's cell sort."""
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    tt, ttb, *_ = O.bin_sort(_orc_params(p), pos)
    ps = nb.sort_posit(ctx, ttb, pos)
    assert np.array_equal(ps.view(np.int32), pos[ttb - 1].view(np.int32))
    v = s.velocity.astype(np.float32)
    assert np.array_equal(nb.sort_posit(ctx, ttb, v), v[ttb - 1])
    assert np.array_equal(nb.sort_posit(ctx, ttb, s.q), s.q[ttb - 1])
    sb, n1, n2, n3 = nb.sort_specbond_numbond(ctx, tt, s.specbond, s.num1bond, s.num2bond,
                                              s.num3bond)
    want = np.zeros_like(s.specbond)
    for i in range(s.np_atoms):
        k = s.num3bond[i]
        want[tt[i] - 1, :k] = tt[s.specbond[i, :k] - 1]
    assert np.array_equal(sb, want)
    assert np.array_equal(n3, s.num3bond[ttb - 1]) and np.array_equal(n1, s.num1bond[ttb - 1])
    assert np.array_equal(n2, s.num2bond[ttb - 1])
    bl = nb.sort_list(ctx, tt, s.bonds, 2)
    assert np.array_equal(bl[:, :2], tt[s.bonds[:, :2] - 1]) and np.array_equal(bl[:, 2], s.bonds[:, 2])
    dl = nb.sort_list(ctx, tt, s.dihedrals, 4)
    assert np.array_equal(dl[:, :4], tt[s.dihedrals[:, :4] - 1])
    bad = s.bonds.copy()
    bad[3, 0] = s.np_atoms + 5
    with pytest.raises(RuntimeError):
        nb.sort_list(ctx, tt, bad, 2)


def test_pbc_matches_reference_loops(ctx):
    from molecular_simulation_code_b200.system import wrap_positions
    s = small_system()
    rng = np.random.default_rng(8)
    pos = s.position_aos().copy()
    L = float(s.box)
    pos[:, :3] += rng.integers(-3, 4, size=(s.np_atoms, 3)).astype(np.float32) * np.float32(L)
    pos[:5, 0] = [0.0, -0.0, L, -L, 2 * L]
    out = nb.pbc(ctx, pos, s.box)
    assert np.array_equal(out[:, :3], wrap_positions(pos[:, :3], s.box))
    assert np.array_equal(out[:, 3].view(np.int32), pos[:, 3].view(np.int32))
    far = pos.copy()
    far[7, 1] = np.float32(1000 * L)
    with pytest.raises(RuntimeError):
        nb.pbc(ctx, far, s.box)


def test_improper_matches_oracle(ctx):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos().copy()
    rng = np.random.default_rng(6)
    pos[:100, :3] += rng.normal(0, 0.1, (100, 3)).astype(np.float32)
    coeff = np.array([[1.1, 3.0]])
    off, oe, ovir = O.improper_harmonic(_orc_params(p), pos, s.impropers, coeff)
    ff, e, vir = nb.improper_harmonic(ctx, pos, s.impropers, coeff, p)
    assert abs(e - oe) <= FP64_TOL * abs(oe)
    assert rel_err(vir, ovir) <= 1e-9
    # the reference rounds ff_impro to real*4 after every improper; the device once
    assert rel_err(ff, off) <= 1e-6
    with pytest.raises(RuntimeError):
        bad = s.impropers.copy()
        bad[0, 4] = 7
        nb.improper_harmonic(ctx, pos, bad, coeff, p)


@pytest.mark.parametrize("which", ["12", "13", "14"])
def test_correct_1x_matches_oracle(ctx, which):
    s = small_system()
    p = ref_params(s)
    pos = s.position_aos()
    g = O.calculate_gewald(float(p.cut_coul))
    lst, a, b, fudge = {"12": (s.bonds, 0, 1, 0.0), "13": (s.angles, 0, 2, 0.0),
                        "14": (s.dihedrals, 0, 3, float(np.float32(1.0) / np.float32(1.2)))}[which]
    offc, oe, ovir = O.correct_pairs(_orc_params(p), pos, s.q, lst, a, b, g, fudge)
    ffc, e, vir = nb.correct_1x_bonds(ctx, pos, s.q, lst, a, b, g, fudge, p)
    assert abs(e - oe) <= FP64_TOL * abs(oe)
    assert rel_err(vir, ovir) <= 1e-9
    assert rel_err(ffc, offc) <= 1e-6


def _cluster_case(seed, n_gly, n_wat, crystal):
    from molecular_simulation_code_b200.system import make_system
    s = make_system(n_gly, n_wat, seed)
    pos = s.position_aos()
    if crystal:
        # pack glycine molecules onto a tight sub-lattice so clusters, ties and
        # surface molecules appear
        rng = np.random.default_rng(seed)
        L = float(s.box)
        g = pos[:10 * n_gly, :3].reshape(n_gly, 10, 3).astype(np.float64)
        g = g - L * np.round((g - g[:, :1, :]) / L)  # unwrap each molecule about its atom 1
        cen = g.mean(axis=1, keepdims=True)
        k = int(np.ceil(n_gly ** (1 / 3)))
        sites = np.array([(i, j, l) for i in range(k) for j in range(k) for l in range(k)])[:n_gly]
        origin = rng.uniform(0, float(s.box), 3)
        spacing = rng.uniform(4.5, 5.5)
        newc = origin + sites * spacing + rng.normal(0, 0.6, size=(n_gly, 3))
        g = g - cen + newc[:, None, :]
        g = np.mod(g, float(s.box))
        g[g == 0] = float(s.box)
        pos[:10 * n_gly, :3] = g.reshape(-1, 3).astype(np.float32)
    return s, pos


@pytest.mark.parametrize("seed,crystal,greatest_in", [(1, True, 0), (2, True, 7), (3, False, 0),
                                                      (4, False, 5), (5, True, 0)])
def test_greatest_cluster_bit_exact(ctx, seed, crystal, greatest_in):
    s, pos = _cluster_case(seed, 64, 1500, crystal)
    gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
    # permute atom order (as a cell sort would) but keep global ids
    perm = np.random.default_rng(seed).permutation(s.np_atoms)
    pos_p = np.ascontiguousarray(pos[perm])
    gid_p = np.ascontiguousarray(gid[perm])
    ptta0 = np.random.default_rng(seed + 100).uniform(0, float(s.box), (64 * 10, 3))
    box = s.box
    ibox = np.float32(1.0 / np.float64(box))
    vol = np.float32(np.float32(box * box) * box)
    for densmin in (3, 6):
        pt_o = ptta0.copy()
        osz, og, od, ob = O.greatest_cluster(pos_p, gid_p, 64, 10, box, ibox, vol, 9.0, 6.0,
                                             densmin, pt_o, greatest_in)
        pt_g = ptta0.copy()
        gsz, gg, gd, gb = nb.get_greatest_cluster(ctx, pos_p, gid_p, 64, 10, box, 9.0, 6.0,
                                                  densmin, pt_g, greatest_in)
        assert gsz == osz and gg == og
        assert np.array_equal(gd, od) and np.array_equal(gb, ob)
        assert np.array_equal(pt_g, pt_o)


def test_neighbor_list_sets_bit_exact_90k(ctx):
    """The 90,000-atom configuration (rc 10 A, skin 2 A): identical sorted rows."""
    from molecular_simulation_code_b200.system import make_workload
    s = make_workload("gly1500_wat25000_90k", seed=2000)
    p = ref_params(s, cut=10.0, pad=2.0)
    pos = s.position_aos()
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 1024)
    onl, onn, ona = O.neighbor_wrapper(_orc_params(p), pos, s.specbond, s.num3bond, 1024)
    assert np.array_equal(nn, onn)
    rows_gpu = [np.sort(nl[i * na:i * na + nn[i]]) for i in range(0, s.np_atoms, 7)]
    rows_orc = [np.sort(onl[i * ona:i * ona + onn[i]]) for i in range(0, s.np_atoms, 7)]
    assert all(np.array_equal(g, o) for g, o in zip(rows_gpu, rows_orc))


def test_check_neighbor_matches_oracle(ctx):
    import ctypes as C
    rng = np.random.default_rng(4)
    for scale in (0.3, 1.0, 1.49, 1.51):
        d = (rng.normal(size=(3, 5000)) * scale / np.sqrt(3)).astype(np.float32)
        L = O.lib()
        L.orc_check_neighbor.argtypes = [C.c_int, np.ctypeslib.ndpointer(np.float32),
                                         np.ctypeslib.ndpointer(np.float32),
                                         np.ctypeslib.ndpointer(np.float32), C.c_double]
        L.orc_check_neighbor.restype = C.c_int
        want = L.orc_check_neighbor(5000, d[0].copy(), d[1].copy(), d[2].copy(), 1.5 ** 2)
        got = nb.check_neighbor(ctx, d[0].copy(), d[1].copy(), d[2].copy(), 1.5 ** 2)
        assert got == want
