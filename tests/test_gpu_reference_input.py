"""GPU parity on the reference's own input: the minimized glycine_1500 and
glycine_2500 snapshots (45,255 and 74,524 atoms, AMBER Rmin/2 force field) with
the run input's cut-offs
(rcut = cut_coul = 12 A, padding 1.5 A, alpha 0.22 1/A, cluster radii 9 / 6 A,
densmin 11), loaded from the committed fixture and wrapped into (0, box] as pbc
does.

Bars: bit-exact neighbour rows (as sets) and cluster outputs; FP64 potential,
e_coul and forces within 1e-10 relative of the oracle; mixed forces within
1e-6 RMS relative of FP64; snapshot/rollback and checkpoint/resume replay the
same trajectory bit for bit.
"""
import os

import numpy as np
import pytest

from molecular_simulation_code_b200 import mixed as M
from molecular_simulation_code_b200 import nonbond as nb
from molecular_simulation_code_b200 import snapio as S
from molecular_simulation_code_b200.system import wrap_positions
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-10


@pytest.fixture(scope="module", params=["glycine_1500_solv_min", "glycine_2500_solv_min"])
def ref(request):
    s, run = S.load_fixture(os.path.join(GOLDEN, request.param + ".npz"))
    s.xyz = wrap_positions(s.xyz, s.box)
    p = nb.DsfParams(alpha=float(run["alpha"]), box=s.box, cut_coul=float(run["cut_coul"]),
                     rcut=float(run["rcut"]), neighbor_pad=float(run["pad"]))
    op = O.params(p.alpha, p.box, p.cut_coul, p.rcut, p.neighbor_pad)
    pos = s.position_aos()
    onl, onn, ona = O.neighbor_wrapper(op, pos, s.specbond, s.num3bond, 1024)
    return s, run, p, op, pos, (onl, onn, ona)


def _sorted_rows(nl, nn, na):
    n = nn.shape[0]
    m = nl.reshape(n, na).astype(np.int64)
    m = np.where(np.arange(na)[None, :] < nn[:, None], m, np.iinfo(np.int64).max)
    return np.sort(m, axis=1)


def test_neighbor_list_bit_exact(ctx, ref):
    s, _, p, _, pos, (onl, onn, ona) = ref
    nl, nn, na = nb.neighbor_wrapper(ctx, pos, s.specbond, s.num3bond, p, 1024)
    assert na == ona and np.array_equal(nn, onn)
    assert np.array_equal(_sorted_rows(nl, nn, na), _sorted_rows(onl, onn, ona))


def test_fp64_forces_match_oracle(ctx, ref):
    s, _, p, op, pos, (onl, onn, ona) = ref
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    off, off64, opot, oec, ovir = O.force_dsf(op, pos, s.q, lj, s.ntypes, onl, onn, ona)
    ff, pot, ec, vir = nb.lj_cut_coul_dsf_nonewton(ctx, pos, s.q, lj, s.ntypes, onl, onn, ona, p)
    assert abs(pot - opot) <= FP64_TOL * abs(opot)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert np.abs(vir - ovir).max() <= FP64_TOL * np.abs(ovir).max()
    assert np.abs(ff - off).max() <= 2 * np.spacing(np.abs(off).max())


def test_real_space_ewald_matches_oracle(ctx, ref):
    """The PME path's pair term on the reference input (gewald of cut_coul 12 A)."""
    s, _, p, op, pos, (onl, onn, ona) = ref
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    g = nb.calculate_gewald(p.cut_coul)
    off, _, opot, oec, ovir = O.force_long(op, pos, s.q, lj, s.ntypes, onl, onn, ona, g)
    ff, pot, ec, vir = nb.lj_cut_coul_long_nonewton(ctx, pos, s.q, lj, s.ntypes, onl, onn, ona,
                                                    p, g)
    assert abs(pot - opot) <= FP64_TOL * abs(opot)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert np.abs(vir - ovir).max() <= FP64_TOL * np.abs(ovir).max()
    assert np.abs(ff - off).max() <= 2 * np.spacing(np.abs(off).max())


def test_cluster_pair_path(ctx, ref):
    """Production path on the reference system: FP64 within 1e-10 of the oracle,
    mixed within 1e-6 RMS of FP64."""
    s, run, p, op, pos, (onl, onn, ona) = ref
    lj = (s.lj1, s.lj2, s.lj3, s.lj4)
    _, off64, opot, oec, _ = O.force_dsf(op, pos, s.q, lj, s.ntypes, onl, onn, ona)
    m = M.System(ctx, s, alpha=p.alpha, cut=p.cut_coul, skin=p.neighbor_pad)
    m.set_state(s.xyz.astype(np.float64))
    e64 = m.compute(M.FP64, rebuild=True)
    f64 = m.get_state()[2]
    assert abs(e64[0] - opot) <= FP64_TOL * abs(opot)
    assert abs(e64[1] - oec) <= FP64_TOL * abs(oec)
    assert M.force_max_rel(f64, off64) <= FP64_TOL
    e32 = m.compute(M.MIXED)
    f32 = m.get_state()[2]
    rms = M.force_rms_rel(f32, f64)
    print("reference input: mixed force rms rel", rms, "max rel", M.force_max_rel(f32, f64))
    assert rms <= 1e-6
    assert abs(e32[1] - e64[1]) <= 1e-5 * abs(e64[1])
    m.close()


def test_pair14_and_exclusion_corrections(ctx, ref):
    s, _, p, op, pos, _ = ref
    dc = np.zeros((2, 4))  # the topology's torsions carry no OPLS coefficients
    offh, oed, oec, op14 = O.dihedral_opls_dsf(op, pos, s.q, s.ntypes, s.lj14, s.dihedrals, dc)
    ffh, ed, ec, p14 = nb.dihedral_opls_dsf(ctx, pos, s.q, s.ntypes, s.lj14, s.dihedrals, dc, p)
    assert abs(ec - oec) <= FP64_TOL * abs(oec)
    assert abs(p14 - op14) <= FP64_TOL * abs(op14)
    assert rel_max(ffh, offh) <= 1e-6
    g = O.calculate_gewald(float(p.cut_coul))
    offc, oe, _ = O.correct_pairs(op, pos, s.q, s.bonds, 0, 1, g, 0.0)
    ffc, e, _ = nb.correct_1x_bonds(ctx, pos, s.q, s.bonds, 0, 1, g, 0.0, p)
    assert abs(e - oe) <= FP64_TOL * abs(oe)
    assert rel_max(ffc, offc) <= 1e-6


def rel_max(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("greatest_in", [0, 3])
def test_greatest_cluster_bit_exact(ctx, ref, greatest_in):
    s, run, _, _, pos, _ = ref
    gid = np.arange(1, s.np_atoms + 1, dtype=np.int32)
    perm = np.random.default_rng(11).permutation(s.np_atoms)
    pos_p = np.ascontiguousarray(pos[perm])
    gid_p = np.ascontiguousarray(gid[perm])
    box = s.box
    ibox = np.float32(1.0 / np.float64(box))
    vol = np.float32(np.float32(box * box) * box)
    ptta0 = pos[:10 * s.n_gly, :3].astype(np.float64)
    mr, dc, dm = float(run["mrcut"]), float(run["denscut"]), int(run["densmin"])
    pt_o = ptta0.copy()
    osz, og, od, ob = O.greatest_cluster(pos_p, gid_p, s.n_gly, 10, box, ibox, vol, mr, dc, dm,
                                         pt_o, greatest_in)
    pt_g = ptta0.copy()
    gsz, gg, gd, gb = nb.get_greatest_cluster(ctx, pos_p, gid_p, s.n_gly, 10, box, mr, dc, dm,
                                              pt_g, greatest_in)
    assert gsz == osz and gg == og
    assert np.array_equal(gd, od) and np.array_equal(gb, ob)
    assert np.array_equal(pt_g, pt_o)


@pytest.fixture(scope="module")
def md_system(ref):
    s, run, p, *_ = ref
    c = nb.Context(0)
    m = M.System(c, s, alpha=p.alpha, cut=p.cut_coul, skin=p.neighbor_pad)
    m.set_state(s.xyz.astype(np.float64), np.zeros((s.np_atoms, 3)))
    m.md_setup(s, dt=float(run["dt"]), temperature=300.0, gamma=0.01, seed=7)
    yield m
    m.close()
    c.close()


def test_md_snapshot_rollback_replays(md_system):
    m = md_system
    m.md_run(10)
    m.snapshot()
    step0 = m.md_step()
    e1 = m.md_run(20, energy_every=20)
    x1, v1, _ = m.get_state()
    assert np.isfinite(e1["total"]) and m.md_step() == step0 + 20
    m.rollback()
    assert m.md_step() == step0
    e2 = m.md_run(20, energy_every=20)
    x2, v2, _ = m.get_state()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert e1 == e2


def test_checkpoint_resume_bit_exact(md_system, ref, tmp_path):
    s, run, p, *_ = ref
    m = md_system
    ck = str(tmp_path / "ck.npz")
    S.save_checkpoint(m, ck)
    m.md_run(15)
    xa = m.get_state()[0]
    c = nb.Context(0)
    m2 = M.System(c, s, alpha=p.alpha, cut=p.cut_coul, skin=p.neighbor_pad)
    m2.md_setup(s, dt=float(run["dt"]), temperature=300.0, gamma=0.01, seed=7)
    S.resume_checkpoint(m2, ck)
    m2.md_run(15)
    assert np.array_equal(m2.get_state()[0], xa)
    # the reference text restart keeps real*4 at six decimals
    rs = str(tmp_path / "restart_15")
    S.dump_restart(m2, rs, s.box, 300.0, 0, 30.0)
    x, v, _ = m2.get_state()
    box, _, _, tclock = S.load_restart(m2, rs)
    xr, vr, _ = m2.get_state()
    assert box == s.box and tclock == 30.0
    assert np.abs(xr - x).max() <= 1e-5
    assert np.abs(vr - v).max() <= 1e-6
    m2.close()
    c.close()
