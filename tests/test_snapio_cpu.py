"""Snapshot and topology I/O in the reference's formats (CPU only).

Covers the .gro reader (read_in_Grofile, Source/mod_GroFile.f90:117-159), the
restart dump (Source/mod_datadump.f90:113-153, 216-252), the topology and
molecule-template parsers (Source/mod_readfile.f90:188-562) and the exclusion
layout of build_spec_bond_list_once (Source/mod_buildbond_lists.f90:80-118),
using the committed fixture of the reference's glycine_1500 input.
"""
import os

import numpy as np
import pytest

from molecular_simulation_code_b200 import snapio as S

FIX = os.path.join(os.path.dirname(__file__), "golden", "glycine_1500_solv_min.npz")


@pytest.fixture(scope="module")
def ref():
    return S.load_fixture(FIX)


def test_fixture_matches_reference_layout(ref):
    s, run = ref
    assert s.np_atoms == 45255 and s.n_gly == 1500 and s.n_wat == 10085
    # box: the f10.5 field 7.76100 as real*4, times 10.0d0, in real*4
    assert s.box == np.float32(np.float64(np.float32(7.761)) * 10.0)
    assert (run["rcut"], run["cut_coul"], run["pad"]) == (12.0, 12.0, 1.5)
    assert (run["mrcut"], run["denscut"], run["densmin"], run["alpha"]) == (9.0, 6.0, 11, 0.22)
    assert s.ntypes == 12 and s.types[:10].tolist() == list(range(1, 11))
    assert s.types[15000:15003].tolist() == [11, 12, 12]
    assert abs(float(np.sum(s.q, dtype=np.float64))) < 1e-3
    # exclusion counts: glycine 1-2/1-3/1-4 partners, water 1-2 + 1-3
    assert s.num3bond.max() <= 12
    assert s.num1bond[:10].tolist() == [3, 4, 4, 1, 1, 1, 1, 1, 1, 1]
    assert s.num3bond[15000:15003].tolist() == [2, 2, 2]


def test_exclusions_symmetric_and_cover_bonds(ref):
    s, _ = ref
    n = s.np_atoms
    rows = np.repeat(np.arange(1, n + 1), 12).reshape(n, 12)
    valid = np.arange(12)[None, :] < s.num3bond[:, None]
    a = rows[valid]
    b = s.specbond[valid]
    fwd = set(zip(a.tolist(), b.tolist()))
    assert all((j, i) in fwd for i, j in fwd)
    assert all(i != j for i, j in fwd)
    for i1, i2, _ in s.bonds[:2000]:
        assert (int(i1), int(i2)) in fwd
    # order inside a row: 1-2 partners first (num1bond of them)
    first = s.specbond[np.arange(n), 0]
    bonded = {(int(i), int(j)) for i, j, _ in s.bonds} | {(int(j), int(i)) for i, j, _ in s.bonds}
    assert all((k + 1, int(first[k])) in bonded for k in range(0, n, 97))


def test_second_fixture_counts_from_residues():
    s, run = S.load_fixture(os.path.join(os.path.dirname(FIX), "glycine_2500_solv_min.npz"))
    assert s.np_atoms == 74524 and s.n_gly == 2500 and s.n_wat == 16508
    assert s.box == np.float32(np.float64(np.float32(9.201)) * 10.0)
    assert s.impropers.shape == (2500, 5) and s.shake.shape[0] == 2500 * 2 + 16508
    assert run["rcut"] == 12.0


def test_shake_groups(ref):
    s, _ = ref
    kinds, counts = np.unique(s.shake[:, 0], return_counts=True)
    assert dict(zip(kinds.tolist(), counts.tolist())) == {-3: 10085, 3: 1500, 4: 1500}
    w = s.shake[s.shake[:, 0] == -3]
    assert np.all(s.types[w[:, 1] - 1] == 11)
    assert np.allclose(s.shake_bond[s.shake[:, 0] == -3], [1.0, 1.0, 1.633])


def test_gro_round_trip(ref, tmp_path):
    s, _ = ref
    p = tmp_path / "snap.gro"
    S.write_gro(str(p), s.xyz, s.box)
    xyz, box, _ = S.read_gro(p.read_text())
    assert box == s.box
    assert np.array_equal(xyz, s.xyz)


def test_gro_reader_both_record_layouts():
    """Records with the atom number apart and merged into the atom name (atom
    number above 9999) parse alike; negatives are kept (pbc wraps later)."""
    text = ("T\n    2\n"
            "    1TTA     C1    1   3.826   3.863   4.074\n"
            "11584SOL     HW45252  -0.009   7.546   5.787\n"
            "   7.76100   7.76100   7.76100\n")
    xyz, box, names = S.read_gro(text)
    want = np.array([[3.826, 3.863, 4.074], [-0.009, 7.546, 5.787]], np.float32)
    assert np.array_equal(xyz, (want.astype(np.float64) * 10.0).astype(np.float32))
    assert names == ["C1", "HW"]
    assert box == np.float32(np.float64(np.float32(7.761)) * 10.0)


def test_restart_round_trip_by_global_id(tmp_path):
    rng = np.random.default_rng(3)
    n = 500
    x = np.round(rng.uniform(0, 77.0, (n, 3)), 6).astype(np.float32)
    v = np.round(rng.normal(0, 0.01, (n, 3)), 6).astype(np.float32)
    order = rng.permutation(n)
    p = tmp_path / "restart_100"
    S.write_restart(str(p), np.float32(77.61), 300.0, 17, 200.0, order + 1, x[order], v[order])
    lines = p.read_text().splitlines()
    assert len(lines) == 4 + n and len(lines[4]) == 5 + 6 * 12
    box, temp, num, tclock, xr, vr = S.read_restart(str(p), n)
    assert box == np.float32(77.61) and temp == 300.0 and num == 17 and tclock == 200.0
    assert np.array_equal(xr, np.array([[np.float32(f"{c:.6f}") for c in r] for r in x]))
    assert np.array_equal(vr, np.array([[np.float32(f"{c:.6f}") for c in r] for r in v]))


def test_restart_fields_that_touch(tmp_path):
    """A full-width f12.6 field leaves no blank before it; ids wider than i5."""
    p = tmp_path / "r"
    p.write_text(" 77.61\n 300\n 0\n 0\n"
                 "123456-1234.567890    1.000000    2.000000   -0.001000    0.002000    0.003000\n")
    j, xx, vv = S._restart_record(p.read_text().splitlines()[4])
    assert j == 123456
    assert xx == [np.float32(-1234.56789), np.float32(1.0), np.float32(2.0)]
    assert vv == [np.float32(-0.001), np.float32(0.002), np.float32(0.003)]


def test_restart_truncated_or_bad_ids_fail(tmp_path):
    p = tmp_path / "r"
    gid = np.arange(1, 11)
    x = np.ones((10, 3), np.float32)
    S.write_restart(str(p), 10.0, 0.0, 0, 0.0, gid, x, x)
    with pytest.raises(ValueError):
        S.read_restart(str(p), 11)          # one atom record missing
    S.write_restart(str(p), 10.0, 0.0, 0, 0.0, gid + 5, x, x)
    with pytest.raises(ValueError):
        S.read_restart(str(p), 10)          # ids outside 1..np
    S.write_restart(str(p), 10.0, 0.0, 0, 0.0, np.ones(10, int), x, x)
    with pytest.raises(ValueError):
        S.read_restart(str(p), 10)          # duplicate ids leave atoms unset


_WATER_TOP = """!--- nonbonded
2
#type, tag, name, rmin/2, eps, q, mass
1 63 OW 1.7768 0.1554 -0.8476 15.999
2 64 HW 0.0 0.0 0.4238 1.008

!--- bonds
1 2
# moltype type a1 a2 kb r0
1 1 1 2 600.0 1.0
1 1 1 3 600.0 1.0

!--- angles
1 1 ***
# moltype type a1 a2 a3 k theta
1 1 2 1 3 75.0 109.47

!--- torsions
0 0
#

!--- impropers
0 0
#

!--- rigid bonds
!---
1
#num
#moltype atoms lengths
-3
1 1 2 3 1.0 1.0 1.633
"""

_WATER_MOL = """!--- water
1
#type, no, x, y, z
4
3
1 1 0.0 0.0 0.0
2 2 1.0 0.0 0.0
2 3 -0.3 0.9 0.0
"""


def test_topology_parser_and_exclusion_layout():
    mol = S.parse_mol(_WATER_MOL)
    top = S.parse_topol(_WATER_TOP, 1)
    assert mol["counts"].tolist() == [4] and mol["natoms"].tolist() == [3]
    assert top["bonds"].shape == (2, 6) and top["angles"].shape == (1, 7)
    assert top["diheds"].shape == (0, 9) and top["shake"].shape == (1, 9)
    xyz = np.zeros((12, 3), np.float32)
    s = S.build_reference_system(mol, top, xyz, np.float32(20.0))
    assert s.np_atoms == 12
    # O: 1-2 partners 2, 3 in bond order; H: O then the other H (1-3)
    assert s.specbond[0, :2].tolist() == [2, 3] and s.specbond[1, :2].tolist() == [1, 3]
    assert s.specbond[5, :2].tolist() == [4, 5]
    assert s.num1bond[:3].tolist() == [2, 1, 1] and s.num3bond[:3].tolist() == [2, 2, 2]
    assert s.shake[:, 0].tolist() == [-3] * 4 and s.shake[1, 1:4].tolist() == [4, 5, 6]
    assert np.isclose(s.angle_coeff[0, 1], np.deg2rad(109.47))
    assert np.isclose(s.q.sum(), 0.0, atol=1e-6)


def test_unknown_shake_kind_rejected():
    with pytest.raises(ValueError):
        S.parse_topol(_WATER_TOP.replace("\n-3\n", "\n5\n"), 1)
