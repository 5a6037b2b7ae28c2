"""GPU parity of the residency kernels and of the force-driver merge against the
oracle, through sofia_system_md_forces (one step's forces without stepping).

Systems: the 9,000-atom synthetic glycine/water configuration (rc 10 A, skin
2 A, alpha 0.2/A) and the reference's glycine_1500 snapshot (rc 12 A, pad
1.5 A, alpha 0.22/A).  Positions are rounded to a 2^-10 A grid inside the box:
every coordinate and every coordinate difference is then exact in real*4, so
the reference's real*4 bond vectors (mod_force_bond.f90:6-75 and the other
bonded routines) and the device's FP64 ones are the same numbers, and the
comparisons below are FP64 against FP64.

Bars:
  * bond, angle, torsion + 1-4, improper and the merged nonbond + torsion + 1-4
    forces (force_wrapper_DSF, mod_force.f90:510-554): energies within 1e-10
    relative; forces within 1e-10 of max |f| plus, per atom, half a fixed-point
    quantum (2^-33 kcal/mol/A) for every term that adds to it (the device sums
    each term's force in 64-bit fixed point with 2^-32 resolution); the
    improper's oracle stores real*4 forces, so its forces are compared at real*4
    level;
  * SHAKE (mod_shake.f90:8-85, 888-913): constraint forces within 1e-10 of their
    max, predicted positions x + dt v + dt^2 f/m within 1e-11 A;
  * Langevin (mod_langevin.f90:15-43, gconst of get_started.f90:81-84): friction
    exact, the noise (f + fric m v) / (gconst sqrt(m)) uniform in [-1/2, 1/2)
    with mean 0 and variance 1/12 within 5 standard errors, a fresh draw per step.
"""
import os

import numpy as np
import pytest

from molecular_simulation_code_b200 import _lib as L
from molecular_simulation_code_b200 import mixed as M
from molecular_simulation_code_b200 import snapio as S
from molecular_simulation_code_b200.system import make_system, wrap_positions
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KCAL2AMU = float(np.float32(0.0004184))
KBOLTZ = float(np.float32(0.001987204181))
BONDED = (L.SOFIA_TERM_BOND | L.SOFIA_TERM_ANGLE | L.SOFIA_TERM_TORSION | L.SOFIA_TERM_PAIR14 |
          L.SOFIA_TERM_IMPROPER)


def _grid(x, box):
    """Positions on a 2^-10 A grid in [0, box)."""
    q = np.round(np.asarray(x, np.float64) * 1024.0) / 1024.0
    q = np.mod(q, float(box))
    q[q >= float(box)] -= 1.0 / 1024.0
    return q


@pytest.fixture(scope="module", params=["syn9k", "glycine_1500"])
def case(request):
    if request.param == "syn9k":
        s = make_system(150, 2500, 1)
        cut, pad, alpha = 10.0, 2.0, 0.2
    else:
        s, run = S.load_fixture(os.path.join(GOLDEN, "glycine_1500_solv_min.npz"))
        s.xyz = wrap_positions(s.xyz, s.box)
        cut, pad, alpha = float(run["cut_coul"]), float(run["pad"]), float(run["alpha"])
    x = _grid(s.xyz, s.box)
    assert np.array_equal(x.astype(np.float32).astype(np.float64), x)
    rng = np.random.default_rng(11)
    mass = np.asarray(s.mass_type, np.float64)[np.asarray(s.types) - 1]
    kT = KBOLTZ * 300.0
    v = rng.standard_normal((s.np_atoms, 3)) * np.sqrt(kT * KCAL2AMU / mass)[:, None]
    pos = s.position_aos().copy()
    pos[:, :3] = x.astype(np.float32)
    op = O.params(alpha, s.box, cut, cut, pad)
    return dict(s=s, x=x, v=v, mass=mass, pos=pos, op=op, cut=cut, pad=pad, alpha=alpha)


@pytest.fixture(scope="module")
def fp64_md(ctx, case):
    s = case["s"]
    m = M.System(ctx, s, alpha=case["alpha"], cut=case["cut"], skin=case["pad"],
                 precision=M.FP64)
    m.set_state(case["x"], case["v"])
    m.md_setup(s, dt=2.0, temperature=300.0, gamma=0.001, seed=17, terms=31,
               shake_maxiter=200, shake_tol=1e-12)
    yield m
    m.close()


def _close(f, fo, rel=1e-10, count=None):
    """|f - fo| <= rel * max|fo| + count * 2^-33 per atom (count: terms adding to it)."""
    den = np.abs(fo).max()
    tol = rel * den
    if count is not None:
        tol = tol + np.asarray(count, np.float64)[:, None] * 2.0 ** -33
    d = np.abs(f - fo)
    return bool((d <= tol).all()), float(d.max() / den)


def _count(n, lst, natoms_per_row):
    """How many rows of a 1-based bonded list touch each atom."""
    ids = np.asarray(lst)[:, :natoms_per_row].ravel() - 1
    return np.bincount(ids, minlength=n)


def test_bond_and_angle_match_oracle(fp64_md, case):
    s, p, pos = case["s"], case["op"], case["pos"]
    n = s.np_atoms
    f, e = fp64_md.md_forces(L.SOFIA_TERM_BOND)
    fo, eo = O.bond_harmonic(p, pos, s.bonds, s.bond_coeff)
    assert e["bond"] == pytest.approx(eo, rel=1e-10)
    ok, err = _close(f, fo, count=_count(n, s.bonds, 2))
    assert ok, err
    f, e = fp64_md.md_forces(L.SOFIA_TERM_ANGLE)
    fo, eo = O.angle_harmonic(p, pos, s.angles, s.angle_coeff)
    assert e["angle"] == pytest.approx(eo, rel=1e-10)
    ok, err = _close(f, fo, count=_count(n, s.angles, 3))
    assert ok, err
    assert e["bond"] == 0.0 and e["lj"] == 0.0  # terms left out carry no energy


def test_torsion_and_pair14_match_oracle(fp64_md, case):
    s, p, pos = case["s"], case["op"], case["pos"]
    f, e = fp64_md.md_forces(L.SOFIA_TERM_TORSION | L.SOFIA_TERM_PAIR14)
    _, ed, ec, p14, fo = O.dihedral_opls_dsf(p, pos, s.q, s.ntypes, s.lj14, s.dihedrals,
                                             s.dihed_coeff, want_f64=True)
    assert e["torsion"] == pytest.approx(ed, rel=1e-10, abs=1e-12)
    assert e["coul14"] == pytest.approx(ec, rel=1e-10)
    assert e["lj14"] == pytest.approx(p14, rel=1e-10)
    ok, err = _close(f, fo, count=_count(s.np_atoms, s.dihedrals, 4))
    assert ok, err


def test_improper_matches_oracle(fp64_md, case):
    s, p, pos = case["s"], case["op"], case["pos"]
    if len(s.impropers) == 0:
        pytest.skip("no impropers in this topology")
    f, e = fp64_md.md_forces(L.SOFIA_TERM_IMPROPER)
    ffo, eo, _ = O.improper_harmonic(p, pos, s.impropers, s.impro_coeff)
    assert e["improper"] == pytest.approx(eo, rel=1e-10)
    # the oracle keeps ff_impro in real*4 like the reference
    ok, err = _close(f, ffo.astype(np.float64), rel=4 * np.finfo(np.float32).eps)
    assert ok, err


def test_force_driver_merge_matches_oracle(fp64_md, case):
    """Nonbonded pairs + torsions with their 1-4 pairs, merged ff += ffh as the
    DSF force driver does, against the oracle's reference-list forces plus its
    dihedral_opls_DSF."""
    s, p, pos = case["s"], case["op"], case["pos"]
    f, e = fp64_md.md_forces(L.SOFIA_TERM_NONBOND | L.SOFIA_TERM_TORSION | L.SOFIA_TERM_PAIR14)
    nl, nn, na = O.neighbor_wrapper(p, pos, s.specbond, s.num3bond, 1024)
    _, ff64, pot, ec, _ = O.force_dsf(p, pos, s.q, (s.lj1, s.lj2, s.lj3, s.lj4), s.ntypes,
                                      nl, nn, na)
    _, ed, ec14, p14, fh = O.dihedral_opls_dsf(p, pos, s.q, s.ntypes, s.lj14, s.dihedrals,
                                               s.dihed_coeff, want_f64=True)
    assert e["lj"] == pytest.approx(pot, rel=1e-10)
    assert e["coul"] == pytest.approx(ec, rel=1e-10)
    assert e["coul14"] == pytest.approx(ec14, rel=1e-10)
    ok, err = _close(f, ff64 + fh)
    assert ok, err


def test_shake_matches_oracle(fp64_md, case):
    s = case["s"]
    terms = L.SOFIA_TERM_NONBOND | BONDED
    f0, _ = fp64_md.md_forces(terms, energy=False)
    f1, _ = fp64_md.md_forces(terms | L.SOFIA_TERM_SHAKE, energy=False)
    fo, st = O.shake(case["x"], case["v"], f0, case["mass"], float(s.box), s.shake,
                     s.shake_bond, 2.0, KCAL2AMU, iflag=1, maxiter=200, tolerance=1e-12)
    assert st == 0
    g, go = f1 - f0, fo - f0
    ok, err = _close(g, go)
    assert ok, err
    dtsq = 4.0 * KCAL2AMU / case["mass"][:, None]
    xs = case["x"] + 2.0 * case["v"] + dtsq * f1
    xo = case["x"] + 2.0 * case["v"] + dtsq * fo
    assert np.abs(xs - xo).max() <= 1e-11
    # the predicted positions satisfy the constraints
    L_box = float(s.box)
    for grp, b in zip(s.shake[:200], s.shake_bond[:200]):
        num, a = int(grp[0]), grp[1:] - 1
        pairs = {1: [(0, 1)], 3: [(0, 1), (0, 2)], 4: [(0, 1), (0, 2), (0, 3)],
                 -3: [(0, 1), (0, 2), (1, 2)]}[num]
        for k, (u, w) in enumerate(pairs):
            d = xs[a[u]] - xs[a[w]]
            d -= L_box * np.round(d / L_box)
            assert abs(np.linalg.norm(d) - b[k]) < 1e-9


def test_langevin_force_statistics(fp64_md, case):
    s, v, mass = case["s"], case["v"], case["mass"]
    gamma, dt, T = 0.001, 2.0, 300.0
    # the reference's constants: fric and gconst*amu2e (get_started.f90:81-84)
    gconst = np.sqrt(12.0 * KBOLTZ * KCAL2AMU * T * gamma / (0.5 * dt)) / KCAL2AMU
    fric = gamma / KCAL2AMU
    f, _ = fp64_md.md_forces(L.SOFIA_TERM_LANGEVIN, energy=False)
    u = (f + fric * mass[:, None] * v) / (gconst * np.sqrt(mass)[:, None])
    n = u.size
    assert u.min() >= -0.5 - 1e-9 and u.max() < 0.5 + 1e-9
    assert abs(u.mean()) < 5.0 * np.sqrt(1.0 / 12.0 / n)
    # var of U(-1/2,1/2) = 1/12, standard error sqrt(1/180/n)
    assert abs(u.var() - 1.0 / 12.0) < 5.0 * np.sqrt(1.0 / 180.0 / n)
    # components and atoms are uncorrelated
    assert abs(np.corrcoef(u[:, 0], u[:, 1])[0, 1]) < 5.0 / np.sqrt(s.np_atoms)
    # the same step counter gives the same draw; the next step a fresh one
    f2, _ = fp64_md.md_forces(L.SOFIA_TERM_LANGEVIN, energy=False)
    assert np.array_equal(f, f2)
    fp64_md.set_md_step(fp64_md.md_step() + 1)
    f3, _ = fp64_md.md_forces(L.SOFIA_TERM_LANGEVIN, energy=False)
    u3 = (f3 + fric * mass[:, None] * v) / (gconst * np.sqrt(mass)[:, None])
    assert abs(np.corrcoef(u.ravel(), u3.ravel())[0, 1]) < 5.0 / np.sqrt(n)
    fp64_md.set_md_step(fp64_md.md_step() - 1)
