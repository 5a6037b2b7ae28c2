"""Seeded synthetic glycine-zwitterion / SPC/E-water systems in the reference's units.

The reference (Sofia) works in Angstrom, kcal/mol, amu and fs and stores its
module state as ``position(np)`` = {real*4 x,y,z; integer type} (AoS, 16 B per
atom, ``Source/global.f90:82-85,99``), ``q(np)`` real*4 (``global.f90:107``),
``lj1..lj4`` real*4 tables of ``ntype**2`` entries (``global.f90:462``),
``specbond(12,np)`` 1-based 1-2/1-3/1-4 partner lists with cumulative
``num1bond/num2bond/num3bond`` counts (``Source/mod_buildbond_lists.f90:80-118``).
This module builds exactly that state for the seeded synthetic systems
(glycine zwitterions + SPC/E water on a cubic lattice at 1.0 g/cm^3) so the
library, the oracle and the tests all see the same arrays.

Molecule layout follows the reference molecule template
(``input_files/mol_cndo_alpha.input``: C1, C2, N, O1, O2, H1, H2, H3, H4, H5
for glycine; OW, HW, HW for water), glycine first, so the first
``n_gly*10`` global ids are glycine atoms as ``Source/mod_build_ptta.f90:116-164``
assumes.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# Element parameters of the synthetic force field: sigma (nm), eps (kJ/mol),
# charge (e), mass (amu).  Types are 1-based like the reference.
TYPE_NAMES = ["C", "CA", "N", "O", "HN", "HA", "OW", "HW"]
_SIG_NM = [0.375, 0.350, 0.325, 0.296, 0.0, 0.250, 0.3166, 0.0]
_EPS_KJ = [0.439, 0.276, 0.711, 0.879, 0.0, 0.126, 0.650, 0.0]
_CHARGE = [0.70, 0.09, -0.30, -0.80, 0.33, 0.06, -0.8476, 0.4238]
_MASS = [12.011, 12.011, 14.007, 15.999, 1.008, 1.008, 15.999, 1.008]

# glycine template order (reference mol file): C1(C) C2(CA) N O1 O2 H1 H2 H3(HN) H4 H5(HA)
GLY_TYPES = [1, 2, 3, 4, 4, 5, 5, 5, 6, 6]
WAT_TYPES = [7, 8, 8]
GLY_MASS = sum(_MASS[t - 1] for t in GLY_TYPES)
WAT_MASS = sum(_MASS[t - 1] for t in WAT_TYPES)

# bonds (0-based template indices): C-CA, C-O1, C-O2, CA-N, CA-HA1, CA-HA2, N-H1..3
GLY_BONDS = [(0, 1), (0, 3), (0, 4), (1, 2), (1, 8), (1, 9), (2, 5), (2, 6), (2, 7)]
WAT_BONDS = [(0, 1), (0, 2)]
# bond r0 (Angstrom) and kb (kcal/mol/A^2; kb values from input_files/topol_cndo.top:17-28)
_BOND_R0 = {(0, 1): 1.52, (0, 3): 1.25, (0, 4): 1.25, (1, 2): 1.47, (1, 8): 1.09,
            (1, 9): 1.09, (2, 5): 1.01, (2, 6): 1.01, (2, 7): 1.01}
_BOND_K = {(0, 1): 328.30, (0, 3): 648.00, (0, 4): 648.00, (1, 2): 293.60, (1, 8): 338.70,
           (1, 9): 338.70, (2, 5): 369.00, (2, 6): 369.00, (2, 7): 369.00}
# angles (i, middle, k) with k (kcal/mol/rad^2, topol_cndo.top:31-49) and ideal theta0 (deg)
_TET = 109.47
GLY_ANGLES = [
    ((1, 0, 3), 68.03, 120.0), ((1, 0, 4), 68.03, 120.0), ((3, 0, 4), 78.17, 120.0),
    ((0, 1, 2), 65.07, _TET), ((0, 1, 8), 47.23, _TET), ((0, 1, 9), 47.23, _TET),
    ((2, 1, 8), 49.02, _TET), ((2, 1, 9), 49.02, _TET), ((8, 1, 9), 39.04, _TET),
    ((1, 2, 5), 46.19, _TET), ((1, 2, 6), 46.19, _TET), ((1, 2, 7), 46.19, _TET),
    ((5, 2, 6), 40.52, _TET), ((5, 2, 7), 40.52, _TET), ((6, 2, 7), 40.52, _TET),
]
WAT_ANGLES = [((1, 0, 2), 75.00, _TET)]
# proper dihedrals, one per 1-4 pair, in the order of input_files/topol_cndo.top:53-68
GLY_DIHEDRALS = [
    ((3, 0, 1, 2), 1), ((4, 0, 1, 2), 1), ((3, 0, 1, 8), 1), ((3, 0, 1, 9), 1),
    ((4, 0, 1, 8), 1), ((4, 0, 1, 9), 1),
    ((0, 1, 2, 5), 2), ((0, 1, 2, 6), 2), ((0, 1, 2, 7), 2),
    ((8, 1, 2, 5), 2), ((8, 1, 2, 6), 2), ((8, 1, 2, 7), 2),
    ((9, 1, 2, 5), 2), ((9, 1, 2, 6), 2), ((9, 1, 2, 7), 2),
]
# the carboxylate improper (reference topol_cndo.top:72: atoms 2 4 1 5, central atom third,
# k = 1.1 kcal/mol/rad^2); omega0 is taken from the template geometry
GLY_IMPROPER = (1, 3, 0, 4)
GLY_IMPROPER_K = 1.1
# SHAKE groups (reference topol_cndo.top:78-87): CH2 (num 3), NH3 (num 4), rigid water (-3)
WATER_OH = 1.0
WATER_HH = 2.0 * WATER_OH * math.sin(math.radians(_TET) / 2.0)

AMU_PER_A3_TO_GCC = 1.66053906660  # 1 amu/A^3 = 1.6605 g/cm^3


@dataclasses.dataclass
class SofiaSystem:
    """Module state of one Sofia replica (reference layout, 1-based ids)."""

    n_gly: int
    n_wat: int
    box: np.float32                 # real*4 box length (Angstrom)
    position: np.ndarray            # (np,4) structured-like: float32 xyz view + int32 type
    xyz: np.ndarray                 # (np,3) float32
    types: np.ndarray               # (np,) int32, 1-based
    q: np.ndarray                   # (np,) float32
    mass_type: np.ndarray           # (ntype,) float64 per type
    ntypes: int
    lj1: np.ndarray                 # (ntype*ntype,) float32, offset = ntype*(it-1)+jt (1-based)
    lj2: np.ndarray
    lj3: np.ndarray
    lj4: np.ndarray
    lj14: np.ndarray                # (4, ntype, ntype) float64 (lj14_1..4)
    specbond: np.ndarray            # (np,12) int32, 1-based partner ids (0 = unused)
    num1bond: np.ndarray            # (np,) int32 cumulative counts
    num2bond: np.ndarray
    num3bond: np.ndarray
    bonds: np.ndarray               # (nb,3) int32: i1,i2 (1-based), type
    bond_coeff: np.ndarray          # (nbt,2) float64: kb, r0
    angles: np.ndarray              # (na,4) int32: i1,i2(middle),i3, type
    angle_coeff: np.ndarray         # (nat,2) float64: k, theta0 (rad)
    dihedrals: np.ndarray           # (nd,5) int32: i1..i4, type
    dihed_coeff: np.ndarray         # (ndt,4) float64: OPLS k1..k4 (zero, as the reference DSF path sees)
    shake: np.ndarray               # (ns,5) int32: num, a1..a4 (1-based, 0 unused)
    shake_bond: np.ndarray          # (ns,3) float64 bond lengths
    velocity: np.ndarray            # (np,3) float32 Angstrom/fs
    seed: int
    impropers: np.ndarray = dataclasses.field(
        default_factory=lambda: np.zeros((0, 5), np.int32))   # (ni,5) int32: i1..i4, type
    impro_coeff: np.ndarray = dataclasses.field(
        default_factory=lambda: np.zeros((1, 2), np.float64))  # (nit,2): k, omega0 (rad)

    @property
    def np_atoms(self) -> int:
        return int(self.types.shape[0])

    @property
    def n_mol(self) -> int:
        return self.n_gly + self.n_wat

    def position_aos(self) -> np.ndarray:
        """16-byte AoS records {float x,y,z; int32 type} exactly like ``type(ainfo)``."""
        out = np.empty((self.np_atoms, 4), dtype=np.float32)
        out[:, :3] = self.xyz
        out[:, 3] = self.types.view(np.float32)
        return out

    def mol_id(self) -> np.ndarray:
        """0-based molecule index of every atom."""
        g = np.repeat(np.arange(self.n_gly, dtype=np.int32), 10)
        w = self.n_gly + np.repeat(np.arange(self.n_wat, dtype=np.int32), 3)
        return np.concatenate([g, w])


def improper_omega(xyz: np.ndarray, box: float, quads: np.ndarray) -> np.ndarray:
    """The improper angle omega (rad) of improper_harmonic_lammps14
    (Source/mod_force_dihed.f90:1572-1620) for 0-based atom quadruples (m,4):
    the angle between the planes (1,2,3) and (2,3,4), minimum image."""
    x = np.asarray(xyz, np.float64)
    L = float(box)

    def mi(d):
        return d - L * np.round(d / L)
    q = np.asarray(quads)
    v1 = mi(x[q[:, 0]] - x[q[:, 1]])
    v2 = mi(x[q[:, 2]] - x[q[:, 1]])
    v3 = mi(x[q[:, 3]] - x[q[:, 2]])
    r1 = 1.0 / np.linalg.norm(v1, axis=1)
    r2 = 1.0 / np.linalg.norm(v2, axis=1)
    r3 = 1.0 / np.linalg.norm(v3, axis=1)
    c0 = (v1 * v3).sum(1) * r1 * r3
    c1 = (v1 * v2).sum(1) * r1 * r2
    c2 = -(v3 * v2).sum(1) * r3 * r2
    s1 = 1.0 / np.maximum(1.0 - c1 * c1, 0.001)
    s2 = 1.0 / np.maximum(1.0 - c2 * c2, 0.001)
    c = np.clip((c1 * c2 + c0) * np.sqrt(s1 * s2), -1.0, 1.0)
    return np.arccos(c)


def lj_tables_4eps(ntypes: int, sig_a: np.ndarray, eps_kcal: np.ndarray):
    """LJ tables in the 4-eps form with geometric sigma/eps mixing.

    The table-driven kernel (``Source/mod_force_nonbond.f90:156-158``) evaluates
    ``F*r = dr6i*(lj1*dr6i - lj2)``, ``E = dr6i*(dr6i*lj3 - lj4)``; the 4-eps
    assignment is the alternative written at ``Source/mod_readfile.f90:606-609``
    and the 1-4 tables are half of the main ones (``mod_readfile.f90:612-615``).
    """
    lj1 = np.zeros(ntypes * ntypes, np.float32)
    lj2 = np.zeros_like(lj1)
    lj3 = np.zeros_like(lj1)
    lj4 = np.zeros_like(lj1)
    lj14 = np.zeros((4, ntypes, ntypes), np.float64)
    for a in range(ntypes):
        for b in range(ntypes):
            e = math.sqrt(eps_kcal[a] * eps_kcal[b])
            s = math.sqrt(sig_a[a] * sig_a[b])
            off = ntypes * a + b
            s6 = s ** 6
            s12 = s ** 12
            lj1[off] = 48.0 * e * s12
            lj2[off] = 24.0 * e * s6
            lj3[off] = 4.0 * e * s12
            lj4[off] = 4.0 * e * s6
            lj14[0, a, b] = 0.5 * 48.0 * e * s12
            lj14[1, a, b] = 0.5 * 24.0 * e * s6
            lj14[2, a, b] = 0.5 * 4.0 * e * s12
            lj14[3, a, b] = 0.5 * 4.0 * e * s6
    return lj1, lj2, lj3, lj4, lj14


def lj_tables_rmin(ntypes: int, rmin_half: np.ndarray, eps_kcal: np.ndarray):
    """AMBER Rmin/2 tables exactly as ``check_topol_file`` builds them
    (``Source/mod_readfile.f90:597-615``): R = Rmin/2_i + Rmin/2_j, eps geometric."""
    lj1 = np.zeros(ntypes * ntypes, np.float32)
    lj2 = np.zeros_like(lj1)
    lj3 = np.zeros_like(lj1)
    lj4 = np.zeros_like(lj1)
    lj14 = np.zeros((4, ntypes, ntypes), np.float64)
    for a in range(ntypes):
        for b in range(ntypes):
            e = math.sqrt(eps_kcal[a] * eps_kcal[b])
            r = rmin_half[a] + rmin_half[b]
            off = ntypes * a + b
            lj1[off] = 12.0 * e * r ** 12
            lj2[off] = 12.0 * e * r ** 6
            lj3[off] = e * r ** 12
            lj4[off] = 2.0 * e * r ** 6
            lj14[0, a, b] = 0.5 * 12.0 * e * r ** 12
            lj14[1, a, b] = 0.5 * 12.0 * e * r ** 6
            lj14[2, a, b] = 0.5 * e * r ** 12
            lj14[3, a, b] = e * r ** 6
    return lj1, lj2, lj3, lj4, lj14


def _rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _unit(v):
    return v / np.linalg.norm(v)


def _tetra_pair(center, a, b, length):
    """Two remaining tetrahedral substituent positions of ``center`` given neighbours a, b."""
    u = _unit(a - center)
    v = _unit(b - center)
    bis = -_unit(u + v)
    n = _unit(np.cross(u, v))
    half = math.radians(_TET) / 2.0
    d1 = math.cos(half) * bis + math.sin(half) * n
    d2 = math.cos(half) * bis - math.sin(half) * n
    return center + length * d1, center + length * d2


def glycine_template() -> np.ndarray:
    """Zwitterion glycine (template order C, CA, N, O1, O2, HN1-3, HA1-2), Angstrom."""
    ca = np.zeros(3)
    c = np.array([1.52, 0.0, 0.0])
    th = math.radians(_TET)
    n = 1.47 * np.array([math.cos(th), math.sin(th), 0.0])
    # carboxylate: O's at 120 deg around C in the N-CA-C plane
    u = _unit(ca - c)
    perp = np.array([-u[1], u[0], 0.0])
    o1 = c + 1.25 * (math.cos(math.radians(120)) * u + math.sin(math.radians(120)) * perp)
    o2 = c + 1.25 * (math.cos(math.radians(120)) * u - math.sin(math.radians(120)) * perp)
    ha1, ha2 = _tetra_pair(ca, c, n, 1.09)
    # ammonium: three H staggered around the CA-N axis
    axis = _unit(n - ca)
    ref = _unit(np.cross(axis, np.array([0.0, 0.0, 1.0])))
    ref2 = np.cross(axis, ref)
    hs = []
    for k in range(3):
        phi = 2.0 * math.pi * k / 3.0
        radial = math.cos(phi) * ref + math.sin(phi) * ref2
        d = math.cos(math.pi - th) * axis + math.sin(math.pi - th) * radial
        hs.append(n + 1.01 * _unit(d))
    pts = np.array([c, ca, n, o1, o2, hs[0], hs[1], hs[2], ha1, ha2])
    return pts - pts.mean(axis=0)


def water_template() -> np.ndarray:
    th = math.radians(_TET) / 2.0
    o = np.zeros(3)
    h1 = WATER_OH * np.array([math.sin(th), math.cos(th), 0.0])
    h2 = WATER_OH * np.array([-math.sin(th), math.cos(th), 0.0])
    pts = np.array([o, h1, h2])
    return pts - pts.mean(axis=0)


def box_length(n_gly: int, n_wat: int, density_gcc: float = 1.0) -> float:
    mass = n_gly * GLY_MASS + n_wat * WAT_MASS
    return (mass * AMU_PER_A3_TO_GCC / density_gcc) ** (1.0 / 3.0)


def wrap_positions(xyz: np.ndarray, box: np.float32) -> np.ndarray:
    """Wrap to (0, box] in float32 exactly like ``pbc`` (``Source/mod_pbc.f90:6-39``)."""
    out = xyz.astype(np.float32).copy()
    b = np.float32(box)
    for _ in range(8):
        hi = out > b
        lo = out <= np.float32(0.0)
        if not hi.any() and not lo.any():
            break
        out[hi] = out[hi] - b
        out[lo] = out[lo] + b
    return out


def _push_apart(xyz: np.ndarray, mol: np.ndarray, n_mol: int, L: float,
                d_min: float = 2.2, rounds: int = 40, step_cap: float = 0.4) -> np.ndarray:
    """Rigidly translate molecules apart until no inter-molecular atom pair is closer
    than ``d_min`` Angstrom (or ``rounds`` is reached).

    A lattice at 1.0 g/cm^3 with randomly oriented glycines puts some atoms of
    neighbouring molecules on top of each other; this removes those clashes
    without changing any intramolecular geometry, so forces stay finite and
    the fixed-point force range is respected.
    """
    from scipy.spatial import cKDTree

    x = np.mod(xyz, L)
    for _ in range(rounds):
        tree = cKDTree(np.mod(x, L), boxsize=L)
        pairs = tree.query_pairs(d_min, output_type="ndarray")
        if len(pairs) == 0:
            break
        inter = mol[pairs[:, 0]] != mol[pairs[:, 1]]
        pairs = pairs[inter]
        if len(pairs) == 0:
            break
        d = x[pairs[:, 0]] - x[pairs[:, 1]]
        d -= L * np.round(d / L)
        r = np.linalg.norm(d, axis=1)
        if r.min() > d_min - 0.4:
            break  # no clash left (closest contact >= d_min - 0.4 A)
        r = np.maximum(r, 1e-3)
        push = (0.5 * (d_min - r) / r)[:, None] * d
        disp = np.zeros((n_mol, 3))
        np.add.at(disp, mol[pairs[:, 0]], push)
        np.add.at(disp, mol[pairs[:, 1]], -push)
        nrm = np.linalg.norm(disp, axis=1)
        scale = np.where(nrm > step_cap, step_cap / np.maximum(nrm, 1e-12), 1.0)
        disp *= scale[:, None]
        x = x + disp[mol]
    return x


def _partner_lists(n_atoms: int, bonds: list[tuple[int, int]]):
    adj = [set() for _ in range(n_atoms)]
    for a, b in bonds:
        adj[a].add(b)
        adj[b].add(a)
    p12, p13, p14 = [], [], []
    for i in range(n_atoms):
        s12 = sorted(adj[i])
        s13 = sorted({k for j in adj[i] for k in adj[j]} - {i} - set(s12))
        s14 = sorted({l for k in s13 for l in adj[k]} - {i} - set(s12) - set(s13))
        # a 1-4 partner must be reachable by a 3-bond path through a 1-2 then 1-3 atom
        s14 = [l for l in s14 if any(l in adj[k] and k in {m for j in adj[i] for m in adj[j]}
                                     for k in adj[l])]
        p12.append(s12)
        p13.append(s13)
        p14.append(s14)
    return p12, p13, p14


def _nucleus_centres(k: int, spacing: float, L: float) -> np.ndarray:
    """k points of an fcc lattice (nearest-neighbour distance ``spacing``) closest to
    the box centre: a compact, crystal-like glycine nucleus."""
    a = spacing * math.sqrt(2.0)
    n = int(math.ceil((4.0 * k) ** (1.0 / 3.0))) + 2
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(-n, n + 1)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pts = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    order = np.argsort(np.einsum("ij,ij->i", pts, pts), kind="stable")
    return pts[order[:k]] + 0.5 * L


def make_system(n_gly: int, n_wat: int, seed: int, *, jitter_a: float = 0.2,
                density_gcc: float = 1.0, temperature: float = 300.0, nucleus: int = 0,
                nucleus_spacing: float = 5.5) -> SofiaSystem:
    """Build a seeded glycine/water system: cubic lattice, random orientation, jitter.

    ``nucleus`` > 0 places that many glycine molecules (the first ones) as a
    compact fcc cluster with one common orientation at the box centre, centres
    ``nucleus_spacing`` A apart, so that the largest-cluster analysis finds a
    solid nucleus; the other molecules fill the lattice sites away from it."""
    rng = np.random.default_rng(seed)
    L = box_length(n_gly, n_wat, density_gcc)
    box = np.float32(L)
    n_mol = n_gly + n_wat
    nuc = min(max(int(nucleus), 0), n_gly)
    centres_nuc = _nucleus_centres(nuc, nucleus_spacing, L) if nuc else np.zeros((0, 3))
    m = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    while True:
        a = L / m
        grid = np.arange(m ** 3)
        cen = (np.stack([grid % m, (grid // m) % m, grid // (m * m)], -1) + 0.5) * a
        if nuc:
            d = cen[:, None, :] - centres_nuc[None, :, :]
            d -= L * np.round(d / L)
            free = (np.einsum("ijk,ijk->ij", d, d) > (0.75 * nucleus_spacing) ** 2).all(axis=1)
        else:
            free = np.ones(m ** 3, bool)
        if free.sum() >= n_mol - nuc:
            break
        m += 1
    sites = rng.permutation(np.nonzero(free)[0])[:n_mol - nuc]
    # glycine molecules take the first n_gly of the permuted sites
    gt = glycine_template()
    wt = water_template()
    coords = []
    rot_nuc = _rotation(rng)
    for mol in range(n_mol):
        if mol < nuc:
            coords.append(gt @ rot_nuc.T + centres_nuc[mol])
            continue
        s = int(sites[mol - nuc])
        centre = cen[s]
        rot = _rotation(rng)
        tmpl = gt if mol < n_gly else wt
        pts = tmpl @ rot.T + centre
        pts = pts + rng.uniform(-jitter_a, jitter_a, size=3)  # rigid per-molecule jitter
        coords.append(pts)
    xyz = np.concatenate(coords).astype(np.float64)
    mol = np.concatenate([np.full(10, k, np.int64) for k in range(n_gly)] +
                         [np.full(3, n_gly + k, np.int64) for k in range(n_wat)])
    xyz = _push_apart(xyz, mol, n_mol, L)
    xyz32 = wrap_positions(xyz.astype(np.float32), box)

    types = np.array(GLY_TYPES * n_gly + WAT_TYPES * n_wat, dtype=np.int32)
    q = np.array([_CHARGE[t - 1] for t in types], dtype=np.float32)
    ntypes = len(TYPE_NAMES)
    sig_a = np.array(_SIG_NM) * 10.0
    eps_kcal = np.array(_EPS_KJ) / 4.184
    lj1, lj2, lj3, lj4, lj14 = lj_tables_4eps(ntypes, sig_a, eps_kcal)

    return _assemble(n_gly, n_wat, box, xyz32, types, q, np.array(_MASS, np.float64), ntypes,
                     (lj1, lj2, lj3, lj4, lj14), rng, temperature, seed)


def _assemble(n_gly, n_wat, box, xyz32, types, q, mass_type, ntypes, tables, rng,
              temperature, seed, *, water_shake=(WATER_OH, WATER_OH, WATER_HH)):
    lj1, lj2, lj3, lj4, lj14 = tables
    np_atoms = n_gly * 10 + n_wat * 3
    # exclusion partners per template
    g12, g13, g14 = _partner_lists(10, GLY_BONDS)
    w12, w13, w14 = _partner_lists(3, WAT_BONDS)
    specbond = np.zeros((np_atoms, 12), np.int32)
    n1 = np.zeros(np_atoms, np.int32)
    n2 = np.zeros(np_atoms, np.int32)
    n3 = np.zeros(np_atoms, np.int32)

    def fill(base, p12, p13, p14, natom):
        for k in range(natom):
            i = base + k
            parts = [base + j + 1 for j in p12[k]] + [base + j + 1 for j in p13[k]] + \
                    [base + j + 1 for j in p14[k]]
            assert len(parts) <= 12
            specbond[i, :len(parts)] = parts
            n1[i] = len(p12[k])
            n2[i] = len(p12[k]) + len(p13[k])
            n3[i] = len(parts)

    bonds, angles, diheds, shake, shake_bond, impros = [], [], [], [], [], []
    bond_types = {}
    bond_coeff = []
    for key in GLY_BONDS:
        bond_types[key] = len(bond_coeff) + 1
        bond_coeff.append((_BOND_K[key], _BOND_R0[key]))
    wat_bond_type = len(bond_coeff) + 1
    bond_coeff.append((600.0, WATER_OH))
    angle_coeff = [(k, math.radians(t0)) for (_, k, t0) in GLY_ANGLES] + \
                  [(WAT_ANGLES[0][1], math.radians(WAT_ANGLES[0][2]))]
    for g in range(n_gly):
        base = 10 * g
        fill(base, g12, g13, g14, 10)
        for key in GLY_BONDS:
            bonds.append((base + key[0] + 1, base + key[1] + 1, bond_types[key]))
        for t, (idx, _, _) in enumerate(GLY_ANGLES):
            angles.append((base + idx[0] + 1, base + idx[1] + 1, base + idx[2] + 1, t + 1))
        for idx, t in GLY_DIHEDRALS:
            diheds.append(tuple(base + i + 1 for i in idx) + (t,))
        # CH2: centre CA with HA1, HA2; NH3: centre N with HN1..3
        shake.append((3, base + 2, base + 9, base + 10, 0))
        shake_bond.append((1.09, 1.09, 0.0))
        shake.append((4, base + 3, base + 6, base + 7, base + 8))
        shake_bond.append((1.01, 1.01, 1.01))
        impros.append(tuple(base + i + 1 for i in GLY_IMPROPER) + (1,))
    for w in range(n_wat):
        base = 10 * n_gly + 3 * w
        fill(base, w12, w13, w14, 3)
        bonds.append((base + 1, base + 2, wat_bond_type))
        bonds.append((base + 1, base + 3, wat_bond_type))
        angles.append((base + 2, base + 1, base + 3, len(GLY_ANGLES) + 1))
        shake.append((-3, base + 1, base + 2, base + 3, 0))
        shake_bond.append(water_shake)

    # Maxwell-Boltzmann velocities in Angstrom/fs: sigma_v = sqrt(kB T / m) with
    # kB T in kcal/mol converted through kcal2amu (reference get_started.f90:32,38).
    impro_arr = np.array(impros, np.int32).reshape(-1, 5)
    omega0 = float(np.mean(improper_omega(xyz32, box, impro_arr[:, :4] - 1))) if n_gly else 0.0
    kboltz = 0.001987204181
    kcal2amu = 0.0004184
    m_atom = mass_type[types - 1]
    sig = np.sqrt(kboltz * temperature * kcal2amu / m_atom)
    vel = (rng.normal(size=(np_atoms, 3)) * sig[:, None]).astype(np.float32)

    return SofiaSystem(
        n_gly=n_gly, n_wat=n_wat, box=np.float32(box), position=None, xyz=xyz32, types=types,
        q=q, mass_type=mass_type, ntypes=ntypes, lj1=lj1, lj2=lj2, lj3=lj3, lj4=lj4, lj14=lj14,
        specbond=specbond, num1bond=n1, num2bond=n2, num3bond=n3,
        bonds=np.array(bonds, np.int32).reshape(-1, 3),
        bond_coeff=np.array(bond_coeff, np.float64),
        angles=np.array(angles, np.int32).reshape(-1, 4),
        angle_coeff=np.array(angle_coeff, np.float64),
        dihedrals=np.array(diheds, np.int32).reshape(-1, 5),
        dihed_coeff=np.zeros((2, 4), np.float64),
        shake=np.array(shake, np.int32).reshape(-1, 5),
        shake_bond=np.array(shake_bond, np.float64).reshape(-1, 3),
        velocity=vel, seed=seed, impropers=impro_arr,
        impro_coeff=np.array([[GLY_IMPROPER_K, omega0]], np.float64))


# Named workloads (composition, seeds).  N = 10*n_gly + 3*n_wat.
WORKLOADS = {
    "gly150_wat2500_9k": (150, 2500),
    "gly1500_wat25000_90k": (1500, 25000),
    "gly3500_wat80000_275k": (3500, 80000),
}


def make_workload(name: str, seed: int = 0) -> SofiaSystem:
    n_gly, n_wat = WORKLOADS[name]
    return make_system(n_gly, n_wat, seed)


def random_replica(rng: np.random.Generator, n_min: int, n_max: int, gly_frac=(0.05, 0.20),
                   seed: int = 0, nucleus: int = 0) -> SofiaSystem:
    """A replica of N ~ U[n_min, n_max] atoms with glycine a seeded fraction of molecules."""
    n_target = int(rng.integers(n_min, n_max + 1))
    f = float(rng.uniform(*gly_frac))
    # N = 10 g + 3 w, g = f (g + w)  =>  g = f N / (10 f + 3 (1 - f))
    n_gly = max(1, int(round(f * n_target / (10 * f + 3 * (1 - f)))))
    n_wat = max(1, int(round((n_target - 10 * n_gly) / 3)))
    return make_system(n_gly, n_wat, seed, nucleus=min(nucleus, n_gly))
