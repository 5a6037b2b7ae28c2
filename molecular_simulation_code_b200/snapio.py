"""Snapshot and topology I/O in the reference's formats.

* ``.gro`` coordinates: ``read_in_Grofile`` / ``read_in_Grofile_box``
  (Source/mod_GroFile.f90:89-159).  Coordinates in nm are read as real*4 and
  scaled by 10.0d0 into real*4 Angstrom; the box is the first f10.5 field of the
  last line, scaled the same way.
* restart dumps: ``dump_global_velocity_id_mpi`` / ``read_dump_global_id_v``
  (Source/mod_datadump.f90:113-153, 216-252): box, temperature, cluster size,
  time, then one ``(i5,6f12.6)`` record per atom (global id, x, y, z in A,
  vx, vy, vz in A/fs).  The reference's i5 field overflows above 99,999 atoms;
  the writer here widens the id field instead (the reader accepts both).
* topology (``read_topol``, Source/mod_readfile.f90:227-562) and molecule
  templates (``read_gro_input``, :188-225).
* ``build_reference_system`` lays out the module state exactly as the reference
  does (``assign_atom_types``/``assign_charge_types``, Source/mod_assign_types.f90:7-66;
  ``build_spec_bond_list_once``, Source/mod_buildbond_lists.f90:80-118;
  AMBER Rmin/2 tables of ``check_topol_file``, Source/mod_readfile.f90:597-615).
"""
from __future__ import annotations

import math

import numpy as np

from .system import SofiaSystem, improper_omega, lj_tables_rmin


def _f32_times10(v):
    """real*4 value read from text, times 10.0d0, stored in real*4."""
    return np.float32(np.float64(np.float32(v)) * 10.0)


# ------------------------------------------------------------------ .gro
def read_gro(text: str):
    """Returns (xyz float32 (N,3) in A, box float32 in A, atom names)."""
    lines = text.splitlines()
    n = int(lines[1].split()[0])
    xyz = np.empty((n, 3), np.float32)
    names = []
    for i in range(n):
        ln = lines[2 + i]
        names.append(ln[10:15].strip())
        vals = (ln[20:28], ln[28:36], ln[36:44])
        xyz[i] = [_f32_times10(float(v)) for v in vals]
    box = _f32_times10(float(lines[2 + n][0:10]))
    return xyz, box, names


def write_gro(path: str, xyz, box, names=None, resnames=None, resids=None, title="SOFIA"):
    n = xyz.shape[0]
    with open(path, "w") as f:
        f.write(f"{title}\n{n:5d}\n")
        for i in range(n):
            rn = resids[i] if resids is not None else 1
            rname = resnames[i] if resnames is not None else "MOL"
            an = names[i] if names is not None else "X"
            x, y, z = (float(c) / 10.0 for c in xyz[i])
            f.write(f"{rn % 100000:5d}{rname:<5s}{an:>5s}{(i + 1) % 100000:5d}"
                    f"{x:8.3f}{y:8.3f}{z:8.3f}\n")
        b = float(box) / 10.0
        f.write(f"{b:10.5f}{b:10.5f}{b:10.5f}\n")


# ------------------------------------------------------------- restart
def write_restart(path: str, box, temp, cluster_num, time_fs, gid, x, v):
    """Reference restart dump; records in input order with their global ids."""
    n = len(gid)
    width = max(5, len(str(int(np.max(gid))))) if n else 5
    with open(path, "w") as f:
        f.write(f" {float(np.float32(box)):.9g}\n {float(temp):.17g}\n {int(cluster_num)}\n"
                f" {float(time_fs):.17g}\n")
        for i in range(n):
            f.write(f"{int(gid[i]):{width}d}" + "".join(f"{float(c):12.6f}" for c in x[i]) +
                    "".join(f"{float(c):12.6f}" for c in v[i]) + "\n")


def _restart_record(ln: str):
    """One ``(i5,6f12.6)`` record; list-directed like the reference, with a
    fixed-column fallback for fields that touch (a full f12.6 field or an id
    wider than i5)."""
    f = ln.split()
    if len(f) != 7:
        body = ln.rstrip("\n")
        f = [body[:-72]] + [body[len(body) - 72 + 12 * k:len(body) - 60 + 12 * k] for k in range(6)]
    return int(f[0]), [np.float32(float(c)) for c in f[1:4]], [np.float32(float(c)) for c in f[4:7]]


def read_restart(path: str, np_atoms: int):
    """read_dump_global_id_v: box, temperature, cluster size, time, then x (N,3)
    and v (N,3) placed by global id, all real*4."""
    with open(path) as f:
        box = np.float32(float(f.readline()))
        temp = float(f.readline())
        num = int(float(f.readline()))
        tclock = float(f.readline())
        x = np.zeros((np_atoms, 3), np.float32)
        v = np.zeros((np_atoms, 3), np.float32)
        seen = np.zeros(np_atoms, bool)
        for _ in range(np_atoms):
            ln = f.readline()
            if not ln.strip():
                raise ValueError(f"restart file {path}: fewer than {np_atoms} atom records")
            j, xx, vv = _restart_record(ln)
            if not 1 <= j <= np_atoms:
                raise ValueError(f"restart file {path}: global id {j} outside 1..{np_atoms}")
            x[j - 1] = xx
            v[j - 1] = vv
            seen[j - 1] = True
    if not seen.all():
        raise ValueError(f"restart file {path}: {int((~seen).sum())} atoms missing")
    return box, temp, num, tclock, x, v


# --------------------------------------------------- list-directed records
class _Records:
    """Fortran list-directed reading over text records: ``skip`` is ``read(u,*)``
    with no items; ``values(n)`` reads n items, passing over blank records and
    ignoring what follows the n-th item on its record."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.k = 0

    def skip(self, n: int = 1):
        self.k += n

    def values(self, n: int) -> list[str]:
        out: list[str] = []
        while len(out) < n:
            if self.k >= len(self.lines):
                raise ValueError("unexpected end of file")
            f = self.lines[self.k].split()
            self.k += 1
            out += f[:n - len(out)]
        return out


# -------------------------------------------------- molecule templates
def parse_mol(text: str) -> dict:
    """read_gro_input (Source/mod_readfile.f90:188-225): molecule types, their
    counts, atoms per molecule and the atom type of each template atom."""
    r = _Records(text)
    r.skip()
    nmt = int(r.values(1)[0])
    counts, natoms, types = [], [], []
    for _ in range(nmt):
        r.skip()
        counts.append(int(r.values(1)[0]))
        natoms.append(int(r.values(1)[0]))
        for _ in range(natoms[-1]):
            types.append(int(r.values(5)[0]))  # type, atom no, x, y, z
    return {"counts": np.array(counts, np.int32), "natoms": np.array(natoms, np.int32),
            "types": np.array(types, np.int32)}


# ------------------------------------------------------------ topology
_SHAKE_SHAPE = {1: (2, 1), 3: (3, 2), 4: (4, 3), -3: (3, 3)}  # atoms, bond lengths


def parse_topol(text: str, n_moltypes: int) -> dict:
    """read_topol (Source/mod_readfile.f90:227-562) as numeric arrays.

    types (nt,4): Rmin/2, eps, q, mass.  bonds: moltype, type, a1, a2, kb, r0.
    angles: moltype, type, a1, a2 (middle), a3, k, theta0 (degrees).  diheds:
    moltype, type, a1..a4, K, multiplicity, shift.  impros: moltype, type,
    a1..a4, k, sign, multiplicity.  shake (groups, 9): num, moltype, a1..a4
    (0 unused), bond lengths 1..3.  Atom numbers are 1-based within a molecule.
    """
    r = _Records(text)
    r.skip()
    nt = int(r.values(1)[0])
    r.skip()
    types = []
    for _ in range(nt):
        f = r.values(7)
        types.append([float(f[3]), float(f[4]), float(f[5]), float(f[6])])

    def section(ncols):
        r.skip(2)
        ntyp, nrows = (int(v) for v in r.values(2))
        r.skip()
        rows = [[float(v) for v in r.values(ncols)] for _ in range(nrows)]
        return ntyp, np.array(rows, np.float64).reshape(-1, ncols)

    nbt, bonds = section(6)
    nat, angles = section(7)
    ndt, diheds = section(9)
    nit, impros = section(9)
    r.skip(3)
    per_mol = [int(r.values(1)[0]) for _ in range(n_moltypes)]
    r.skip(2)
    groups = []
    for _ in range(sum(per_mol)):
        num = int(r.values(1)[0])
        if num not in _SHAKE_SHAPE:
            raise ValueError(f"unknown SHAKE group kind {num}")
        na, nb = _SHAKE_SHAPE[num]
        f = r.values(1 + na + nb)
        atoms = [int(v) for v in f[1:1 + na]] + [0] * (4 - na)
        lens = [float(v) for v in f[1 + na:]] + [0.0] * (3 - nb)
        groups.append([num, int(f[0])] + atoms + lens)
    return {"types": np.array(types, np.float64), "nbondtypes": nbt, "bonds": bonds,
            "nangletypes": nat, "angles": angles, "ndihedtypes": ndt, "diheds": diheds,
            "nimprotypes": nit, "impros": impros,
            "shake": np.array(groups, np.float64).reshape(-1, 9)}


# --------------------------------------------------- module state build
def build_reference_system(mol: dict, top: dict, xyz: np.ndarray, box,
                           velocity: np.ndarray | None = None) -> SofiaSystem:
    ntypes = top["types"].shape[0]
    rmin_half = top["types"][:, 0]
    eps = top["types"][:, 1]
    qtype = top["types"][:, 2].astype(np.float32)  # q is real*4
    mass_type = top["types"][:, 3].astype(np.float64)
    lj1, lj2, lj3, lj4, lj14 = lj_tables_rmin(ntypes, rmin_half, eps)
    counts, natoms = mol["counts"], mol["natoms"]
    tstart = np.concatenate([[0], np.cumsum(natoms)])
    # per-moltype partner lists in reference order (1-2 from bonds, 1-3 from angles,
    # 1-4 from torsions; Source/mod_readfile.f90:292-402)
    part = []
    for mt in range(len(counts)):
        na = int(natoms[mt])
        p12 = [[] for _ in range(na)]
        p13 = [[] for _ in range(na)]
        p14 = [[] for _ in range(na)]
        for r in top["bonds"]:
            if int(r[0]) == mt + 1:
                a1, a2 = int(r[2]) - 1, int(r[3]) - 1
                p12[a1].append(a2)
                p12[a2].append(a1)
        for r in top["angles"]:
            if int(r[0]) == mt + 1:
                a1, a3 = int(r[2]) - 1, int(r[4]) - 1
                p13[a1].append(a3)
                p13[a3].append(a1)
        for r in top["diheds"]:
            if int(r[0]) == mt + 1:
                a1, a4 = int(r[2]) - 1, int(r[5]) - 1
                p14[a1].append(a4)
                p14[a4].append(a1)
        part.append((p12, p13, p14))
    n = int(np.sum(counts * natoms))
    types = np.empty(n, np.int32)
    specbond = np.zeros((n, 12), np.int32)
    n1 = np.zeros(n, np.int32)
    n2 = np.zeros(n, np.int32)
    n3 = np.zeros(n, np.int32)
    bonds, angles, diheds, shake, sbond, impros = [], [], [], [], [], []
    base = 0
    for mt in range(len(counts)):
        na = int(natoms[mt])
        tmpl_types = mol["types"][tstart[mt]:tstart[mt + 1]]
        p12, p13, p14 = part[mt]
        for _ in range(int(counts[mt])):
            for a in range(na):
                i = base + a
                types[i] = tmpl_types[a]
                lst = [base + j + 1 for j in p12[a] + p13[a] + p14[a]]
                if len(lst) > 12:
                    raise ValueError("more than 12 exclusion partners")
                specbond[i, :len(lst)] = lst
                n1[i] = len(p12[a])
                n2[i] = len(p12[a]) + len(p13[a])
                n3[i] = len(lst)
            for r in top["bonds"]:
                if int(r[0]) == mt + 1:
                    bonds.append((base + int(r[2]), base + int(r[3]), int(r[1])))
            for r in top["angles"]:
                if int(r[0]) == mt + 1:
                    angles.append((base + int(r[2]), base + int(r[3]), base + int(r[4]),
                                   int(r[1])))
            for r in top["diheds"]:
                if int(r[0]) == mt + 1:
                    diheds.append(tuple(base + int(r[c]) for c in (2, 3, 4, 5)) + (int(r[1]),))
            for r in top["impros"]:
                if int(r[0]) == mt + 1:
                    impros.append(tuple(base + int(r[c]) for c in (2, 3, 4, 5)) + (int(r[1]),))
            for g in top["shake"]:
                if int(g[1]) == mt + 1:
                    num = int(g[0])
                    atoms = [base + int(a) if int(a) > 0 else 0 for a in g[2:6]]
                    shake.append([num] + atoms)
                    sbond.append(list(g[6:9]))
            base += na
    q = qtype[types - 1]
    bond_coeff = np.zeros((max(top["nbondtypes"], 1), 2))
    for r in top["bonds"]:
        bond_coeff[int(r[1]) - 1] = [r[4], r[5]]
    angle_coeff = np.zeros((max(top["nangletypes"], 1), 2))
    for r in top["angles"]:
        angle_coeff[int(r[1]) - 1] = [r[5], r[6] * (2.0 * math.acos(-1.0) / 360.0)]
    n_gly = int(counts[0]) if natoms[0] == 10 else 0
    vel = velocity if velocity is not None else np.zeros((n, 3), np.float32)
    # impropers: k from the topology; the reference reads no equilibrium angle
    # (read_topol leaves theta0 unset, Source/mod_readfile.f90:433), so omega0 is the
    # mean angle of each improper type in the given snapshot
    impro_arr = np.array(impros, np.int32).reshape(-1, 5)
    nit = max(int(top["nimprotypes"]), 1)
    impro_coeff = np.zeros((nit, 2))
    for r in top["impros"]:
        impro_coeff[int(r[1]) - 1, 0] = r[6]
    for t in range(nit):
        sel = impro_arr[impro_arr[:, 4] == t + 1]
        if len(sel):
            impro_coeff[t, 1] = float(np.mean(improper_omega(xyz, box, sel[:, :4] - 1)))
    return SofiaSystem(
        n_gly=n_gly, n_wat=int(np.sum(counts)) - n_gly, box=np.float32(box), position=None,
        xyz=np.ascontiguousarray(xyz, np.float32), types=types, q=q, mass_type=mass_type,
        ntypes=ntypes, lj1=lj1, lj2=lj2, lj3=lj3, lj4=lj4, lj14=lj14, specbond=specbond,
        num1bond=n1, num2bond=n2, num3bond=n3,
        bonds=np.array(bonds, np.int32).reshape(-1, 3), bond_coeff=bond_coeff,
        angles=np.array(angles, np.int32).reshape(-1, 4), angle_coeff=angle_coeff,
        dihedrals=np.array(diheds, np.int32).reshape(-1, 5),
        dihed_coeff=np.zeros((max(top["ndihedtypes"], 1), 4)),
        shake=np.array(shake, np.int32).reshape(-1, 5),
        shake_bond=np.array(sbond, np.float64).reshape(-1, 3), velocity=vel, seed=0,
        impropers=impro_arr, impro_coeff=impro_coeff)


def load_fixture(path: str):
    """(SofiaSystem, run parameters) from a fixture written by
    tests/golden/make_fixtures.py: .gro fields stored as integers of 0.001 nm,
    converted exactly as read_in_Grofile does (real*4 nm times 10.0d0)."""
    d = np.load(path, allow_pickle=False)
    nm = (d["xyz_mnm"].astype(np.float64) / 1000.0).astype(np.float32)
    xyz = (nm.astype(np.float64) * 10.0).astype(np.float32)
    box = _f32_times10(float(d["box_nm_1e5"]) / 1e5)
    mol = {k[4:]: d[k] for k in d.files if k.startswith("mol_")}
    top = {k[4:]: (d[k] if d[k].ndim else d[k].item()) for k in d.files if k.startswith("top_")}
    run = {k[4:]: (d[k] if d[k].ndim else d[k].item()) for k in d.files if k.startswith("run_")}
    return build_reference_system(mol, top, xyz, box), run


# ------------------------------------------------ checkpoint / resume
def dump_restart(system, path: str, box, temp: float = 0.0, cluster_num: int = 0,
                 time_fs: float = 0.0):
    """Reference restart dump of a resident replica (``mixed.System``): the
    device state read back, rounded to real*4 and written as ``(i5,6f12.6)``
    records in global-id order, like dump_global_velocity_id_mpi."""
    x, v, _ = system.get_state()
    gid = np.arange(1, x.shape[0] + 1)
    write_restart(path, box, temp, cluster_num, time_fs, gid, x.astype(np.float32),
                  v.astype(np.float32))


def load_restart(system, path: str):
    """read_dump_global_id_v into a resident replica; returns (box, temp, cluster size, time)."""
    box, temp, num, tclock, x, v = read_restart(path, system.n)
    system.set_state(x.astype(np.float64), v.astype(np.float64))
    return box, temp, num, tclock


def save_checkpoint(system, path: str):
    """Exact checkpoint: FP64 positions and velocities and the thermostat step
    counter, so a resumed run continues bit for bit (the text restart keeps
    six decimals of real*4 only).  The checkpoint is taken at a snapshot, which
    makes this run rebuild its lists from the saved positions just as the
    resumed run will, so both continue identically."""
    system.snapshot()
    x, v, _ = system.get_state()
    np.savez(path, x=x, v=v, step=np.int64(system.md_step()))


def resume_checkpoint(system, path: str):
    d = np.load(path, allow_pickle=False)
    system.set_state(d["x"], d["v"])
    system.set_md_step(int(d["step"]))
