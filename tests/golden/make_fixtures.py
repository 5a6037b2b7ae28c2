"""Generates the reference-input fixture used by the parity tests.

Reads the reference's own input files (the minimized glycine_1500 and
glycine_2500 snapshots,
its topology, molecule templates and run input) from the reference checkout,
parses them with ``molecular_simulation_code_b200.snapio`` and writes the
parsed numbers to ``glycine_1500_solv_min.npz`` and ``glycine_2500_solv_min.npz``
beside this script:

* ``xyz_mnm`` int16 (N,3): the .gro coordinates in units of 0.001 nm (the
  file's 8.3 fields, exactly);
* ``box_nm_1e5``: the box line's f10.5 value times 1e5;
* ``mol_*``: molecule counts (from the snapshot's residues), atoms per molecule,
  template atom types;
* ``top_*``: topology tables as parsed by ``snapio.parse_topol``;
* ``run_*``: cutoffs, padding, cluster radii, DSF alpha, time step and the
  1-2/1-3/1-4 factors of the run input.

Run it from the repository root:  python tests/golden/make_fixtures.py REFERENCE_ROOT
(REFERENCE_ROOT = the checkout holding input_files/).
The tests only read the .npz; the reference checkout is not needed to run them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from molecular_simulation_code_b200 import snapio  # noqa: E402


def _run_input(text: str) -> dict:
    """The few numbers of the run input the kernels need, by their labels."""
    lines = text.splitlines()

    def after(label):
        for k, ln in enumerate(lines):
            if ln.startswith(label):
                return lines[k + 1].split()
        raise KeyError(label)

    cut = after("!---rcuts")
    return {"rcut": float(cut[0]), "cut_coul": float(cut[1]), "pad": float(cut[2]),
            "mrcut": float(cut[3]), "denscut": float(cut[4]), "densmin": int(cut[5]),
            "alpha": float(after("!---alpha")[0]), "dt": float(after("!---deltat")[0]),
            "fudge": np.array([float(v) for v in after("!---12 13 14")[:4]])}


def fixture(d: str, gro_name: str):
    gro = open(os.path.join(d, gro_name)).read()
    lines = gro.splitlines()
    n = int(lines[1].split()[0])
    mnm = np.empty((n, 3), np.int32)
    for i in range(n):
        ln = lines[2 + i]
        for c in range(3):
            mnm[i, c] = int(round(float(ln[20 + 8 * c:28 + 8 * c]) * 1000.0))
    assert np.abs(mnm).max() < 32768
    box_1e5 = int(round(float(lines[2 + n][:10]) * 1e5))
    mol = snapio.parse_mol(open(os.path.join(d, "mol_cndo_alpha.input")).read())
    # molecule counts of this snapshot from its residues (the molecule template file
    # holds the counts of the 1500-glycine system): 10-atom glycine, 3-atom water
    resnames = [lines[2 + i][5:10].strip() for i in range(n)]
    n_gly = sum(1 for r in resnames if r != "SOL") // 10
    n_wat = sum(1 for r in resnames if r == "SOL") // 3
    assert 10 * n_gly + 3 * n_wat == n
    mol["counts"] = np.array([n_gly, n_wat], np.int32)
    top = snapio.parse_topol(open(os.path.join(d, "topol_cndo.top")).read(), len(mol["counts"]))
    run = _run_input(open(os.path.join(d, "input")).read())
    out = {"xyz_mnm": mnm.astype(np.int16), "box_nm_1e5": np.int64(box_1e5)}
    out.update({"mol_" + k: v for k, v in mol.items()})
    out.update({"top_" + k: np.asarray(v) for k, v in top.items()})
    out.update({"run_" + k: np.asarray(v) for k, v in run.items()})
    path = os.path.join(HERE, gro_name.replace(".gro", ".npz"))
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes;", n, "atoms;", n_gly, "glycine,", n_wat, "water")


def main(ref_root: str):
    d = os.path.join(ref_root, "input_files")
    for name in ("glycine_1500_solv_min.gro", "glycine_2500_solv_min.gro"):
        fixture(d, name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py REFERENCE_ROOT")
    main(sys.argv[1])
