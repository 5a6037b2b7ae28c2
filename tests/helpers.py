"""Shared test helpers: seeded systems, parameter sets and pair-set utilities."""
from __future__ import annotations

import functools

import numpy as np

from molecular_simulation_code_b200.system import make_system


@functools.lru_cache(maxsize=None)
def small_system(n_gly=10, n_wat=300, seed=3):
    return make_system(n_gly, n_wat, seed)


def ref_params(s, cut=7.0, pad=1.5, alpha=0.2):
    """Cut-offs for small boxes (>= 3 cells per side), reference units."""
    from molecular_simulation_code_b200.nonbond import DsfParams
    return DsfParams(alpha=alpha, box=s.box, cut_coul=cut, rcut=cut, neighbor_pad=pad)


def pair_set(nlist, numneigh, neigh_alloc, ids=None):
    """Set of (i, j) 1-based pairs of a full list; ``ids`` maps list ids to global ids."""
    out = set()
    n = numneigh.shape[0]
    for i in range(n):
        row = nlist[i * neigh_alloc:i * neigh_alloc + numneigh[i]]
        gi = i + 1 if ids is None else int(ids[i])
        for j in row:
            out.add((gi, int(j) if ids is None else int(ids[j - 1])))
    return out


def rows(nlist, numneigh, neigh_alloc):
    return [nlist[i * neigh_alloc:i * neigh_alloc + numneigh[i]].tolist()
            for i in range(numneigh.shape[0])]


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
