"""ctypes wrapper of the CPU restatement (``sofia_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / reference arm of ``bench.py``.  PARITY UNPINNED (the
Fortran reference cannot be built here and ships no golden outputs).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ["alpha", "EWALD_F", "EWALD_P", "A1", "A2", "A3", "A4", "A5", "MY_PIS",
                 "MY_PIS_INV", "e_shift", "f_shift"]] + \
               [("coulpre", C.c_float), ("box", C.c_float), ("ibox", C.c_float),
                ("vol", C.c_float), ("cut_coul", C.c_float), ("rcut", C.c_float),
                ("neighbor_pad", C.c_float)] + \
               [(n, C.c_double) for n in ["rcut2", "cut_coulsq", "rv", "rv2", "rvrc2"]]


def build() -> None:
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


_libs: dict[str, C.CDLL] = {}


def lib(fast: bool = False) -> C.CDLL:
    name = "libsofia_oracle_fast.so" if fast else "libsofia_oracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(_BUILD, name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    L.orc_init_params.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_float, C.c_float,
                                  C.c_float, C.c_float]
    L.orc_cell_grid.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float,
                                C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.orc_stencil.argtypes = [C.c_int, C.c_int, _i32p]
    L.orc_bin_sort.argtypes = [C.c_int, _f32p, C.c_float, C.c_float, C.c_int, C.c_int,
                               _i32p, _i32p, _i32p, _i32p, _i32p]
    L.orc_build_neighbor_nonewton.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _i32p,
                                              _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                                              C.c_int, C.c_int]
    L.orc_build_neighbor_nonewton.restype = C.c_int
    L.orc_neighbor_wrapper.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _i32p, _i32p,
                                       _i32p, _i32p, C.c_int, C.c_int]
    L.orc_neighbor_wrapper.restype = C.c_int
    L.orc_build_neighbor_n2.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _i32p, _i32p,
                                        _i32p, _i32p, C.c_int]
    L.orc_build_neighbor_n2.restype = C.c_int
    L.orc_force_dsf_nonewton.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _f32p, _f32p,
                                         _f32p, _f32p, _f32p, C.c_int, _i32p, _i32p, C.c_int,
                                         _f32p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         _f64p, C.c_void_p, C.c_int]
    L.orc_force_long_nonewton.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _f32p, _f32p,
                                          _f32p, _f32p, _f32p, C.c_int, _i32p, _i32p, C.c_int,
                                          C.c_double, _f32p, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), _f64p, C.c_void_p, C.c_int]
    L.orc_improper_harmonic.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, C.c_int, _i32p,
                                        _f64p, _f32p, C.POINTER(C.c_double), _f64p]
    L.orc_force_dsf_n2.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _f32p, _f32p, _f32p,
                                   _f32p, _f32p, C.c_int, _i32p, _i32p, _i32p, _i32p, _f64p,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_dihedral_opls_dsf.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p, _f32p, C.c_int,
                                        _f64p, C.c_int, _i32p, _f64p, _f32p,
                                        C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.c_void_p]
    L.orc_correct_pairs.argtypes = [C.POINTER(OrcParams), _f32p, _f32p, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_int, C.c_double, C.c_double, _f32p,
                                    C.POINTER(C.c_double), _f64p]
    L.orc_calculate_gewald.argtypes = [C.c_float]
    L.orc_calculate_gewald.restype = C.c_double
    L.orc_e_self_dsf.argtypes = [C.POINTER(OrcParams), C.c_int, _f32p]
    L.orc_e_self_dsf.restype = C.c_double
    L.orc_greatest_cluster.argtypes = [C.c_int, _f32p, _i32p, C.c_int, C.c_int, C.c_float,
                                       C.c_float, C.c_float, C.c_double, C.c_double, C.c_int,
                                       _f64p, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p]
    L.orc_greatest_cluster.restype = C.c_int
    L.orc_bond_harmonic.argtypes = [C.POINTER(OrcParams), _f32p, C.c_int, _i32p, _f64p, _f64p,
                                    C.POINTER(C.c_double)]
    L.orc_angle_harmonic.argtypes = [C.POINTER(OrcParams), _f32p, C.c_int, _i32p, _f64p, _f64p,
                                     C.POINTER(C.c_double)]
    L.orc_shake.argtypes = [C.c_int, _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_int, _i32p,
                            _f64p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double]
    L.orc_shake.restype = C.c_int
    _libs[name] = L
    return L


def params(alpha: float, box: float, cut_coul: float, rcut: float, pad: float) -> OrcParams:
    p = OrcParams()
    lib().orc_init_params(C.byref(p), float(alpha), np.float32(box), np.float32(cut_coul),
                          np.float32(rcut), np.float32(pad))
    return p


def cell_grid(p: OrcParams):
    rn = C.c_float()
    nt = C.c_int()
    nd = C.c_int()
    lib().orc_cell_grid(p.box, p.vol, p.cut_coul, p.rcut, C.byref(rn), C.byref(nt), C.byref(nd))
    return float(rn.value), int(nt.value), int(nd.value)


def stencil(ncellT: int, ncellD: int) -> np.ndarray:
    out = np.zeros(27 * ncellT, np.int32)
    lib().orc_stencil(ncellT, ncellD, out)
    return out


def bin_sort(p: OrcParams, pos: np.ndarray):
    """new_nlist + sort_posit_charge: returns tt, ttb (1-based), start, endposit, atombin."""
    rn, nt, nd = cell_grid(p)
    n = pos.shape[0]
    tt = np.zeros(n, np.int32)
    ttb = np.zeros(n, np.int32)
    st = np.zeros(nt, np.int32)
    en = np.zeros(nt, np.int32)
    ab = np.zeros(n, np.int32)
    lib().orc_bin_sort(n, np.ascontiguousarray(pos, np.float32), p.box, np.float32(rn), nt, nd,
                       tt, ttb, st, en, ab)
    return tt, ttb, st, en, ab


def neighbor_wrapper(p: OrcParams, pos: np.ndarray, specbond: np.ndarray, num3bond: np.ndarray,
                     neigh_alloc: int, nthreads: int = 0, fast: bool = False):
    """Full reference list in input index space; grows neigh_alloc like the redo loop."""
    n = pos.shape[0]
    while True:
        nlist = np.zeros(n * neigh_alloc, np.int32)
        numneigh = np.zeros(n, np.int32)
        mx = lib(fast).orc_neighbor_wrapper(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                                            np.ascontiguousarray(specbond, np.int32),
                                            np.ascontiguousarray(num3bond, np.int32), nlist,
                                            numneigh, neigh_alloc, nthreads)
        if mx <= neigh_alloc:
            return nlist, numneigh, neigh_alloc
        neigh_alloc = int(mx * 1.2)
        neigh_alloc += (-neigh_alloc) % 16


def build_neighbor_sorted(p: OrcParams, pos_sorted, atombin, start, endposit, cnum, specbond_s,
                          num3bond_s, neigh_alloc: int, nthreads: int = 0, fast: bool = False):
    n = pos_sorted.shape[0]
    nlist = np.zeros(n * neigh_alloc, np.int32)
    numneigh = np.zeros(n, np.int32)
    mx = lib(fast).orc_build_neighbor_nonewton(C.byref(p), n, pos_sorted, atombin, start,
                                               endposit, cnum, specbond_s, num3bond_s, nlist,
                                               numneigh, neigh_alloc, nthreads)
    return nlist, numneigh, mx


def neighbor_n2(p: OrcParams, pos, specbond, num3bond, neigh_alloc: int):
    n = pos.shape[0]
    nlist = np.zeros(n * neigh_alloc, np.int32)
    numneigh = np.zeros(n, np.int32)
    mx = lib().orc_build_neighbor_n2(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                                     np.ascontiguousarray(specbond, np.int32),
                                     np.ascontiguousarray(num3bond, np.int32), nlist, numneigh,
                                     neigh_alloc)
    assert mx <= neigh_alloc
    return nlist, numneigh


def force_dsf(p: OrcParams, pos, q, lj, ntypes, nlist, numneigh, neigh_alloc, nthreads=0,
              fast: bool = False):
    """lj_cut_coul_dsf_nonewton: returns ff (float32), ff64, potential, e_coul, virial3."""
    n = pos.shape[0]
    ff = np.zeros(n * 3, np.float32)
    ff64 = np.zeros(n * 3, np.float64)
    pot = C.c_double()
    ec = C.c_double()
    vir = np.zeros(3, np.float64)
    lib(fast).orc_force_dsf_nonewton(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                                     np.ascontiguousarray(q, np.float32), lj[0], lj[1], lj[2],
                                     lj[3], ntypes, nlist, numneigh, neigh_alloc, ff,
                                     C.byref(pot), C.byref(ec), vir,
                                     ff64.ctypes.data_as(C.c_void_p), nthreads)
    return ff.reshape(n, 3), ff64.reshape(n, 3), pot.value, ec.value, vir


def force_long(p: OrcParams, pos, q, lj, ntypes, nlist, numneigh, neigh_alloc, gewald: float,
               nthreads=0, fast: bool = False):
    """lj_cut_coul_long_nonewton (real-space Ewald): ff (float32), ff64, potential,
    e_coul, virial3."""
    n = pos.shape[0]
    ff = np.zeros(n * 3, np.float32)
    ff64 = np.zeros(n * 3, np.float64)
    pot = C.c_double()
    ec = C.c_double()
    vir = np.zeros(3, np.float64)
    lib(fast).orc_force_long_nonewton(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                                      np.ascontiguousarray(q, np.float32), lj[0], lj[1], lj[2],
                                      lj[3], ntypes, nlist, numneigh, neigh_alloc, float(gewald),
                                      ff, C.byref(pot), C.byref(ec), vir,
                                      ff64.ctypes.data_as(C.c_void_p), nthreads)
    return ff.reshape(n, 3), ff64.reshape(n, 3), pot.value, ec.value, vir


def improper_harmonic(p: OrcParams, pos, improlist, improcoeff):
    """improper_harmonic_lammps14: ff_impro (float32, rounded per improper), e, virial3."""
    n = pos.shape[0]
    ff = np.zeros(n * 3, np.float32)
    e = C.c_double(0.0)
    vir = np.zeros(3, np.float64)
    il = np.ascontiguousarray(improlist, np.int32)
    lib().orc_improper_harmonic(C.byref(p), n, np.ascontiguousarray(pos, np.float32), il.shape[0],
                                il, np.ascontiguousarray(improcoeff, np.float64), ff, C.byref(e),
                                vir)
    return ff.reshape(n, 3), e.value, vir


def force_dsf_n2(p: OrcParams, pos, q, lj, ntypes, specbond, n1, n2, n3):
    n = pos.shape[0]
    ff64 = np.zeros(n * 3, np.float64)
    pot = C.c_double()
    ec = C.c_double()
    lib().orc_force_dsf_n2(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                           np.ascontiguousarray(q, np.float32), lj[0], lj[1], lj[2], lj[3],
                           ntypes, np.ascontiguousarray(specbond, np.int32),
                           np.ascontiguousarray(n1, np.int32), np.ascontiguousarray(n2, np.int32),
                           np.ascontiguousarray(n3, np.int32), ff64, C.byref(pot), C.byref(ec))
    return ff64.reshape(n, 3), pot.value, ec.value


def dihedral_opls_dsf(p: OrcParams, pos, q, ntypes, lj14, dihedlist, dihedcoeff,
                      want_f64: bool = False):
    """Returns (ffh real*4 (n,3), e_dihedral, e_coul_14, pot_14), plus the same forces
    summed in double as a fifth item when ``want_f64``."""
    n = pos.shape[0]
    ffh = np.zeros(n * 3, np.float32)
    f64 = np.zeros(n * 3) if want_f64 else None
    ed = C.c_double(0.0)
    ec = C.c_double(0.0)
    p14 = C.c_double(0.0)
    lib().orc_dihedral_opls_dsf(C.byref(p), n, np.ascontiguousarray(pos, np.float32),
                                np.ascontiguousarray(q, np.float32), ntypes,
                                np.ascontiguousarray(lj14, np.float64), dihedlist.shape[0],
                                np.ascontiguousarray(dihedlist, np.int32),
                                np.ascontiguousarray(dihedcoeff, np.float64), ffh, C.byref(ed),
                                C.byref(ec), C.byref(p14),
                                None if f64 is None else f64.ctypes.data_as(C.c_void_p))
    if want_f64:
        return ffh.reshape(n, 3), ed.value, ec.value, p14.value, f64.reshape(n, 3)
    return ffh.reshape(n, 3), ed.value, ec.value, p14.value


def correct_pairs(p: OrcParams, pos, q, lst: np.ndarray, col_a: int, col_b: int, gewald: float,
                  fudge: float):
    """correct_12/13/14_bonds over rows of ``lst`` (columns col_a, col_b, 1-based ids)."""
    n = pos.shape[0]
    lst = np.ascontiguousarray(lst, np.int32)
    stride = lst.shape[1]
    ffc = np.zeros(n * 3, np.float32)
    e = C.c_double(0.0)
    vir = np.zeros(3, np.float64)
    base = lst.ctypes.data
    lib().orc_correct_pairs(C.byref(p), np.ascontiguousarray(pos, np.float32),
                            np.ascontiguousarray(q, np.float32), lst.shape[0],
                            C.c_void_p(base + 4 * col_a), C.c_void_p(base + 4 * col_b), stride,
                            float(gewald), float(fudge), ffc, C.byref(e), vir)
    return ffc.reshape(n, 3), e.value, vir


def calculate_gewald(cut_coul: float) -> float:
    return lib().orc_calculate_gewald(np.float32(cut_coul))


def e_self(p: OrcParams, q) -> float:
    return lib().orc_e_self_dsf(C.byref(p), len(q), np.ascontiguousarray(q, np.float32))


def greatest_cluster(pos, global_id, n_gly, apg, box, ibox, vol, mrcut, denscut, densmin,
                     ptta, greatest_in: int = 0):
    """get_greatestCluster: returns (size, greatest_belongsto, denstrack, belongsto).
    ``ptta`` (n_gly*apg,3) float64 is updated in place like the module array."""
    n = pos.shape[0]
    g = C.c_int32(greatest_in)
    dens = np.zeros(max(n_gly, 1), np.int32)
    bel = np.zeros(max(n_gly, 1), np.int32)
    size = lib().orc_greatest_cluster(n, np.ascontiguousarray(pos, np.float32),
                                      np.ascontiguousarray(global_id, np.int32), n_gly, apg,
                                      np.float32(box), np.float32(ibox), np.float32(vol),
                                      float(mrcut), float(denscut), int(densmin), ptta,
                                      C.byref(g), dens.ctypes.data_as(C.c_void_p),
                                      bel.ctypes.data_as(C.c_void_p))
    return size, g.value, dens[:n_gly], bel[:n_gly]


def bond_harmonic(p, pos, bonds, coeff):
    n = pos.shape[0]
    f = np.zeros(n * 3)
    e = C.c_double(0.0)
    lib().orc_bond_harmonic(C.byref(p), np.ascontiguousarray(pos, np.float32), bonds.shape[0],
                            np.ascontiguousarray(bonds, np.int32),
                            np.ascontiguousarray(coeff, np.float64), f, C.byref(e))
    return f.reshape(n, 3), e.value


def angle_harmonic(p, pos, angles, coeff):
    n = pos.shape[0]
    f = np.zeros(n * 3)
    e = C.c_double(0.0)
    lib().orc_angle_harmonic(C.byref(p), np.ascontiguousarray(pos, np.float32), angles.shape[0],
                             np.ascontiguousarray(angles, np.int32),
                             np.ascontiguousarray(coeff, np.float64), f, C.byref(e))
    return f.reshape(n, 3), e.value


def shake(x, v, f, mass_atom, box, shakeatom, shake_bond, dt, kcal2amu, iflag=1, maxiter=25,
          tolerance=float(np.float32(0.0001))):
    """Force-form SHAKE on FP64 state; returns (f_new, status)."""
    n = x.shape[0]
    fo = np.ascontiguousarray(f, np.float64).copy().reshape(-1)
    st = lib().orc_shake(n, np.ascontiguousarray(x, np.float64).reshape(-1),
                         np.ascontiguousarray(v, np.float64).reshape(-1), fo,
                         np.ascontiguousarray(mass_atom, np.float64), float(box),
                         shakeatom.shape[0], np.ascontiguousarray(shakeatom, np.int32),
                         np.ascontiguousarray(shake_bond, np.float64), float(dt),
                         float(kcal2amu), iflag, maxiter, tolerance)
    return fo.reshape(n, 3), st
