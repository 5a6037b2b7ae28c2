"""Loads ``libsofia_nb.so`` and declares its C ABI (``include/sofia_nb.h``).

There is no CPU fallback: if the shared library is missing or cannot be
loaded, ``lib()`` raises, and every entry point of this package fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsofia_nb.so")

SOFIA_OK = 0
SOFIA_ENEEDGROW = 1
SOFIA_EINVAL = 2
SOFIA_ECUDA = 3
SOFIA_ETIMEOUT = 4
SOFIA_ESTATE = 5
SOFIA_ETOOBIG = 6
SOFIA_NOALLOC_MAX_ATOMS = 65536


class SofiaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sofia error {code}: {msg}")
        self.code = code


class SofiaNbParams(C.Structure):
    _fields_ = [("device", C.c_int), ("flags", C.c_int)]


SOFIA_PREC_MIXED = 0
SOFIA_PREC_FP64 = 1


class SofiaMdDesc(C.Structure):
    _fields_ = [("dt", C.c_double), ("temperature", C.c_double), ("gamma", C.c_double),
                ("seed", C.c_uint64), ("terms", C.c_int), ("nbond", C.c_int),
                ("bonds", C.c_void_p), ("nbondtypes", C.c_int), ("bond_coeff", C.c_void_p),
                ("nangle", C.c_int), ("angles", C.c_void_p), ("nangletypes", C.c_int),
                ("angle_coeff", C.c_void_p), ("ndihed", C.c_int), ("dihedrals", C.c_void_p),
                ("ndihedtypes", C.c_int), ("dihed_coeff", C.c_void_p), ("lj14", C.c_void_p),
                ("nshake", C.c_int), ("shake", C.c_void_p), ("shake_bond", C.c_void_p),
                ("shake_maxiter", C.c_int), ("shake_tol", C.c_double),
                ("nimpro", C.c_int), ("impropers", C.c_void_p), ("nimprotypes", C.c_int),
                ("impro_coeff", C.c_void_p), ("flags", C.c_int)]


# sofia_md_desc.flags and the force terms of sofia_system_md_forces
SOFIA_MD_RATTLE = 1
SOFIA_MD_LJ_SHIFT = 2
SOFIA_TERM_BOND = 1
SOFIA_TERM_ANGLE = 2
SOFIA_TERM_TORSION = 4
SOFIA_TERM_PAIR14 = 8
SOFIA_TERM_IMPROPER = 16
SOFIA_TERM_NONBOND = 32
SOFIA_TERM_SHAKE = 64
SOFIA_TERM_LANGEVIN = 128


SOFIA_MD_NE = 13
MD_ENERGY_NAMES = ["lj", "coul", "self", "bond", "angle", "torsion", "coul14", "lj14", "kinetic",
                   "total", "temperature", "step", "improper"]


class SofiaSystemDesc(C.Structure):
    _fields_ = [("np", C.c_int), ("ntypes", C.c_int), ("box", C.c_float), ("alpha", C.c_double),
                ("cut_coul", C.c_float), ("rcut", C.c_float), ("neighbor_pad", C.c_float),
                ("precision", C.c_int), ("type", C.c_void_p), ("q", C.c_void_p),
                ("lj1", C.c_void_p), ("lj2", C.c_void_p), ("lj3", C.c_void_p),
                ("lj4", C.c_void_p), ("specbond", C.c_void_p), ("num3bond", C.c_void_p),
                ("mass", C.c_void_p)]


_P = C.c_void_p
_I = C.c_int
_F = C.c_float
_D = C.c_double

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "sofia_nb_create": (_I, [C.POINTER(SofiaNbParams), C.POINTER(_P)]),
    "sofia_nb_destroy": (_I, [_P]),
    "sofia_last_error": (C.c_char_p, [_P]),
    "sofia_wait": (_I, [_P]),
    "sofia_stream": (_P, [_P]),
    "sofia_dsf_constants": (_I, [_D, _F, C.POINTER(_D), C.POINTER(_D)]),
    "sofia_cell_grid": (_I, [_F, _F, _F, C.POINTER(_F), C.POINTER(C.c_int32),
                             C.POINTER(C.c_int32)]),
    "sofia_cell_sort": (_I, [_P, _I, _P, _F, _F, _F, _P, _P, _P, _P, _P, _P]),
    "sofia_neighbor_build": (_I, [_P, _I, _P, _P, _P, _F, _D, _F, _F, _P, _P, C.c_int32,
                                  C.POINTER(C.c_int32)]),
    "sofia_force_nonbond_dsf": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P, C.c_int32, _F,
                                     _F, _D, _D, _D, _D, _D, _F, _P, C.POINTER(_D),
                                     C.POINTER(_D), _P]),
    "sofia_force_nonbond_long": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P, C.c_int32,
                                      _F, _F, _D, _D, _D, _F, _P, C.POINTER(_D), C.POINTER(_D),
                                      _P]),
    "sofia_check_neighbor": (_I, [_P, _I, _P, _P, _P, _D, C.POINTER(C.c_int32)]),
    "sofia_sort_gather": (_I, [_P, _I, _I, _P, _P, _P]),
    "sofia_sort_specbond": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "sofia_remap_ids": (_I, [_P, _I, _P, _I, _I, _I, _P]),
    "sofia_pbc": (_I, [_P, _I, _P, _F]),
    "sofia_improper_harmonic": (_I, [_P, _I, _P, _I, _P, _P, _I, _F, _F, _P, C.POINTER(_D),
                                     _P]),
    "sofia_force_nonbond_dsf_noalloc": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P,
                                             C.c_int32, _F, _F, _D, _D, _D, _D, _D, _F, _P,
                                             C.POINTER(_D), C.POINTER(_D), _P]),
    "sofia_pair14_dsf": (_I, [_P, _I, _P, _P, _I, _P, _I, _P, _P, _I, _F, _F, _D, _D, _D, _D, _D, _F,
                              _P, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "sofia_correct_1x": (_I, [_P, _I, _P, _P, _I, _P, _I, _I, _I, _F, _F, _D, _D, _D, _F, _P,
                              C.POINTER(_D), _P]),
    "sofia_greatest_cluster": (_I, [_P, _I, _P, _P, _I, _I, _F, _D, _D, _I, _P,
                                    C.POINTER(C.c_int32), C.POINTER(C.c_int32), _P, _P]),
    "sofia_system_create": (_I, [_P, C.POINTER(SofiaSystemDesc), C.POINTER(_P)]),
    "sofia_system_destroy": (_I, [_P]),
    "sofia_force_nonbond_mixed": (_I, [_P, _P, _P, C.POINTER(_D), C.POINTER(_D), _P]),
    "sofia_system_set_state": (_I, [_P, _P, _P]),
    "sofia_system_get_state": (_I, [_P, _P, _P, _P]),
    "sofia_system_compute_forces": (_I, [_P, _I, _I, _P]),
    "sofia_system_stats": (_I, [_P, _P, _I]),
    "sofia_system_drift": (_I, [_P, _D, _I]),
    "sofia_system_md_setup": (_I, [_P, C.POINTER(SofiaMdDesc)]),
    "sofia_system_md_run": (_I, [_P, _I, _I, _I, _P]),
    "sofia_system_md_forces": (_I, [_P, _I, _P, _P]),
    "sofia_system_list_pairs": (_I, [_P, _I, C.c_int64, _P, C.POINTER(C.c_int64), _P]),
    "sofia_batch_create": (_I, [_P, _P, _I, C.POINTER(_P)]),
    "sofia_batch_destroy": (_I, [_P]),
    "sofia_batch_md_run": (_I, [_P, _I, _I, _P]),
    "sofia_batch_set_systems": (_I, [_P, _P, _I]),
    "sofia_batch_set_segment": (_I, [_P, _I]),
    "sofia_system_set_margin": (_I, [_P, _D]),
    "sofia_system_set_cluster_shape": (_I, [_P, _D]),
    "sofia_system_timers": (_I, [_P, _I, _P]),
    "sofia_system_snapshot": (_I, [_P]),
    "sofia_system_rollback": (_I, [_P]),
    "sofia_system_md_get_step": (_I, [_P, _P]),
    "sofia_system_md_set_step": (_I, [_P, C.c_longlong]),
    "sofia_system_greatest_cluster": (_I, [_P, _I, _I, _D, _D, _I, _P, C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32)]),
    "sofia_system_device_bytes": (_I, [_P, C.POINTER(C.c_int64)]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises if it is missing (no silent fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SofiaError(SOFIA_EINVAL, f"{LIB_PATH} is missing; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols() -> list[str]:
    return list(SIGNATURES)
