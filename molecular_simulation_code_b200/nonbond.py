"""Host-side mirror of the reference's nonbonded subroutines over the C ABI.

Names and argument meaning follow the Fortran routines they replace:

=============================  ===============================================
``neighbor_wrapper``           Source/mod_neighbor.f90:8-86 (+ redo loop :767-802)
``cell_sort``                  Source/mod_neighbor.f90:923-1005 (new_nlist + sort_posit_charge)
``lj_cut_coul_dsf_nonewton``   Source/mod_force_nonbond.f90:105-196
``dihedral_opls_dsf``          Source/mod_force_dihed.f90:816-1092
``correct_1x_bonds``           Source/mod_force_correction.f90:6-278
``get_greatest_cluster``       Source/mod_cluster.f90:15-83
=============================  ===============================================

Arrays may be numpy (host; copied in and out inside the call, like the
reference's offload transfers) or CUDA torch tensors (used in place).
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
import math
import dataclasses

import numpy as np

from ._lib import SOFIA_ENEEDGROW, SOFIA_OK, SofiaError, SofiaNbParams, lib

COULPRE = np.float32(332.06371)  # real*4 (Source/get_started.f90:34)


def ptr(a):
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


_LIVE = weakref.WeakSet()


def _close_all():
    """At interpreter exit, close every live context (its systems and batches first)
    while the CUDA runtime is still up, whatever the caller left open."""
    for c in list(_LIVE):
        try:
            c.close()
        except Exception:
            pass


atexit.register(_close_all)


class Context:
    """One ``sofia_nb_ctx`` (CUDA stream + device buffers) on one GPU."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        p = SofiaNbParams(device, 0)
        rc = self._lib.sofia_nb_create(C.byref(p), C.byref(h))
        if rc != SOFIA_OK:
            raise SofiaError(rc, "sofia_nb_create failed (no usable CUDA device?)")
        self.handle = h
        # systems and batches created on this context hold its stream: they are
        # destroyed before it, whatever order the garbage collector picks
        self._children = weakref.WeakSet()
        _LIVE.add(self)

    def adopt(self, obj):
        """Register an object whose ``close()`` must run before this context's."""
        self._children.add(obj)

    def check(self, rc: int):
        if rc != SOFIA_OK:
            raise SofiaError(rc, self.last_error())
        return rc

    def last_error(self) -> str:
        m = self._lib.sofia_last_error(self.handle)
        return m.decode() if m else ""

    def wait(self):
        self.check(self._lib.sofia_wait(self.handle))

    def close(self):
        if self.handle:
            # batches hold their systems: close them first
            kids = list(getattr(self, "_children", ()))
            for obj in sorted(kids, key=lambda o: getattr(o, "close_rank", 1)):
                obj.close()
            self._lib.sofia_nb_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


@dataclasses.dataclass
class DsfParams:
    """Cut-offs and DSF constants exactly as ``init`` builds them
    (Source/get_started.f90:45-117; real*4 where the reference stores real*4)."""

    alpha: float
    box: np.float32
    cut_coul: np.float32
    rcut: np.float32
    neighbor_pad: np.float32

    def __post_init__(self):
        self.box = np.float32(self.box)
        self.cut_coul = np.float32(self.cut_coul)
        self.rcut = np.float32(self.rcut)
        self.neighbor_pad = np.float32(self.neighbor_pad)
        self.ibox = np.float32(1.0 / np.float64(self.box))
        self.rcut2 = float(np.float32(self.rcut * self.rcut))
        self.cut_coulsq = float(np.float32(self.cut_coul * self.cut_coul))
        rv = float(np.float32(self.neighbor_pad + self.cut_coul))
        self.rv2 = rv * rv
        self.rvrc2 = float(self.neighbor_pad) ** 2
        es = C.c_double()
        fs = C.c_double()
        rc = lib().sofia_dsf_constants(float(self.alpha), self.cut_coul, C.byref(es), C.byref(fs))
        if rc != SOFIA_OK:
            raise SofiaError(rc, "sofia_dsf_constants")
        self.e_shift = es.value
        self.f_shift = fs.value
        self.coulpre = COULPRE


def cell_grid(box, cut_coul, rcut):
    rn = C.c_float()
    nt = C.c_int32()
    nd = C.c_int32()
    rc = lib().sofia_cell_grid(np.float32(box), np.float32(cut_coul), np.float32(rcut),
                               C.byref(rn), C.byref(nt), C.byref(nd))
    if rc != SOFIA_OK:
        raise SofiaError(rc, "sofia_cell_grid")
    return rn.value, nt.value, nd.value


def cell_sort(ctx: Context, position: np.ndarray, p: DsfParams):
    """Returns tt, ttb (1-based), start, endposit (1-based), atombin, position_sorted."""
    n = position.shape[0]
    _, nt, _ = cell_grid(p.box, p.cut_coul, p.rcut)
    tt = np.zeros(n, np.int32)
    ttb = np.zeros(n, np.int32)
    st = np.zeros(nt, np.int32)
    en = np.zeros(nt, np.int32)
    ab = np.zeros(n, np.int32)
    ps = np.zeros((n, 4), np.float32)
    ctx.check(ctx._lib.sofia_cell_sort(ctx.handle, n, ptr(position), p.box, p.cut_coul, p.rcut,
                                       ptr(tt), ptr(ttb), ptr(st), ptr(en), ptr(ab), ptr(ps)))
    return tt, ttb, st, en, ab, ps


def neighbor_wrapper(ctx: Context, position, specbond, num3bond, p: DsfParams,
                     neigh_alloc: int = 512, want_host: bool = True):
    """Builds the reference full list; grows ``neigh_alloc`` like the redo loop.

    Returns (nlist, numneigh, neigh_alloc); with ``want_host=False`` the list stays
    resident in the context (nlist/numneigh returned as None)."""
    n = int(position.shape[0])
    while True:
        if want_host:
            nlist = np.zeros(n * neigh_alloc, np.int32)
            numneigh = np.zeros(n, np.int32)
        else:
            nlist = numneigh = None
        need = C.c_int32()
        rc = ctx._lib.sofia_neighbor_build(ctx.handle, n, ptr(position), ptr(specbond),
                                           ptr(num3bond), p.box, p.rv2, p.cut_coul, p.rcut,
                                           ptr(nlist), ptr(numneigh), neigh_alloc,
                                           C.byref(need))
        if rc == SOFIA_ENEEDGROW:
            neigh_alloc = int(need.value)
            continue
        ctx.check(rc)
        return nlist, numneigh, neigh_alloc


def sort_posit(ctx: Context, ttb, arr):
    """sort_posit_charge (Source/mod_neighbor.f90:946-1005) for one per-atom array:
    returns arr[ttb - 1] (rows of any 4-byte-multiple size)."""
    a = np.ascontiguousarray(arr)
    out = np.empty_like(a)
    n = a.shape[0]
    ctx.check(ctx._lib.sofia_sort_gather(ctx.handle, n, a.nbytes // n, ptr(np.ascontiguousarray(
        ttb, np.int32)), ptr(a), ptr(out)))
    return out


def sort_specbond_numbond(ctx: Context, tt, specbond, num1bond, num2bond, num3bond):
    """sort_specbond_numbond (Source/mod_neighbor.f90:1011-1039): sorted copies."""
    sb = np.array(specbond, np.int32, order="C")
    n1 = np.array(num1bond, np.int32)
    n2 = np.array(num2bond, np.int32)
    n3 = np.array(num3bond, np.int32)
    ctx.check(ctx._lib.sofia_sort_specbond(ctx.handle, sb.shape[0], ptr(np.ascontiguousarray(
        tt, np.int32)), ptr(sb), ptr(n1), ptr(n2), ptr(n3)))
    return sb, n1, n2, n3


def sort_list(ctx: Context, tt, lst, ncols: int):
    """sort_bondlist / sort_anglelist / ... (Source/mod_neighbor.f90:1043-1168): the
    first ncols columns of each row mapped through tt (a sorted copy)."""
    a = np.array(lst, np.int32, order="C")
    n = int(np.asarray(tt).shape[0])
    ctx.check(ctx._lib.sofia_remap_ids(ctx.handle, n, ptr(np.ascontiguousarray(tt, np.int32)),
                                       a.shape[0], a.shape[1], int(ncols), ptr(a)))
    return a


def pbc(ctx: Context, position, box):
    """pbc (Source/mod_pbc.f90:6-39): a wrapped copy of the (np,4) ainfo records."""
    p = np.array(position, np.float32, order="C")
    ctx.check(ctx._lib.sofia_pbc(ctx.handle, p.shape[0], ptr(p), np.float32(box)))
    return p


def check_neighbor(ctx: Context, drx, dry, drz, rvrc2: float) -> int:
    """check_neighbor (Source/mod_neighbor.f90:895-913): 1 if a rebuild is due."""
    flag = C.c_int32()
    ctx.check(ctx._lib.sofia_check_neighbor(ctx.handle, int(len(drx)), ptr(drx), ptr(dry),
                                            ptr(drz), float(rvrc2), C.byref(flag)))
    return flag.value


def lj_cut_coul_dsf_nonewton(ctx: Context, position, q, lj, ntypes: int, nlist, numneigh,
                             neigh_alloc: int, p: DsfParams, ff=None):
    """FP64 LJ + DSF over the full list.  ``nlist=None`` uses the resident list.
    Returns (ff (np,3) float32, potential, e_coul, virial_diag3)."""
    n = int(position.shape[0])
    if ff is None:
        ff = np.zeros((n, 3), np.float32)
    pot = C.c_double()
    ec = C.c_double()
    vir = np.zeros(3, np.float64)
    ctx.check(ctx._lib.sofia_force_nonbond_dsf(
        ctx.handle, n, ptr(position), ptr(q), ptr(lj[0]), ptr(lj[1]), ptr(lj[2]), ptr(lj[3]),
        ntypes, ptr(nlist), ptr(numneigh), int(neigh_alloc), p.box, p.ibox, p.rcut2,
        p.cut_coulsq, float(p.alpha), p.e_shift, p.f_shift, p.coulpre, ptr(ff), C.byref(pot),
        C.byref(ec), ptr(vir)))
    return ff, pot.value, ec.value, vir


def calculate_gewald(cut_coul: float) -> float:
    """Ewald splitting parameter of calculate_gewald (Source/get_started.f90:153-173):
    100 bisection steps on [0, 1] for erfc(g*cut_coul)/cut_coul = 1e-6 (real*4 tolerance)."""
    cc = float(np.float32(cut_coul))
    tol = float(np.float32(0.000001))
    lo, hi, g = 0.0, 1.0, 1.0
    for _ in range(100):
        g = 0.5 * (lo + hi)
        if math.erfc(g * cc) / cc > tol:
            lo = g
        else:
            hi = g
    return g


def lj_cut_coul_long_nonewton(ctx: Context, position, q, lj, ntypes: int, nlist, numneigh,
                              neigh_alloc: int, p: DsfParams, gewald: float, ff=None):
    """Real-space Ewald + LJ over the full list (the PME path's pair term), real*4
    pair arithmetic.  Returns (ff (np,3) float32, potential, e_coul, virial_diag3)."""
    n = int(position.shape[0])
    if ff is None:
        ff = np.zeros((n, 3), np.float32)
    pot = C.c_double()
    ec = C.c_double()
    vir = np.zeros(3, np.float64)
    ctx.check(ctx._lib.sofia_force_nonbond_long(
        ctx.handle, n, ptr(position), ptr(q), ptr(lj[0]), ptr(lj[1]), ptr(lj[2]), ptr(lj[3]),
        ntypes, ptr(nlist), ptr(numneigh), int(neigh_alloc), p.box, p.ibox, p.rcut2,
        p.cut_coulsq, float(gewald), p.coulpre, ptr(ff), C.byref(pot), C.byref(ec), ptr(vir)))
    return ff, pot.value, ec.value, vir


def dihedral_opls_dsf(ctx: Context, position, q, ntypes: int, lj14, dihedlist, dihedcoeff,
                      p: DsfParams, ffh=None):
    """Torsion + 0.5-scaled 1-4 pair.  Returns (ffh, e_dihedral, e_coul_14, pot_14)."""
    n = int(position.shape[0])
    if ffh is None:
        ffh = np.zeros((n, 3), np.float32)
    ed = C.c_double(0.0)
    ec = C.c_double(0.0)
    p14 = C.c_double(0.0)
    dl = np.ascontiguousarray(dihedlist, np.int32)
    dc = np.ascontiguousarray(dihedcoeff, np.float64)
    l14 = np.ascontiguousarray(lj14, np.float64)
    ctx.check(ctx._lib.sofia_pair14_dsf(ctx.handle, n, ptr(position), ptr(q), ntypes, ptr(l14),
                                        int(dl.shape[0]), ptr(dl), ptr(dc), int(dc.shape[0]),
                                        p.box, p.ibox,
                                        p.rcut2, p.cut_coulsq, float(p.alpha), p.e_shift,
                                        p.f_shift, p.coulpre, ptr(ffh), C.byref(ed),
                                        C.byref(ec), C.byref(p14)))
    return ffh, ed.value, ec.value, p14.value


def improper_harmonic(ctx: Context, position, improlist, improcoeff, p: DsfParams,
                      ff_impro=None):
    """improper_harmonic_lammps14: returns (ff_impro (np,3) float32 with the forces
    added, e_improper, virial_diag3)."""
    n = int(position.shape[0])
    if ff_impro is None:
        ff_impro = np.zeros((n, 3), np.float32)
    il = np.ascontiguousarray(improlist, np.int32)
    ic = np.ascontiguousarray(improcoeff, np.float64)
    e = C.c_double(0.0)
    vir = np.zeros(3, np.float64)
    ctx.check(ctx._lib.sofia_improper_harmonic(ctx.handle, n, ptr(position), il.shape[0], ptr(il),
                                               ptr(ic), ic.shape[0], p.box, p.ibox, ptr(ff_impro),
                                               C.byref(e), ptr(vir)))
    return ff_impro, e.value, vir


def correct_1x_bonds(ctx: Context, position, q, lst, col_a: int, col_b: int, gewald: float,
                     fudge: float, p: DsfParams, ffc=None):
    """correct_12/13/14_bonds over rows of ``lst``.  Returns (ffc, e_corr, virial3)."""
    n = int(position.shape[0])
    if ffc is None:
        ffc = np.zeros((n, 3), np.float32)
    lst = np.ascontiguousarray(lst, np.int32)
    e = C.c_double(0.0)
    vir = np.zeros(3, np.float64)
    ctx.check(ctx._lib.sofia_correct_1x(ctx.handle, n, ptr(position), ptr(q), int(lst.shape[0]),
                                        ptr(lst), int(lst.shape[1]), col_a, col_b, p.box,
                                        p.ibox, p.cut_coulsq, float(gewald), float(fudge),
                                        p.coulpre, ptr(ffc), C.byref(e), ptr(vir)))
    return ffc, e.value, vir


def correct_12_bonds(ctx, position, q, bondlist, gewald, fudge_12, p, ffc=None):
    return correct_1x_bonds(ctx, position, q, bondlist, 0, 1, gewald, fudge_12, p, ffc)


def correct_13_bonds(ctx, position, q, anglelist, gewald, fudge_13, p, ffc=None):
    return correct_1x_bonds(ctx, position, q, anglelist, 0, 2, gewald, fudge_13, p, ffc)


def correct_14_bonds(ctx, position, q, dihedlist, gewald, fudge_14_coul, p, ffc=None):
    return correct_1x_bonds(ctx, position, q, dihedlist, 0, 3, gewald, fudge_14_coul, p, ffc)


def get_greatest_cluster(ctx: Context, position, global_id, n_gly: int, atoms_per_gly: int,
                         box, mrcut: float, denscut: float, densmin: int, ptta_full,
                         greatest: int = 0):
    """Returns (size, greatest_belongsto, denstrack, belongsto); ``ptta_full``
    (n_gly*atoms_per_gly, 3) float64 is updated in place like the module array."""
    n = int(position.shape[0])
    g = C.c_int32(int(greatest))
    size = C.c_int32()
    dens = np.zeros(max(n_gly, 1), np.int32)
    bel = np.zeros(max(n_gly, 1), np.int32)
    ctx.check(ctx._lib.sofia_greatest_cluster(ctx.handle, n, ptr(position), ptr(global_id),
                                              n_gly, atoms_per_gly, np.float32(box),
                                              float(mrcut), float(denscut), int(densmin),
                                              ptr(ptta_full), C.byref(g), C.byref(size),
                                              ptr(dens), ptr(bel)))
    return size.value, g.value, dens[:n_gly], bel[:n_gly]
