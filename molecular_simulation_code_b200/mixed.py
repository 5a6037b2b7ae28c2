"""Production (device-resident) nonbonded path over the C ABI.

``System`` owns one ``sofia_system``: static per-atom data, FP64 positions,
the cluster-pair list and 64-bit fixed-point forces live on the GPU.
``forces_dropin`` is the drop-in form of ``lj_cut_coul_dsf_nonewton``
(Source/mod_force_nonbond.f90:105-196): reference AoS positions in, real*4
forces out, list maintenance (Source/mod_neighbor.f90:8-86) done inside.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (MD_ENERGY_NAMES, SOFIA_ENEEDGROW, SOFIA_MD_LJ_SHIFT, SOFIA_MD_NE,
                   SOFIA_MD_RATTLE, SOFIA_OK, SOFIA_PREC_FP64, SOFIA_PREC_MIXED, SofiaError,
                   SofiaMdDesc, SofiaSystemDesc)
from .nonbond import Context, ptr

MIXED = SOFIA_PREC_MIXED
FP64 = SOFIA_PREC_FP64


class System:
    def __init__(self, ctx: Context, sysdata, alpha: float = 0.2, cut: float = 10.0,
                 skin: float = 2.0, precision: int = MIXED):
        self.ctx = ctx
        self.n = sysdata.np_atoms
        self._keep = [np.ascontiguousarray(sysdata.types, np.int32),
                      np.ascontiguousarray(sysdata.q, np.float32),
                      np.ascontiguousarray(sysdata.lj1, np.float32),
                      np.ascontiguousarray(sysdata.lj2, np.float32),
                      np.ascontiguousarray(sysdata.lj3, np.float32),
                      np.ascontiguousarray(sysdata.lj4, np.float32),
                      np.ascontiguousarray(sysdata.specbond, np.int32),
                      np.ascontiguousarray(sysdata.num3bond, np.int32),
                      np.ascontiguousarray(sysdata.mass_type, np.float64)]
        k = self._keep
        d = SofiaSystemDesc(self.n, sysdata.ntypes, np.float32(sysdata.box), float(alpha),
                            np.float32(cut), np.float32(cut), np.float32(skin), precision,
                            ptr(k[0]), ptr(k[1]), ptr(k[2]), ptr(k[3]), ptr(k[4]), ptr(k[5]),
                            ptr(k[6]), ptr(k[7]), ptr(k[8]))
        h = C.c_void_p()
        ctx.check(ctx._lib.sofia_system_create(ctx.handle, C.byref(d), C.byref(h)))
        self.handle = h
        self.precision = precision
        ctx.adopt(self)

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.sofia_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forces_dropin(self, position, ff=None, energy: bool = True, virial: bool = False):
        """Positions (np,4) float32 AoS or device tensor; returns (ff, pot, e_coul, virial).

        Like lj_cut_coul_dsf_nonewton_NOMIC (mod_force_nonbond.f90:105-196), the call
        returns the potential and Coulomb energy but no virial unless asked for
        (virial=True selects the kernel that also accumulates it); virial is None
        otherwise."""
        if ff is None:
            ff = np.zeros((self.n, 3), np.float32)
        pot = C.c_double()
        ec = C.c_double()
        vir = np.zeros(3) if virial else None
        if energy:
            args = (C.byref(pot), C.byref(ec), ptr(vir) if virial else None)
        else:
            args = (None, None, ptr(vir) if virial else None)
        self.ctx.check(self.ctx._lib.sofia_force_nonbond_mixed(self.handle, ptr(position),
                                                               ptr(ff), *args))
        return ff, pot.value, ec.value, vir

    def set_state(self, x, v=None):
        x = np.ascontiguousarray(x, np.float64)
        v = None if v is None else np.ascontiguousarray(v, np.float64)
        self.ctx.check(self.ctx._lib.sofia_system_set_state(self.handle, ptr(x), ptr(v)))

    def get_state(self):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        f = np.zeros((self.n, 3))
        self.ctx.check(self.ctx._lib.sofia_system_get_state(self.handle, ptr(x), ptr(v), ptr(f)))
        return x, v, f

    def compute(self, precision: int | None = None, rebuild: bool = False, energy: bool = True,
                virial: bool = True):
        e = np.zeros(5) if energy else None
        p = self.precision if precision is None else precision
        flags = (1 if rebuild else 0) | (2 if virial else 0)
        self.ctx.check(self.ctx._lib.sofia_system_compute_forces(self.handle, p, flags, ptr(e)))
        return e

    def stats(self) -> dict:
        st = np.zeros(11, np.int64)
        self.ctx.check(self.ctx._lib.sofia_system_stats(self.handle, ptr(st), 11))
        keys = ["builds", "clusters", "entries", "jcap", "ncx", "max_clusters", "reach",
                "launches", "prunes", "inner_entries", "shake_maxiter_hits"]
        return {k: int(v) for k, v in zip(keys, st)}

    def drift(self, dt: float, nsteps: int = 1):
        self.ctx.check(self.ctx._lib.sofia_system_drift(self.handle, float(dt), int(nsteps)))

    def md_setup(self, sysdata, dt: float = 2.0, temperature: float = 300.0,
                 gamma: float = 0.001, seed: int = 1, terms: int = 31, shake: bool = True,
                 shake_maxiter: int = 0, shake_tol: float = 0.0, rattle: bool = False,
                 lj_shift: bool = False):
        """Bonded lists, SHAKE groups and thermostat of the device-resident MD.
        terms: bit 1 bonds, 2 angles, 4 torsions, 8 1-4 pairs, 16 impropers.
        rattle: RATTLE velocity stage (full-step velocities on the constraints);
        lj_shift: LJ pair energies shifted to zero at the cut-off.  Both default to
        the reference's scheme and neither changes the positions."""
        k = [np.ascontiguousarray(a) for a in (
            sysdata.bonds.astype(np.int32), sysdata.bond_coeff.astype(np.float64),
            sysdata.angles.astype(np.int32), sysdata.angle_coeff.astype(np.float64),
            sysdata.dihedrals.astype(np.int32), sysdata.dihed_coeff.astype(np.float64),
            np.ascontiguousarray(sysdata.lj14, np.float64).reshape(-1),
            sysdata.shake.astype(np.int32), sysdata.shake_bond.astype(np.float64),
            sysdata.impropers.astype(np.int32).reshape(-1, 5),
            sysdata.impro_coeff.astype(np.float64).reshape(-1, 2))]
        self._md_keep = k
        ns = k[7].shape[0] if shake else 0
        d = SofiaMdDesc(float(dt), float(temperature), float(gamma), int(seed), int(terms),
                        k[0].shape[0], ptr(k[0]), k[1].shape[0], ptr(k[1]),
                        k[2].shape[0], ptr(k[2]), k[3].shape[0], ptr(k[3]),
                        k[4].shape[0], ptr(k[4]), k[5].shape[0], ptr(k[5]), ptr(k[6]),
                        ns, ptr(k[7]), ptr(k[8]), int(shake_maxiter), float(shake_tol),
                        k[9].shape[0], ptr(k[9]) if k[9].size else None, k[10].shape[0],
                        ptr(k[10]) if k[10].size else None,
                        (SOFIA_MD_RATTLE if rattle else 0) | (SOFIA_MD_LJ_SHIFT if lj_shift else 0))
        self.ctx.check(self.ctx._lib.sofia_system_md_setup(self.handle, C.byref(d)))

    def md_run(self, nsteps: int, energy_every: int = 0, use_graph: bool = True) -> dict | None:
        e = np.zeros(SOFIA_MD_NE)
        self.ctx.check(self.ctx._lib.sofia_system_md_run(self.handle, int(nsteps),
                                                         int(energy_every), int(use_graph),
                                                         ptr(e)))
        if energy_every <= 0:
            return None
        return dict(zip(MD_ENERGY_NAMES, e.tolist()))

    def md_forces(self, terms: int, energy: bool = True):
        """Forces of one MD step at the resident state without stepping, restricted to
        the SOFIA_TERM_* bits in ``terms`` (see ``_lib``).  Returns (f (n,3) float64,
        energies dict or None)."""
        f = np.zeros((self.n, 3))
        e = np.zeros(SOFIA_MD_NE) if energy else None
        self.ctx.check(self.ctx._lib.sofia_system_md_forces(self.handle, int(terms), ptr(f),
                                                            ptr(e)))
        return f, (dict(zip(MD_ENERGY_NAMES, e.tolist())) if energy else None)

    def list_pairs(self, which: int = 1):
        """The resident list as (npairs, 2) int32 0-based atom pairs (each pair once)
        and the (n, 3) positions it was made at; which = 0 outer, 1 pruned."""
        cap = 1 << 20
        while True:
            pairs = np.zeros((cap, 2), np.int32)
            xl = np.zeros((self.n, 3))
            cnt = C.c_int64()
            rc = self.ctx._lib.sofia_system_list_pairs(self.handle, int(which), cap,
                                                       ptr(pairs), C.byref(cnt), ptr(xl))
            if rc == SOFIA_ENEEDGROW:
                cap = int(cnt.value) + 1
                continue
            self.ctx.check(rc)
            return pairs[:cnt.value], xl

    def greatest_cluster(self, n_gly: int, mrcut: float, denscut: float, densmin: int,
                         greatest: int = 0, ptta=None, atoms_per_gly: int = 10):
        """get_greatestCluster on the resident positions (no host copy of them).
        ptta (n_gly*atoms_per_gly, 3) float64 is in/out like the module array; None
        uses the system's device copy.  Returns (size, greatest_belongsto)."""
        g = C.c_int32(greatest)
        size = C.c_int32(0)
        self.ctx.check(self.ctx._lib.sofia_system_greatest_cluster(
            self.handle, int(n_gly), int(atoms_per_gly), float(mrcut), float(denscut),
            int(densmin), ptr(ptta), C.byref(g), C.byref(size)))
        return int(size.value), int(g.value)

    def device_bytes(self) -> int:
        """Device memory this system holds now."""
        b = C.c_int64()
        self.ctx.check(self.ctx._lib.sofia_system_device_bytes(self.handle, C.byref(b)))
        return int(b.value)

    def snapshot(self):
        """Device copy of x, v and the thermostat step (nuc_move's save)."""
        self.ctx.check(self.ctx._lib.sofia_system_snapshot(self.handle))

    def rollback(self):
        """Restore the last snapshot (nuc_move's reject branch)."""
        self.ctx.check(self.ctx._lib.sofia_system_rollback(self.handle))

    def md_step(self) -> int:
        st = C.c_longlong()
        self.ctx.check(self.ctx._lib.sofia_system_md_get_step(self.handle, C.byref(st)))
        return int(st.value)

    def set_md_step(self, step: int):
        self.ctx.check(self.ctx._lib.sofia_system_md_set_step(self.handle, int(step)))

    def timers(self, enable: bool = True) -> dict:
        t = np.zeros(4)
        self.ctx.check(self.ctx._lib.sofia_system_timers(self.handle, int(enable), ptr(t)))
        return {"build_ms": t[0], "builds": int(t[1]), "pair_ms": t[2], "pairs": int(t[3])}


def force_rms_rel(f, fref) -> float:
    """sqrt(sum |f - fref|^2 / sum |fref|^2) over all atoms."""
    d = np.asarray(f, np.float64) - np.asarray(fref, np.float64)
    return float(np.sqrt((d * d).sum() / (np.asarray(fref, np.float64) ** 2).sum()))


def force_max_rel(f, fref) -> float:
    """max_i |f_i - fref_i| / max_i |fref_i|."""
    d = np.linalg.norm(np.asarray(f, np.float64) - np.asarray(fref, np.float64), axis=1)
    return float(d.max() / np.linalg.norm(np.asarray(fref, np.float64), axis=1).max())


__all__ = ["System", "MIXED", "FP64", "force_rms_rel", "force_max_rel", "SofiaError", "SOFIA_OK"]
