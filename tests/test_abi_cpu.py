"""CPU checks of the C ABI: the library loads and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    syms = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(sofia_[a-z0-9_]+)\s*\(", txt):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    from molecular_simulation_code_b200 import _lib
    L = _lib.lib()
    declared = _header_symbols()
    assert declared, "no declarations found"
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    # the Python binding declares exactly the header's functions
    assert set(_lib.declared_symbols()) <= declared


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from molecular_simulation_code_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    p = _lib.SofiaNbParams(0, 0)
    rc = L.sofia_nb_create(C.byref(p), C.byref(h))
    assert rc == _lib.SOFIA_ECUDA and not h.value


def test_host_helpers_without_gpu():
    import numpy as np
    from molecular_simulation_code_b200 import nonbond as nb
    from oracle import oracle as O
    for box, cut, rcut in [(45.385056, 10.0, 10.0), (21.7, 7.0, 7.0), (141.4, 10.0, 10.0),
                           (77.61, 12.0, 12.0)]:
        p = O.params(0.2, box, cut, rcut, 2.0)
        assert nb.cell_grid(box, cut, rcut) == pytest.approx(O.cell_grid(p))
        dp = nb.DsfParams(alpha=0.2, box=box, cut_coul=cut, rcut=rcut, neighbor_pad=2.0)
        assert dp.e_shift == p.e_shift and dp.f_shift == p.f_shift
        assert dp.rv2 == p.rv2 and dp.rcut2 == p.rcut2 and dp.cut_coulsq == p.cut_coulsq
        assert np.float32(dp.ibox) == np.float32(p.ibox)


def test_null_context_is_rejected():
    from molecular_simulation_code_b200 import _lib
    L = _lib.lib()
    assert L.sofia_wait(None) == _lib.SOFIA_EINVAL
    assert L.sofia_nb_destroy(None) == _lib.SOFIA_OK
