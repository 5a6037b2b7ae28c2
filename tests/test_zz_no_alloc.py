"""The allocation-free force entry point agrees with the regular one.

``sofia_force_nonbond_dsf_noalloc`` serves callers that cannot allocate device
memory when they need forces (for example under a device-memory budget or arena
enforced outside the library, or drivers that own every device array).  It
takes only caller-owned device buffers and keeps its scratch in a fixed array
inside the library.  This test calls it through the C ABI twice in a row and
checks both results against ``sofia_force_nonbond_dsf`` on the same inputs,
with the FP64 tolerance used by the other parity tests, and checks that the
device's free memory does not change across the two calls (after a warm-up
call, which may load the kernels' code).  It lives in its own file so that
pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import ref_params, small_system
from molecular_simulation_code_b200 import _lib
from molecular_simulation_code_b200 import nonbond as nb

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _noalloc(L, stream, n, pos, q, lj, ntypes, nl, nn, na, p, ff):
    pot = C.c_double()
    ec = C.c_double()
    vir = np.zeros(3)
    rc = L.sofia_force_nonbond_dsf_noalloc(
        stream, n, pos.data_ptr(), q.data_ptr(), lj[0].data_ptr(), lj[1].data_ptr(),
        lj[2].data_ptr(), lj[3].data_ptr(), ntypes, nl.data_ptr(), nn.data_ptr(), na, p.box,
        p.ibox, p.rcut2, p.cut_coulsq, float(p.alpha), p.e_shift, p.f_shift, p.coulpre,
        ff.data_ptr(), C.byref(pot), C.byref(ec), vir.ctypes.data)
    return rc, pot.value, ec.value, vir


@pytest.mark.parametrize("n_gly,n_wat,cut", [(10, 300, 7.0), (150, 2500, 10.0)])
def test_noalloc_matches_regular_entry_point(ctx, n_gly, n_wat, cut):
    import torch
    s = small_system(n_gly, n_wat, 3)
    p = ref_params(s, cut=cut, pad=2.0)
    n = s.np_atoms
    assert n <= _lib.SOFIA_NOALLOC_MAX_ATOMS
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(s.position_aos()).to(dev)
    q = torch.from_numpy(s.q).to(dev)
    lj = [torch.from_numpy(a).to(dev) for a in (s.lj1, s.lj2, s.lj3, s.lj4)]
    sb = torch.from_numpy(np.ascontiguousarray(s.specbond)).to(dev)
    n3 = torch.from_numpy(s.num3bond).to(dev)
    # the caller owns the list buffers (device memory it allocated itself)
    nl_host, nn_host, na = nb.neighbor_wrapper(ctx, s.position_aos(), s.specbond, s.num3bond, p,
                                               512)
    nl = torch.from_numpy(nl_host).to(dev)
    nn = torch.from_numpy(nn_host).to(dev)
    ff_ref = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    _, pot_ref, ec_ref, vir_ref = nb.lj_cut_coul_dsf_nonewton(ctx, pos, q, lj, s.ntypes, nl, nn,
                                                              na, p, ff=ff_ref)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    ffs = [torch.full((n, 3), float("nan"), dtype=torch.float32, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    rc, *_ = _noalloc(L, stream, n, pos, q, lj, s.ntypes, nl, nn, na, p, ffs[2])  # warm-up
    assert rc == _lib.SOFIA_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    results = []
    for call in range(2):
        results.append(_noalloc(L, stream, n, pos, q, lj, s.ntypes, nl, nn, na, p, ffs[call]))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0, "the calls changed the device's free memory"
    for call, (rc, pot, ec, vir) in enumerate(results):
        ff = ffs[call]
        assert rc == _lib.SOFIA_OK, f"call {call}: rc {rc}"
        assert abs(pot - pot_ref) <= FP64_TOL * abs(pot_ref)
        assert abs(ec - ec_ref) <= FP64_TOL * abs(ec_ref)
        assert np.abs(vir - vir_ref).max() <= FP64_TOL * np.abs(vir_ref).max()
        # forces are the real*4 rounding of FP64 sums: within one real*4 ulp
        a = ff.cpu().numpy()
        b = ff_ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.abs(a - b).max() <= np.spacing(np.abs(b).max())
    del sb, n3


def test_noalloc_rejects_oversize_and_host_buffers(ctx):
    import torch
    s = small_system()
    p = ref_params(s)
    n = s.np_atoms
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(s.position_aos()).to(dev)
    q = torch.from_numpy(s.q).to(dev)
    lj = [torch.from_numpy(a).to(dev) for a in (s.lj1, s.lj2, s.lj3, s.lj4)]
    nl = torch.ones((n * 4,), dtype=torch.int32, device=dev)
    nn = torch.zeros((n,), dtype=torch.int32, device=dev)
    ff = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    big = _lib.SOFIA_NOALLOC_MAX_ATOMS + 1
    rc, *_ = _noalloc(L, stream, big, pos, q, lj, s.ntypes, nl, nn, 4, p, ff)
    assert rc == _lib.SOFIA_ETOOBIG
    host_q = torch.from_numpy(s.q.copy())  # host memory: rejected, nothing is staged
    rc, *_ = _noalloc(L, stream, n, pos, host_q, lj, s.ntypes, nl, nn, 4, p, ff)
    assert rc == _lib.SOFIA_EINVAL
