"""The allocation-free Teter preconditioner entry point.

pw_teter_precond_noalloc serves callers that cannot allocate device memory
where they call it (inside stream capture, allocation-free hosts, pooled
framework memory).  It must give the same result as pw_teter_precond, called
through the C ABI, on two calls in a row (the fixed scratch array keeps the
previous call's contents), within the Teter parity tolerance of the other
GPU tests (1e-12 relative in FP64, 1e-5 in FP32).  This file is collected last
so a failure here does not hide the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from oracle import pw

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


def _ref_and_noalloc(c, r, w_ref, w_new, accumulate=0):
    from pwdft_develop_b200._lib import check, lib
    s = C.c_void_p(0)
    check(lib.pw_teter_precond(c.handle, C.c_void_p(r.data_ptr()), c.ntot, C.c_void_p(w_ref.data_ptr()), c.ntot,
                               r.shape[0], accumulate, s))
    check(lib.pw_teter_precond_noalloc(c.handle, C.c_void_p(r.data_ptr()), c.ntot, C.c_void_p(w_new.data_ptr()),
                                       c.ntot, r.shape[0], accumulate, s))


@pytest.mark.parametrize("prec,nc,nb", [("f64", (24, 24, 24), 7), ("f32", (24, 24, 24), 24),
                                        ("f32", (48, 48, 48), 40)])
def test_noalloc_matches_allocating_entry(prec, nc, nb):
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = pw.make_crystal("Si", (nc[0] // 24,) * 3, 10.26, 0.02, 3)
    c = Context(L, nc, tuple(2 * n for n in nc), precision=prec)
    dt = c.torch_dtype
    g = torch.Generator(device="cuda").manual_seed(11)
    for call in range(2):      # two calls in a row with different inputs
        r = torch.randn((nb, c.ntot), dtype=dt, device="cuda", generator=g)
        w_ref = torch.zeros_like(r)
        w_new = torch.full_like(r, float("nan"))
        _ref_and_noalloc(c, r, w_ref, w_new)
        torch.cuda.synchronize()
        err = float((w_new.double() - w_ref.double()).abs().max() / w_ref.double().abs().max())
        assert err <= TOL[prec], (call, err)
    # after the calls above have loaded every kernel, a further call leaves the
    # device's free memory unchanged: it allocates nothing
    from pwdft_develop_b200._lib import check, lib
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    check(lib.pw_teter_precond_noalloc(c.handle, C.c_void_p(r.data_ptr()), c.ntot, C.c_void_p(w_new.data_ptr()),
                                       c.ntot, nb, 0, C.c_void_p(0)))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # accumulate semantics: w += T r
    r = torch.randn((nb, c.ntot), dtype=dt, device="cuda", generator=g)
    base = torch.randn_like(r)
    w_ref, w_new = base.clone(), base.clone()
    _ref_and_noalloc(c, r, w_ref, w_new, accumulate=1)
    torch.cuda.synchronize()
    err = float((w_new.double() - w_ref.double()).abs().max() / w_ref.double().abs().max())
    assert err <= TOL[prec]
    c.close()
