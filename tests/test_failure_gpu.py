"""Failure detection of the bounded device waits, without a GPU fault.

A wait that nothing releases (pw_wait_probe: an mbarrier no thread arrives
on) gives up after its limit, the call reports PW_ETIMEOUT through the C ABI
and the context stays usable: a tensor-core Gram and an H*psi right after it
give the right numbers.  The run-time limit of the GEMM pipeline waits
(pw_set_wait_limit) can be shortened and restored without changing results."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx():
    from pwdft_develop_b200 import Context
    c = Context((10.26,) * 3, (24, 24, 24), (48, 48, 48), precision="f32")
    c.set_check_errors(True)
    return c


def _gram_ok(c, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    X = torch.randn((40, c.ntot), device="cuda", generator=g)
    G = c.gram(X)
    ref = X.double() @ X.double().T
    assert float((G - ref).abs().max() / ref.abs().max()) < 3e-5


def test_wait_probe_times_out_and_context_survives():
    from pwdft_develop_b200._lib import PW_ETIMEOUT, lib
    c = _ctx()
    _gram_ok(c, 1)
    t0 = time.perf_counter()
    rc = lib.pw_wait_probe(c.handle, C.c_double(0.05))
    dt = time.perf_counter() - t0
    assert rc == PW_ETIMEOUT
    assert b"timed out" in lib.pw_last_error()
    assert 0.04 < dt < 5.0
    # the record is cleared and the device keeps working
    _gram_ok(c, 2)
    import torch
    c.set_vtot(np.zeros(c.ntotFine))
    X = torch.randn((4, c.ntot), device="cuda")
    Y = c.hpsi(X)
    assert bool(torch.isfinite(Y).all())
    c.close()


def test_wait_limit_is_settable():
    from pwdft_develop_b200._lib import PW_EINVAL, check, lib
    c = _ctx()
    check(lib.pw_set_wait_limit(c.handle, C.c_double(0.5)))
    _gram_ok(c, 3)
    assert lib.pw_set_wait_limit(c.handle, C.c_double(-1.0)) == PW_EINVAL
    check(lib.pw_set_wait_limit(c.handle, C.c_double(2.0)))
    _gram_ok(c, 4)
    c.close()
