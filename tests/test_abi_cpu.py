"""The C-ABI library loads, exports every symbol include/*.h declares, and
rejects bad arguments with status codes -- no GPU compute involved."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(pw_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_all_declared_symbols():
    from pwdft_develop_b200 import _lib
    names = _declared()
    assert names, "no declarations found"
    for n in sorted(names):
        assert hasattr(_lib.lib, n), f"missing export {n}"
        assert n in _lib.SIGNATURES, f"no ctypes signature for {n}"


def test_version_and_error_strings():
    from pwdft_develop_b200 import _lib
    assert b"sm_100a" in _lib.lib.pw_version()
    assert isinstance(_lib.lib.pw_last_error(), bytes)


@pytest.mark.parametrize("grid,fine,code", [
    ((24, 24, 23), (48, 48, 46), -1),        # odd coarse size
    ((24, 24, 24), (48, 48, 40), -4),        # fine != 2 * coarse
    ((22, 22, 22), (44, 44, 44), -4),        # FFT length 22 not built
])
def test_ctx_create_rejects_bad_grids(grid, fine, code):
    from pwdft_develop_b200 import _lib
    h = C.c_void_p()
    L = (C.c_double * 3)(10.0, 10.0, 10.0)
    rc = _lib.lib.pw_ctx_create(L, (C.c_int * 3)(*grid), (C.c_int * 3)(*fine), 0, 0, C.byref(h))
    assert rc == code
    assert h.value is None
    assert len(_lib.lib.pw_last_error()) > 0


def test_null_arguments_rejected():
    from pwdft_develop_b200 import _lib
    assert _lib.lib.pw_ctx_create(None, None, None, 0, 0, None) == _lib.PW_EINVAL
    assert _lib.lib.pw_set_vtot(None, None) == _lib.PW_EINVAL
    assert _lib.lib.pw_hpsi(None, None, 0, None, 0, 0, 0, None) == _lib.PW_EINVAL
    assert _lib.lib.pw_ctx_destroy(None) == _lib.PW_OK
