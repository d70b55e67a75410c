"""EIG restart file: the reference's serialize() layout of a DblNumVec
(include/utility.hpp:1183-1189: int32 length, then the doubles) written and
read through the C ABI, parsed independently here.  No GPU needed."""
import struct

import numpy as np
import pytest

from pwdft_develop_b200 import PwError
from pwdft_develop_b200.core import read_eig, write_eig


def test_eig_layout_and_round_trip(tmp_path):
    e = np.array([-0.31, -0.12, 0.0, 0.25, 1e-300, -7.5])
    p = tmp_path / "EIG"
    write_eig(p, e)
    raw = p.read_bytes()
    assert len(raw) == 4 + 8 * e.size
    (n,) = struct.unpack("=i", raw[:4])
    assert n == e.size
    assert np.array_equal(np.frombuffer(raw[4:], dtype=np.float64), e)
    assert np.array_equal(read_eig(p), e)


def test_truncated_file_is_an_error(tmp_path):
    p = tmp_path / "EIG"
    p.write_bytes(struct.pack("=i", 5) + np.zeros(3).tobytes())
    with pytest.raises(PwError, match="truncated"):
        read_eig(p)
