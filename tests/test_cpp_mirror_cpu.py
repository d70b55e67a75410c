"""The C++ host mirror header compiles and links against the library (no GPU
needed to build)."""
import shutil

import pytest

from cpp_mirror import build_demo


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_mirror_demo_builds(tmp_path):
    exe = build_demo(tmp_path / "mirror_demo")
    assert exe.exists()
