"""Build helper for tests: compiles tests/cpp/mirror_demo.cpp against the C++
host mirror (include/pwdft_b200.hpp) and the in-tree library."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def cuda_home() -> Path:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and Path(c, "include", "cuda_runtime.h").exists():
            return Path(c)
    raise RuntimeError("CUDA toolkit headers not found")


def build_demo(out: Path) -> Path:
    lib = ROOT / "pwdft_develop_b200"
    cu = cuda_home()
    cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{cu / 'include'}",
           str(ROOT / "tests" / "cpp" / "mirror_demo.cpp"), "-o", str(out), f"-L{lib}", "-lpwdft_b200",
           f"-L{cu / 'lib64'}", "-lcudart", f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{cu / 'lib64'}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out
