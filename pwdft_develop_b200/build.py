"""Build recipe for the native library ``libpwdft_b200.so`` (sm_100a).

Compiles every ``csrc/*.cu`` / ``csrc/*.cpp`` with nvcc in parallel into
``_build/`` objects and links them in-tree next to this file, so the shared
object travels with the source tree.  Objects are rebuilt when a source or
any header in ``csrc/`` / ``include/`` is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "obj"
LIB = PKG / "libpwdft_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-I", str(ROOT / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.inc")) + \
        list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def grids() -> list[tuple[int, int, int]]:
    """The coarse grids listed in csrc/grids.inc (PWB_GRID(n0, n1, n2) lines)."""
    out = []
    for line in (CSRC / "grids.inc").read_text().splitlines():
        m = re.match(r"\s*PWB_GRID\((\d+),\s*(\d+),\s*(\d+)\)", line)
        if m:
            out.append(tuple(int(x) for x in m.groups()))
    return out


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, jobs: int | None = None, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    extra = list(extra or [])
    inst = CSRC / "grid_instance.cu"
    srcs = [s for s in sorted(CSRC.glob("*.cu")) if s != inst] + sorted(CSRC.glob("*.cpp"))
    hmt = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hmt):
            todo.append((s, o, extra))
    # one object per grid of grids.inc (parallel compilation of the templates)
    for g in grids():
        o = BUILD / f"grid_{g[0]}_{g[1]}_{g[2]}.o"
        objs.append(o)
        if not o.exists() or o.stat().st_mtime < max(inst.stat().st_mtime, hmt):
            todo.append((inst, o, extra + [f"-DPWB_N0={g[0]}", f"-DPWB_N1={g[1]}", f"-DPWB_N2={g[2]}"]))
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o, e) for s, o, e in todo]
            for f in cf.as_completed(futs):
                o, log = f.result()
                if verbose:
                    print(f"built {o.name}", file=sys.stderr)
                    if log.strip():
                        print(log, file=sys.stderr)
    if todo or not LIB.exists():
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + \
            ["-lcublas", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
