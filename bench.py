"""Benchmark: H*psi bands/s on Si64 (2x2x2 diamond Si, a = 20.52 bohr, 48^3
coarse / 96^3 fine grids, 160 bands, HGH LDA with real-space projectors).

One step = one H*psi sweep over the 160-band block (KohnSham::MultSpinor on
every band).  `value` is the device-timed throughput with inputs resident in
HBM (L2 flushed between steps); `e2e` is the same sweep through the host
C-ABI entry pw_hpsi_host (host->device copy of psi and device->host copy of
H*psi inside the timed region).  Under torchrun each rank runs its own
160-band block (bands shard with no exchange: weak scaling) and rank 0 prints
the JSON line with the max-over-ranks time.

--impl reference times the reference algorithm's CPU form (the FP64 NumPy
restatement in oracle/): one worker process per host core, tables built once
per process, each step a bounded sample of single-band H*psi applications.
The end of the JSON line carries a `summary` of the headline figures (FP32
and FP64 sweeps, e2e, SCF mixed vs FP64, Gram tensor fraction, CPU baselines).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SEED = 20261203 + 2          # configuration 2 (Si64)
NC = (48, 48, 48)
NF = (96, 96, 96)
NBAND = 160
A_CELL = 10.26
WORKLOAD = ("Si64 diamond 2x2x2 (a=20.52 bohr, +-0.02 bohr seeded displacements), HGH LDA, "
            "48^3 coarse / 96^3 fine grids, 160 bands (128 occ + 32 extra), real-space projectors")


def si64_atoms():
    rng = np.random.Generator(np.random.Philox(SEED))
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    pos = []
    for cz in range(2):
        for cy in range(2):
            for cx in range(2):
                for f in base:
                    pos.append((np.array([cx, cy, cz]) + f) * A_CELL)
    pos = np.array(pos) + rng.uniform(-0.02, 0.02, size=(64, 3))
    return np.array([2 * A_CELL] * 3), np.full(64, 14, np.int32), pos


EXX_GOLDEN = ROOT / "tests" / "golden" / "si64_exx_energy.json"


def seeded_orthonormal_bands(ntot: int, nb: int, seed: int) -> np.ndarray:
    """nb Gaussian bands (Philox stream `seed`, drawn as an ntot x nb matrix)
    orthonormalised by Cholesky-QR, returned as rows (nb, ntot)."""
    rng = np.random.Generator(np.random.Philox(seed))
    X = rng.standard_normal((ntot, nb))
    U = np.linalg.cholesky(X.T @ X).T
    return np.ascontiguousarray(np.linalg.solve(U.T, X.T))


def synthetic_vtot(n):
    rng = np.random.Generator(np.random.Philox(SEED + 100))
    return rng.uniform(-1.0, 0.5, size=n)


def load_traffic(prec: str, kind: str, npair: int):
    """DRAM bytes per launch of one kernel kind from the committed ncu summary
    (profiles/hpsi_si64_<prec>_dram_traffic.md, captured at 80 pairs per
    launch), scaled to npair pairs; None when no summary exists."""
    f = ROOT / "profiles" / f"hpsi_si64_{prec}_dram_traffic.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) == 6 and cells[0] == kind:
            try:
                return float(cells[4]) * 1e6 * npair / 80.0
            except ValueError:
                return None
    return None


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# algorithmic bytes per launch of each kernel kind for one batch of npair pairs
def algorithmic_bytes(kind: int, npair: int, s: int, nent: int, npmax: int, nslot: int, natom: int) -> float:
    nc = NC[0] * NC[1] * NC[2]
    nf = NF[0] * NF[1] * NF[2]
    nb = NF[2] * (NC[1] + 1) * (NC[0] + 1)
    c = 2 * s
    tables = nent * (4 + npmax * s) + nslot * 12
    if kind == 0:   # coarse xy forward: 2 real bands in, complex field out
        return npair * (2 * nc * s + nc * c)
    if kind == 1:   # z pad: A in, K out, B out (+ ekin table once)
        return npair * (nc * c + nc * c + nb * c) + nc * s
    if kind == 2:   # fine-plane gather: B in, partial dots out (+ tables once)
        return npair * (nb * c + nslot * npmax * c) + tables
    if kind == 3:   # projector reduce
        return npair * (nslot * npmax * c + natom * npmax * c)
    if kind == 4:   # fine-plane apply (dense projector mode): B in, C out, V_loc once
        return npair * 2 * nb * c + nf * s
    if kind == 5:   # z fold: C in, K in, D out
        return npair * (nb * c + 2 * nc * c)
    if kind == 6:   # coarse xy inverse: D in, 2 real bands out
        return npair * (nc * c + 2 * nc * s)
    return 0.0


def hpsi_model_bytes_per_band(s: int, bw: int, nproj: int, natom: int, npts_total: int) -> float:
    """Pinned whole-H*psi model: B_band(s) = 2sN_c + 4s(2H_c+2H_f) + 2sN_f + 4sH_c
    + [sN_f + (s n_proj + 4 n_atom) n_pts]/bw."""
    nc = NC[0] * NC[1] * NC[2]
    nf = NF[0] * NF[1] * NF[2]
    hc = (NC[0] // 2 + 1) * NC[1] * NC[2]
    hf = (NF[0] // 2 + 1) * NF[1] * NF[2]
    npts = npts_total / max(natom, 1)
    return 2 * s * nc + 4 * s * (2 * hc + 2 * hf) + 2 * s * nf + 4 * s * hc + \
        (s * nf + (s * nproj + 4 * natom) * npts) / bw


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        lines = Path(self.file.name).read_text().strip().splitlines()
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


_W = {}


_THREAD_VARS = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")


def _oracle_worker_init(backend: str = "numpy", workers: int = 1):
    """Pool initializer: one thread per process, the Si64 tables built once
    per worker (set-up, outside every timed region)."""
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass
    from oracle import pw
    pw.set_fft_backend(backend, workers)
    L, z, pos = si64_atoms()
    _W["T"], _ = pw.build_tables(L, 14, pos, NC, NF, vtot=synthetic_vtot(int(np.prod(NF))))


def _oracle_worker_hpsi(job):
    """`nb` single-band H*psi applications (FP64 NumPy restatement of the
    reference path) on seeded bands; returns the time spent in mult_spinor."""
    from oracle import pw
    seed, nb = job
    T = _W["T"]
    rng = np.random.Generator(np.random.Philox(SEED + 7 + seed))
    psi = rng.standard_normal((nb, T.dm.ntot))
    t0 = time.perf_counter()
    for b in range(nb):
        pw.mult_spinor(T, psi[b:b + 1])
    return time.perf_counter() - t0


def _oracle_pool(ncores: int):
    """`ncores` spawned worker processes, each limited to one BLAS / OpenMP
    thread (the variables are set before the children import NumPy)."""
    import multiprocessing as mp
    saved = {k: os.environ.get(k) for k in _THREAD_VARS}
    for k in _THREAD_VARS:
        os.environ[k] = "1"
    try:
        return mp.get_context("spawn").Pool(ncores, initializer=_oracle_worker_init)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _pool_sweep(pool, ncores: int, bands_per_core: int, seed0: int):
    """One sample: every worker applies H to `bands_per_core` bands; wall time
    of the whole sample (all workers busy at once) and the summed compute time."""
    t0 = time.perf_counter()
    ts = pool.map(_oracle_worker_hpsi, [(seed0 + i, bands_per_core) for i in range(ncores)], chunksize=1)
    return time.perf_counter() - t0, sum(ts)


REF_HPSI_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "libpwref_hpsi.so")
REF_SAMPLE_NOTE = ("the reference's own Spinor::AddMultSpinorFineR2C (src/SCF/spinor.cpp:377) with IP_c2f / IP_f2c, "
                   "compiled from the reference sources (g++ -O3, OpenMP over bands, one Fourier per thread) over a "
                   "harness whose radix-2/3/4/5 FFT stands in for FFTW (absent from the image)")


class _RefHpsi:
    """The reference's compiled H*psi composition (oracle/_ref, built by
    oracle/build_ref.py) on the Si64 workload: tables built once (set-up),
    one call per sample with the bands spread over `threads` OpenMP threads."""

    def __init__(self):
        import ctypes as C
        from oracle import pw
        self.lib = C.CDLL(REF_HPSI_LIB)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        self.lib.ref_add_mult_spinor_omp.argtypes = [ip, ip, dp, dp, dp, C.c_int, ip, ip, ip, dp, dp, C.c_int, dp,
                                                     dp, C.c_int]
        L, z, pos = si64_atoms()
        T, _ = pw.build_tables(L, 14, pos, NC, NF, vtot=synthetic_vtot(int(np.prod(NF))))
        self.ntot = T.dm.ntot
        self.args = (np.array(NC, np.int32), np.array(NF, np.int32), np.array(L, np.float64),
                     np.ascontiguousarray(T.ekin.ravel()), np.ascontiguousarray(T.vtot), len(T.pseudo),
                     np.array([len(at[0].idx) for at in T.pseudo], np.int32),
                     np.array([len(at) for at in T.pseudo], np.int32),
                     np.concatenate([at[0].idx for at in T.pseudo]).astype(np.int32),
                     np.concatenate([pp.val[:, 0] for at in T.pseudo for pp in at]).astype(np.float64),
                     np.array([pp.wgt for at in T.pseudo for pp in at], np.float64))

    def sweep(self, nb: int, threads: int, seed: int) -> float:
        """Seconds for one call applying H to `nb` seeded bands."""
        rng = np.random.Generator(np.random.Philox(SEED + 7 + seed))
        psi = np.ascontiguousarray(rng.standard_normal((nb, self.ntot)))
        a3 = np.zeros_like(psi)
        t0 = time.perf_counter()
        rc = self.lib.ref_add_mult_spinor_omp(*self.args, nb, psi, a3, threads)
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError("compiled reference H*psi failed")
        return dt


def _ref_hpsi():
    return _RefHpsi() if os.path.exists(REF_HPSI_LIB) else None


def cpu_baseline(bands_per_core: int = 4):
    """The reference path on all host cores.  Where the reference's own H*psi
    composition was compiled (oracle/_ref travels with the repository), that is
    the baseline (kind "reference"): one call over ncores x bands_per_core
    bands on ncores OpenMP threads.  Beside it, or instead of it when it is
    absent, the FP64 NumPy restatement (kind "port": one process per core,
    one band per call, tables built once per process), and the same bands with
    scipy.fft on `nproc` threads in one process (batched transforms)."""
    ncores = os.cpu_count() or 1
    nb = ncores * bands_per_core
    with _oracle_pool(ncores) as pool:
        _pool_sweep(pool, ncores, 1, 10_000)               # warm: imports, FFT plans
        wall, busy = _pool_sweep(pool, ncores, bands_per_core, 0)
    port = {"value": nb / wall, "unit": "bands/s", "cores": ncores, "kind": "port",
            "sample": f"{nb} single-band H*psi applications of the Si64 workload through the FP64 NumPy restatement "
                      f"of the reference path (oracle/pw.py), {ncores} processes x {bands_per_core} bands, tables "
                      f"built once per process, {wall:.1f} s wall ({busy / nb * 1e3:.0f} ms per band per core)"}
    ref = _ref_hpsi()
    if ref is not None:
        ref.sweep(ncores, ncores, 20_000)                  # warm: first touch of the per-thread buffers
        dt = ref.sweep(nb, ncores, 0)
        out = {"value": nb / dt, "unit": "bands/s", "cores": ncores, "kind": "reference",
               "sample": f"{nb} bands of the Si64 workload (FP64) through {REF_SAMPLE_NOTE}; {ncores} threads, "
                         f"{dt:.1f} s", "port": port}
    else:
        out = port
    # scipy.fft with nproc worker threads on a block of bands in one process
    from oracle import pw
    L, z, pos = si64_atoms()
    T, _ = pw.build_tables(L, 14, pos, NC, NF, vtot=synthetic_vtot(int(np.prod(NF))))
    pw.set_fft_backend("scipy", ncores)
    try:
        rng = np.random.Generator(np.random.Philox(SEED + 7))
        psi = rng.standard_normal((nb, T.dm.ntot))
        pw.mult_spinor(T, psi[:2])
        t0 = time.perf_counter()
        for b0 in range(0, nb, 16):
            pw.mult_spinor(T, psi[b0:b0 + 16])
        dt = time.perf_counter() - t0
    finally:
        pw.set_fft_backend("numpy", 1)
    out["scipy_fft"] = {"value": nb / dt, "unit": "bands/s", "threads": ncores,
                        "sample": f"{nb} bands in blocks of 16 through the same restatement with scipy.fft "
                                  f"(workers={ncores}), {dt:.1f} s"}
    return out


def scf_bench(device: int, max_iter: int = 60):
    """SCF time to |E_free - E_Harris| / N_atom < 1e-6 Ha/atom on Si64 with
    ChebFSI (degree 10): plain FP64 against the mixed form (FP32 H*psi and
    Chebyshev filter, split-BF16 tensor-core Gram products, FP64 Cholesky /
    Rayleigh-Ritz / mixing, FP64 refinement once |E_free - E_Harris| / N_atom
    falls below 3e-6, i.e. within a factor 3 of the tolerance: the FP32 fixed
    point itself is biased by ~2e-6 Ha/atom).  Each run
    is bracketed by CUDA events on the device."""
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = si64_atoms()
    out = {}
    for mode in ("f64", "mixed"):
        c = Context(L, NC, NF, precision="f64", device=device)
        c.set_atoms(z, pos)
        c.set_band_batch(NBAND)
        if mode == "mixed":
            c.build_twin()          # set-up, like set_atoms: FP32 tables and projector matrix
        # untimed warm-up on the timed path (solver handles, first-use buffers and
        # kernel modules of both eigensolver precisions): 3 SCF iterations, then
        # one iteration forced to the FP64 refinement
        kw = dict(nocc=128, nextra=32, ecut=20.0, solver="chebfsi", mixed=(mode == "mixed"), cheby_degree=10,
                  seed=SEED, graphs=True)
        c.scf(cheby_first_cycles=5, tol_efree=1e-6, refine_threshold=3e-6, max_iter=3, **kw)
        c.scf(cheby_first_cycles=1, tol_efree=1e-6, refine_threshold=1e9, max_iter=1, **kw)
        torch.cuda.synchronize()
        # three timed runs (the SCF makes many small host round trips per iteration,
        # so a busy shared host shows up as run-to-run spread); the fastest is reported
        samples, sample_it = [], []
        best = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r_, eig_, _ = c.scf(cheby_first_cycles=5, tol_efree=1e-6, refine_threshold=3e-6, max_iter=max_iter,
                                verbose=int(os.environ.get("PWB_SCF_VERBOSE", "0")), **kw)
            e1.record()
            torch.cuda.synchronize()
            samples.append(e0.elapsed_time(e1) / 1e3)
            sample_it.append([r_["iterations"], r_["refine_iter"]])
            if best is None or samples[-1] <= min(samples):
                best = (r_, eig_)
        res, eig = best
        out[mode] = dict(seconds=min(samples), samples_s=samples, samples_iterations_refine=sample_it,
                         iterations=res["iterations"],
                         converged=bool(res["converged"]), efree=res["efree"], etot=res["etot"],
                         refine_iter=res["refine_iter"], hpsi_bands=res["hpsi_bands"], homo=float(eig[127]),
                         lumo=float(eig[128]))
        if os.environ.get("PWB_SCF_PHASES"):
            res2, _, _ = c.scf(nocc=128, nextra=32, ecut=20.0, solver="chebfsi", mixed=(mode == "mixed"),
                               cheby_degree=10, cheby_first_cycles=5, tol_efree=1e-6, refine_threshold=3e-6,
                               max_iter=max_iter, seed=SEED, verbose=2)
            out[mode]["phase_s"] = res2["phase_s"]
            out[mode]["sub_s"] = res2["sub_s"]
        c.close()
    out["speedup_mixed_vs_f64"] = out["f64"]["seconds"] / out["mixed"]["seconds"]
    out["efree_agreement_per_atom"] = abs(out["f64"]["efree"] - out["mixed"]["efree"]) / 64
    out["workload"] = ("Si64, ChebFSI degree 10 (5 cycles in the first SCF step), Anderson(8, 0.7), 300 K, "
                       "tol 1e-6 Ha/atom, Chebyshev filter replayed from a CUDA graph; fastest of three timed runs")
    return out


def solvers_bench(device: int, max_iter: int = 60):
    """The block eigensolvers of the reference in the Si64 SCF (FP64, 128
    occupied + 32 extra bands, tol 1e-6 Ha/atom, eig_max_iter 3): LOBPCG (the
    reference's default PW_Solver, its [X W P] subspace of 3 x 160 = 480
    through the library's generalized eigensolver twice per iteration), PPCG
    (sub-block size 1) and Davidson (2 blocks).  One untimed 2-iteration
    warm-up per solver, then one timed run bracketed by CUDA events."""
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = si64_atoms()
    out = {}
    for solver in ("lobpcg", "ppcg", "davidson"):
        c = Context(L, NC, NF, precision="f64", device=device)
        c.set_atoms(z, pos)
        c.set_band_batch(NBAND)
        kw = dict(nocc=128, nextra=32, ecut=20.0, solver=solver, seed=SEED, tol_efree=1e-6)
        c.scf(max_iter=2, **kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r_, _, _ = c.scf(max_iter=max_iter, **kw)
        e1.record()
        torch.cuda.synchronize()
        out[solver] = dict(seconds=e0.elapsed_time(e1) / 1e3, iterations=r_["iterations"],
                           converged=bool(r_["converged"]), efree=r_["efree"], hpsi_bands=r_["hpsi_bands"])
        c.close()
    out["workload"] = ("Si64 FP64, 160 bands, Anderson(8, 0.7), 300 K, tol 1e-6 Ha/atom, 3 eigensolver "
                       "iterations per SCF step")
    return out


def dense_bench(device: int):
    """The library's FP64 dense kernels at the subspace sizes of the Si64
    eigensolvers: the symmetric eigen-decomposition (pw_dense_syev) at
    n = 160 (ChebFSI Rayleigh-Ritz), 480 (LOBPCG's 3n) and 1440 (LOBPCG at 480
    bands), Cholesky and triangular inverse at n = 160.  Random symmetric
    matrices (seeded); median of 5 calls after 2 untimed, each synchronous."""
    import ctypes as C
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200._lib import check, lib
    c = Context((10.26,) * 3, (12, 12, 12), (24, 24, 24), precision="f64", device=device)

    def P(t):
        return C.c_void_p(t.data_ptr())
    out = {}
    dev = torch.device("cuda", device)
    for n in (160, 480, 1440):
        g = torch.Generator().manual_seed(n)
        M = torch.randn(n, n, generator=g, dtype=torch.float64)
        A = (M + M.T).to(dev)
        w = torch.empty(n, dtype=torch.float64, device=dev)
        sw = C.c_int(0)
        ts = []
        for r in range(7):
            B = A.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            check(lib.pw_dense_syev(c.handle, n, P(B), n, P(w), C.byref(sw)))
            ts.append(time.perf_counter() - t0)
        V = B.T
        res = float((A @ V - V * w).abs().max() / A.abs().max())
        orth = float((V.T @ V - torch.eye(n, dtype=torch.float64, device=dev)).abs().max())
        out[f"syev_n{n}"] = dict(ms=float(np.median(ts[2:])) * 1e3, residual=res, orthogonality=orth,
                                 jacobi_sweeps=sw.value)
    n = 160
    M = torch.randn(n, n, generator=torch.Generator().manual_seed(3), dtype=torch.float64)
    S = (M @ M.T + n * torch.eye(n, dtype=torch.float64)).to(dev)
    tp, tt = [], []
    for r in range(7):
        B = S.clone()
        Ui = torch.empty_like(B)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.pw_dense_potrf(c.handle, n, P(B), n))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        check(lib.pw_dense_trtri(c.handle, n, P(B), n, P(Ui), n))
        torch.cuda.synchronize()
        tp.append(t1 - t0)
        tt.append(time.perf_counter() - t1)
    out["potrf_n160_ms"] = float(np.median(tp[2:])) * 1e3
    out["trtri_n160_ms"] = float(np.median(tt[2:])) * 1e3
    c.close()
    return out


def hybrid_bench(device: int):
    """HSE06 SCF time to solution on Si64 (48^3 / 96^3, 128 occupied + 32 extra
    bands, ChebFSI degree 10, mixed precision): the reference's nested scheme
    -- a PBE SCF to |E_free - E_Harris| / N_atom < 1e-6 Ha/atom, then phi
    iterations (ACE from the bands, inner SCF with the ACE term, FP64) until
    dExx < 1e-6 Ha.  One untimed short run warms the path; one timed run."""
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = si64_atoms()
    c = Context(L, NC, NF, precision="f64", device=device)
    c.set_atoms(z, pos)
    c.set_band_batch(NBAND)
    c.build_twin()
    kw = dict(nocc=128, nextra=32, ecut=20.0, solver="chebfsi", mixed=True, cheby_degree=10, seed=SEED,
              graphs=True, xc="hse06", refine_threshold=3e-6)
    c.scf(cheby_first_cycles=5, tol_efree=1e-6, max_iter=2, phi_max_iter=1, phi_tol=1e-6, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res, eig, _ = c.scf(cheby_first_cycles=5, tol_efree=1e-6, max_iter=60, phi_max_iter=10, phi_tol=1e-6, **kw)
    e1.record()
    torch.cuda.synchronize()
    c.close()
    return {"workload": "Si64 HSE06 (nested phi iterations with ACE), mixed-precision ChebFSI, tol 1e-6 Ha/atom, "
                        "dExx < 1e-6",
            "seconds": e0.elapsed_time(e1) / 1e3, "converged": bool(res["converged"]),
            "scf_iterations": res["iterations"], "phi_iterations": res["phi_iterations"], "dexx": res["dexx"],
            "efock": res["efock"], "efree": res["efree"], "hpsi_bands": res["hpsi_bands"]}


def exx_bench(device: int, reps: int = 3):
    """Hybrid exchange on Si64 (48^3 coarse grid, 160 bands, 128 occupied;
    PBE0 mixing 0.25, Coulomb kernel with the divergence correction): time of
    V_x psi over all (band, occupied orbital) pairs in FP32 and FP64, the ACE
    build, and the FP32 exchange energy against the FP64 one (per atom)."""
    import torch
    from pwdft_develop_b200 import Context
    L, z, pos = si64_atoms()
    nb, nocc = 160, 128
    gold = json.loads(EXX_GOLDEN.read_text()) if EXX_GOLDEN.exists() else None
    X64 = torch.tensor(seeded_orthonormal_bands(NC[0] * NC[1] * NC[2], nb, gold["psi_seed"] if gold else SEED + 7),
                       device="cuda")
    occ = np.zeros(nb)
    occ[:nocc] = 1.0
    out = {"workload": "Si64 48^3, 160 bands x 128 occupied orbitals, PBE0 fraction 0.25, divergence type 1",
           "pairs": nb * nocc}
    energies = {}
    for prec in ("f32", "f64"):
        c = Context(L, NC, NF, precision=prec, device=device)
        c.set_atoms(z, pos)
        c.exx_setup(0.25, 0.0, 1, 20.0)
        X = X64.to(c.torch_dtype).contiguous()
        c.exx_set_phi(X, occ)
        Y = torch.empty_like(X)
        c.exx_apply(X, out=Y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            c.exx_apply(X, out=Y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        s = 4 if prec == "f32" else 8
        ntot = NC[0] * NC[1] * NC[2]
        hc = (NC[0] // 2 + 1) * NC[1] * NC[2]
        pair_bytes = 4 * s * ntot + 8 * s * hc
        peak, peak_kind = load_peaks()
        d = {"vx_psi_ms": ms, "pairs_per_s": nb * nocc / (ms / 1e3),
             "model_bytes_per_pair": pair_bytes,
             "model_frac_of_hbm": nb * nocc * pair_bytes / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind}
        energies[prec] = c.exx_energy(X, occ)
        e0.record()
        c.ace_build(X)
        e1.record()
        torch.cuda.synchronize()
        d["ace_build_ms"] = e0.elapsed_time(e1)
        d["exchange_energy"] = energies[prec]
        out[prec] = d
        c.close()
    out["exchange_energy_error_per_atom_f32"] = abs(energies["f32"] - energies["f64"]) / 64
    if gold is not None:
        # against the FP64 oracle's energy of the same bands (committed fixture)
        out["oracle_exchange_energy"] = gold["exchange_energy"]
        out["exchange_energy_error_per_atom_vs_oracle"] = {
            p: abs(energies[p] - gold["exchange_energy"]) / gold["natom"] for p in ("f32", "f64")}
    return out


def cells_bench(device: int, reps: int = 5):
    """48 independent uneven cells (Si8/16/64, Al4/32, Ecut 8-20 Ha, grids
    20^3-48^3, 12-160 bands) applied sequentially, on forked streams, and as
    one captured CUDA graph; FP32, synthetic V_loc and bands."""
    import torch
    from pwdft_develop_b200 import CellBatch, Context
    from pwdft_develop_b200.cells import uneven_cells
    cells = uneven_cells(48)
    rng = np.random.Generator(np.random.Philox(SEED + 11))
    ctxs, psis, outs = [], [], []
    for cell in cells:
        c = Context(cell["length"], cell["numGrid"], cell["numGridFine"], precision="f32", device=device)
        c.set_atoms([cell["znuc"]] * len(cell["positions"]), cell["positions"])
        c.set_vtot(rng.uniform(-1.0, 0.5, c.ntotFine))
        c.set_band_batch(cell["nband"])
        x = torch.tensor(rng.standard_normal((cell["nband"], c.ntot)) / np.sqrt(c.ntot), dtype=torch.float32,
                         device="cuda")
        ctxs.append(c)
        psis.append(x)
        outs.append(torch.empty_like(x))
    nbands = sum(c["nband"] for c in cells)
    b = CellBatch(ctxs, psis, outs)
    g = b.capture()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_seq = timed(lambda: [c.hpsi(x, out=o) for c, x, o in zip(ctxs, psis, outs)])
    t_bat = timed(b.hpsi)
    t_gr = timed(g.replay)
    nodes = g.nodes
    g.close()
    for c in ctxs:
        c.close()
    return {"workload": "48 seeded cells (Si8/16/64, Al4/32, Ecut 8-20 Ha, 20^3-48^3 grids), FP32",
            "bands": nbands, "sequential_ms": t_seq, "streams_ms": t_bat, "graph_ms": t_gr, "graph_nodes": nodes,
            "graph_bands_per_s": nbands / (t_gr / 1e3), "sequential_bands_per_s": nbands / (t_seq / 1e3)}


def gram_bench(device: int, reps: int = 10):
    """Eigensolver Gram blocks X^T Y on the Si64 grid (K = 110,592) in FP32
    contexts: split-BF16 tcgen05 GEMM (3 products, FP32 accumulation, split-K
    with an FP64 reduction), for the ChebFSI / Cholesky-QR width (160) and the
    LOBPCG [X W P] width (480).  Reports the whole pw_gram call (operand
    split + GEMM + reduction) and the tensor-core kernel alone."""
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.core import KERNEL_KINDS
    L, z, pos = si64_atoms()
    c = Context(L, NC, NF, precision="f32", device=device)
    K = c.ntot
    peaks = {}
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        peaks = json.loads(p.read_text())
    tpeak = float(peaks.get("bf16_tflops", 1590.0))
    out = {"K": K, "tensor_peak_tflops": tpeak,
           "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"}
    g = torch.Generator(device="cuda").manual_seed(SEED + 21)
    gkind = [k for k, v in KERNEL_KINDS.items() if v == "gram"][0]
    for n in (160, 480):
        X = torch.randn((n, K), dtype=torch.float32, device="cuda", generator=g)
        c.gram(X)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            c.gram(X)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        c.profile(True)
        for _ in range(reps):
            c.gram(X)
        torch.cuda.synchronize()
        kms, kn = c.profile_read(gkind)
        c.profile(False)
        useful = 2.0 * K * n * n
        kern_ms = kms / kn if kn else None                  # tensor-core GEMM + split-K reduction
        out[f"n{n}"] = {"call_ms": ms, "useful_tflops": useful / (ms / 1e3) / 1e12,
                        "tensor_tflops_3products": 3 * useful / (ms / 1e3) / 1e12,
                        "tensor_frac": 3 * useful / (ms / 1e3) / 1e12 / tpeak,
                        "gemm_and_reduce_ms": kern_ms,
                        "gemm_tensor_frac": (3 * useful / (kern_ms / 1e3) / 1e12 / tpeak) if kern_ms else None,
                        "operand_bytes": 2 * n * K * 4,
                        "hbm_frac_of_operand_reads": 2 * n * K * 4 / (ms / 1e3) / 1e9 / load_peaks()[0]}
        # the subspace rotation X C (n x n coefficients) on the same tensor cores
        import ctypes as C
        from pwdft_develop_b200._lib import check, lib
        Cm = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
        Out = torch.empty_like(X)
        rot = lambda: check(lib.pw_rotate(c.handle, C.c_void_p(X.data_ptr()), K, n, C.c_void_p(Cm.data_ptr()), n,  # noqa
                                          n, C.c_void_p(Out.data_ptr()), K, 0, None))
        rot()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            rot()
        e1.record()
        torch.cuda.synchronize()
        rms = e0.elapsed_time(e1) / reps
        out[f"n{n}"]["rotation"] = {"call_ms": rms, "useful_tflops": useful / (rms / 1e3) / 1e12,
                                    "tensor_frac": 3 * useful / (rms / 1e3) / 1e12 / tpeak,
                                    "hbm_frac_of_in_out": 2 * n * K * 4 / (rms / 1e3) / 1e9 / load_peaks()[0]}
    c.close()
    return out


def kpoint_bench(device: int, reps: int = 5):
    """Si8 complex bands on a 4x4x4 Monkhorst-Pack k-mesh (64 k-points, 24
    bands each, 24^3 / 48^3 grids, Ecut 10 Ha) in one batched H(k) psi pass, FP32."""
    import torch
    from pwdft_develop_b200 import Context
    rng = np.random.Generator(np.random.Philox(SEED + 3))
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    pos = base * A_CELL + rng.uniform(-0.02, 0.02, size=(8, 3))
    L, z = np.array([A_CELL] * 3), 14
    nc, nf, nb = (24, 24, 24), (48, 48, 48), 24
    b = 2 * np.pi / A_CELL
    mp = [(2 * i - 3) / 8.0 for i in range(4)]
    kpts = np.array([[x, y, w] for x in mp for y in mp for w in mp]) * b
    c = Context(L, nc, nf, precision="f32", device=device)
    c.set_atoms([z] * len(pos), pos)
    c.set_vtot(synthetic_vtot(c.ntotFine))
    c.set_band_batch(2 * 256)
    c.set_kpoints(kpts)
    g = torch.Generator(device="cuda").manual_seed(SEED + 9)
    X = torch.randn((len(kpts), nb, c.ntot), dtype=torch.complex64, device="cuda", generator=g)
    Y = torch.empty_like(X)
    c.hpsi_kbatch(X, out=Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        c.hpsi_kbatch(X, out=Y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    c.close()
    return {"workload": "Si8 4x4x4 MP (64 k), 24 complex bands per k, 24^3/48^3, FP32",
            "ms_per_pass": ms, "k_bands_per_s": len(kpts) * nb / (ms / 1e3)}


def gspace_bench(device: int, reps: int = 10):
    """Sphere-cut (G-space) H*psi on the Si64 cell: 96^3 G-space grid, Ecut
    25 Ha, 160 bands of half-sphere coefficients, Fourier-space HGH
    projectors; device-timed per sweep with the L2 flushed in between.  Byte
    model per band pair: the slot field (N x (n+1)^2 complex) is written by
    the scatter, read and written by the fine-plane kernel and read by the
    gather (4 passes), and the two bands are read once and written once
    (2 x 2 x 2 ns s)."""
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.core import KERNEL_KINDS
    L, z, pos = si64_atoms()
    N, ecut = (96, 96, 96), 25.0
    peak = load_peaks()[0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"workload": "Si64 sphere-cut: 96^3 G-space grid, Ecut 25 Ha, 160 bands, Fourier-space HGH projectors "
                       "(Use_Real_Space 0)"}
    for prec in ("f32", "f64"):
        c = Context.gspace(L, N, ecut, precision=prec, device=device)
        c.set_atoms(z, pos)
        c.set_vtot(synthetic_vtot(c.ntotFine))
        c.set_band_batch(NBAND)
        g = torch.Generator(device="cuda").manual_seed(SEED + 11)
        X = torch.randn((NBAND, c.ntot), dtype=c.torch_dtype, device="cuda", generator=g)
        X[:, 1] = 0                                    # Im c_0
        Y = torch.empty_like(X)
        for _ in range(3):
            c.hpsi(X, out=Y)
        torch.cuda.synchronize()
        c.profile(True)
        ms = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            c.hpsi(X, out=Y)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms /= reps
        kern = {}
        rename = {"z_pad": "sphere_scatter_z_inverse", "z_fold": "z_forward_sphere_gather",
                  "gram": "projector_gemm", "other": "bf16_split"}
        for kind, name in KERNEL_KINDS.items():
            t, n = c.profile_read(kind)
            if n:
                kern[rename.get(name, name)] = {"launches": n, "avg_us": t / n * 1e3}
        c.profile(False)
        s = 4 if prec == "f32" else 8
        ns = c.ns
        field = N[2] * (N[1] // 2 + 1) * (N[0] // 2 + 1) * 2 * s
        pair_bytes = 4 * field + 2 * (2 * 2 * ns * s)
        bands_per_s = NBAND / (ms / 1e3)
        out[prec] = {"ns": ns, "ms_per_sweep": ms, "bands_per_s": bands_per_s,
                     "model_bytes_per_band": pair_bytes / 2,
                     "model_frac_of_hbm": pair_bytes / 2 * bands_per_s / (peak * 1e9), "kernels": kern}
        # sphere-cut exact exchange (HSE06 kernel): 32 bands x 128 occupied
        # orbitals, pair products on the full 96^3 grid (axis FFTs in the
        # context's precision)
        nk, nphi = 32, 128
        c.exx_setup(0.25, 0.106, 1, ecut)
        c.exx_set_phi(X[:nphi].contiguous(), np.ones(nphi))
        Xk = X[:nk].contiguous()
        V = c.exx_apply(Xk)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c.exx_apply(Xk, out=V)
        e1.record()
        torch.cuda.synchronize()
        xms = e0.elapsed_time(e1)
        out["exx_" + prec] = {"workload": "sphere-cut V_x psi, 32 bands x 128 orbitals (64 pair fields per band), "
                                          "96^3 grid, HSE06 kernel (mu 0.106)",
                              "ms": xms, "pairs_per_s": nk * nphi / (xms / 1e3)}
        c.close()
    return out


def f64_sweep_bench(device: int, steps: int, warmup: int):
    """The same Si64 sweep in FP64 (the reference path's precision):
    device-timed per 160-band sweep with the L2 flushed in between, and the
    dominant kernel's achieved bandwidth on its algorithmic bytes."""
    import torch
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.core import KERNEL_KINDS
    L, z, pos = si64_atoms()
    c = Context(L, NC, NF, precision="f64", device=device)
    c.set_vtot(synthetic_vtot(c.ntotFine))
    c.set_atoms(z, pos)
    c.set_band_batch(NBAND)
    g = torch.Generator(device="cuda").manual_seed(SEED)
    X = torch.randn((NBAND, c.ntot), dtype=torch.float64, device="cuda", generator=g) / math.sqrt(c.ntot)
    Y = torch.empty_like(X)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        c.hpsi(X, out=Y)
    torch.cuda.synchronize()
    ms = 0.0
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        c.hpsi(X, out=Y)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= steps
    c.profile(True)
    for _ in range(steps):
        flush.zero_()
        c.hpsi(X, out=Y)
    torch.cuda.synchronize()
    kern = {}
    for k in range(12):
        t, n = c.profile_read(k)
        if n:
            kern[KERNEL_KINDS[k]] = {"launches": n, "avg_us": t / n * 1e3, "total_ms": t}
    c.profile(False)
    c.close()
    dom = max((k for k in kern if k != "library_gemm"), key=lambda k: kern[k]["total_ms"])
    kind = [k for k, v in KERNEL_KINDS.items() if v == dom][0]
    alg = algorithmic_bytes(kind, NBAND // 2, 8, 0, 5, 0, len(pos))
    peak, peak_kind = load_peaks()
    ach = alg / (kern[dom]["avg_us"] * 1e-6) / 1e9
    return {"value": NBAND / (ms / 1e3), "unit": "bands/s", "ms_per_sweep": ms, "dtype": "f64",
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg,
                         "avg_launch_us": kern[dom]["avg_us"]},
            "kernels": kern}


def summary(line: dict) -> dict:
    """The headline figures of the line, gathered at its end."""
    out = {"hpsi_f32_bands_per_s": line.get("value"), "e2e_bands_per_s": line.get("e2e", {}).get("value"),
           "roofline_frac": line.get("roofline", {}).get("frac"),
           "hpsi_model_frac": line.get("hpsi_model", {}).get("frac")}
    if "f64_sweep" in line:
        out["hpsi_f64_bands_per_s"] = line["f64_sweep"]["value"]
        out["f64_roofline_frac"] = line["f64_sweep"]["roofline"]["frac"]
    if "scf" in line:
        sc = line["scf"]
        out["scf_f64_s"] = sc["f64"]["seconds"]
        out["scf_mixed_s"] = sc["mixed"]["seconds"]
        out["scf_speedup_mixed_vs_f64"] = sc["speedup_mixed_vs_f64"]
        out["scf_efree_agreement_per_atom"] = sc["efree_agreement_per_atom"]
    if "solvers" in line:
        for k in ("lobpcg", "ppcg", "davidson"):
            out[f"scf_{k}_f64_s"] = line["solvers"][k]["seconds"]
    if "dense" in line:
        out["syev_n480_ms"] = line["dense"]["syev_n480"]["ms"]
        out["syev_n1440_ms"] = line["dense"]["syev_n1440"]["ms"]
    if "exx" in line and "exchange_energy_error_per_atom_vs_oracle" in line["exx"]:
        out["exx_energy_error_per_atom_vs_oracle"] = line["exx"]["exchange_energy_error_per_atom_vs_oracle"]
    if "gram" in line:
        out["gram_n480_tensor_frac"] = line["gram"]["n480"]["tensor_frac"]
        out["gram_n160_tensor_frac"] = line["gram"]["n160"]["tensor_frac"]
        if "rotation" in line["gram"]["n160"]:
            out["rotation_n160_ms"] = line["gram"]["n160"]["rotation"]["call_ms"]
            out["rotation_n480_tensor_frac"] = line["gram"]["n480"]["rotation"]["tensor_frac"]
    if "cpu_baseline" in line:
        cb = line["cpu_baseline"]
        out["cpu_baseline_bands_per_s"] = cb["value"]
        out["cpu_baseline_cores"] = cb["cores"]
        if "scipy_fft" in cb:
            out["cpu_scipy_fft_bands_per_s"] = cb["scipy_fft"]["value"]
    return out


def run_reference(args):
    """The reference path's CPU form on the host cores, each step a bounded
    sample of the Si64 sweep of ncores x `--ref-bands-per-core` bands: the
    reference's own H*psi composition compiled from its sources (oracle/_ref)
    on ncores OpenMP threads when it was built, else the FP64 NumPy
    restatement with one process per core (tables built once per process,
    outside the timed steps)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ncores = os.cpu_count() or 1
    bpc = args.ref_bands_per_core
    nb_step = ncores * bpc
    ref = _ref_hpsi()
    if ref is not None:
        for w in range(args.warmup):
            ref.sweep(ncores, ncores, 100_000 + w * ncores)
        wall = sum(ref.sweep(nb_step, ncores, s * nb_step) for s in range(args.steps))
        nb = args.steps * nb_step
        cb = {"kind": "reference", "cores": ncores,
              "sample": f"each step: {nb_step} bands through {REF_SAMPLE_NOTE}; {ncores} threads"}
    else:
        with _oracle_pool(ncores) as pool:
            for w in range(args.warmup):
                _pool_sweep(pool, ncores, 1, 100_000 + w * ncores)
            wall = busy = 0.0
            for s in range(args.steps):
                dw, db = _pool_sweep(pool, ncores, bpc, s * ncores)
                wall += dw
                busy += db
        nb = args.steps * nb_step
        cb = {"kind": "port", "cores": ncores,
              "sample": f"each step: {ncores} processes x {bpc} single-band H*psi through the FP64 NumPy "
                        f"restatement of the reference path (oracle/pw.py), tables built once per process; "
                        f"{busy / nb * 1e3:.0f} ms per band per core"}
    v = nb / wall
    line = {"impl": "reference", "metric": "H*psi bands/s", "value": v, "unit": "bands/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "sample_bands_per_step": nb_step},
            "cpu_baseline": dict(value=v, unit="bands/s", **cb),
            "e2e": {"value": v, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    global NBAND
    NBAND = args.bands
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from pwdft_develop_b200 import Context
    from pwdft_develop_b200.core import KERNEL_KINDS

    prec = args.precision
    L, z, pos = si64_atoms()
    ctx = Context(L, NC, NF, precision=prec, device=local)
    ctx.set_vtot(synthetic_vtot(ctx.ntotFine))
    ctx.set_atoms(z, pos)
    ctx.set_band_batch(NBAND)
    if args.autotune:
        tune = ctx.autotune(NBAND)      # set-up (untimed): band batch and projector GEMM tiles
    else:
        tune = {"band_batch": NBAND, "gemm_bn": 0, "gemm_bn_store": 0, "fft_variant": args.fft_variant}
        ctx.set_fft_variant(args.fft_variant)
    dt_t = ctx.torch_dtype
    g = torch.Generator(device="cuda").manual_seed(SEED + rank)
    X = torch.randn((NBAND, ctx.ntot), dtype=torch.float64, device="cuda", generator=g)
    R = torch.linalg.cholesky(X @ X.T).T                     # Cholesky-QR (set-up, untimed)
    X = torch.linalg.solve_triangular(R, X, upper=True, left=True).contiguous()
    X = X.to(dt_t).contiguous()
    Y = torch.empty_like(X)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        ctx.hpsi(X, out=Y)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    l0 = ctx.launches()
    lc0 = ctx.library_calls()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        ctx.hpsi(X, out=Y)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
    launches = ctx.launches() - l0
    lib_calls = ctx.library_calls() - lc0
    ck = clocks.stop()
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * NBAND * args.steps / (total_ms / 1e3)

    # per-kernel device time (event-bracketed launches, same stream)
    ctx.profile(True)
    for _ in range(args.steps):
        flush.zero_()
        ctx.hpsi(X, out=Y)
    torch.cuda.synchronize()
    kern = {}
    for k in range(12):
        ms, n = ctx.profile_read(k)
        if n:
            kern[KERNEL_KINDS[k]] = {"launches": n, "avg_us": ms / n * 1e3, "total_ms": ms}
    ctx.profile(False)
    dom_name = max((k for k in kern if k != "library_gemm"), key=lambda k: kern[k]["total_ms"])
    dom_kind = [k for k, v in KERNEL_KINDS.items() if v == dom_name][0]
    s = 4 if prec == "f32" else 8
    npts_total = 0
    natom = len(pos)
    from pwdft_develop_b200.core import hgh_atom_projectors
    idx0, val0, _ = hgh_atom_projectors(L, NF, 14, pos[0])
    npts_total = sum(len(hgh_atom_projectors(L, NF, 14, p)[0]) for p in pos)
    # tile slots ~ atoms x fine planes they touch (exact count from the library is not exported)
    nslot_est = int(natom * (2 * 3.5 / (2 * A_CELL) * NF[2] + 1))
    alg = algorithmic_bytes(dom_kind, tune["band_batch"] // 2, s, npts_total, 5, nslot_est, natom)
    achieved = alg / (kern[dom_name]["avg_us"] * 1e-6) / 1e9
    peak, peak_kind = load_peaks()
    traffic = load_traffic(prec, dom_name, tune["band_batch"] // 2)
    model = hpsi_model_bytes_per_band(s, NBAND, 5 * natom, natom, npts_total)

    # end to end through the host C-ABI entry (pinned host buffers)
    Xh = X.cpu().pin_memory()
    Yh = torch.empty_like(Xh).pin_memory()
    import ctypes as C
    from pwdft_develop_b200._lib import check, lib
    for _ in range(max(1, args.warmup)):
        check(lib.pw_hpsi_host(ctx.handle, C.c_void_p(Xh.data_ptr()), ctx.ntot, C.c_void_p(Yh.data_ptr()),
                               ctx.ntot, NBAND, 0))
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        check(lib.pw_hpsi_host(ctx.handle, C.c_void_p(Xh.data_ptr()), ctx.ntot, C.c_void_p(Yh.data_ptr()),
                               ctx.ntot, NBAND, 0))
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    bytes_io = NBAND * ctx.ntot * s

    if rank == 0:
        line = {
            "metric": "H*psi bands/s", "value": value, "unit": "bands/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": prec, "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(NC), "fine_grid": list(NF), "bands": NBAND,
                       "nonlocal": "dense coarse-grid projector matrix (GEMM)",
                       "band_batch": tune["band_batch"], "gemm_tiles": [tune["gemm_bn"], tune["gemm_bn_store"]],
                       "fft_variant": tune.get("fft_variant", 0),
                       "l2": "flushed between steps (256 MB device write)",
                       "parallelism": f"band blocks, {world} replica(s)"},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "traffic_source": (f"profiles/hpsi_si64_{prec}_dram_traffic.md (ncu dram__bytes of a "
                                            f"separate capture, scaled to this batch; not measured in this run)"
                                            if traffic is not None else None),
                         "algorithmic_bytes_per_launch": alg, "avg_launch_us": kern[dom_name]["avg_us"]},
            "hpsi_model": {"bytes_per_band": model, "achieved_GBs": model * value / world / 1e9,
                           "frac": model * value / world / 1e9 / peak},
            "kernels": kern,
            "gpu_launches": launches,
            "library_calls": lib_calls,
            "e2e": {"value": world * NBAND * args.steps / (e2e_ms / 1e3), "unit": "bands/s",
                    "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
            "clocks": ck,
        }
        if prec == "f32" and args.f64_sweep and world == 1:
            line["f64_sweep"] = f64_sweep_bench(local, args.steps, args.warmup)
        if args.scf and world == 1:
            line["scf"] = scf_bench(local)
        if args.solvers and world == 1:
            line["solvers"] = solvers_bench(local)
        if args.dense and world == 1:
            line["dense"] = dense_bench(local)
        if args.exx and world == 1:
            line["exx"] = exx_bench(local)
            line["hybrid_scf"] = hybrid_bench(local)
        if args.kpoints and world == 1:
            line["kpoints"] = kpoint_bench(local)
        if args.gspace and world == 1:
            line["gspace"] = gspace_bench(local)
        if args.cells and world == 1:
            line["cells"] = cells_bench(local)
        if args.grams and world == 1:
            line["gram"] = gram_bench(local)
        if args.cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(args.cpu_bands)
        line["summary"] = summary(line)     # last key: the headline figures in one place
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-f64-sweep", dest="f64_sweep", action="store_false", help="skip the FP64 sweep leg")
    ap.add_argument("--no-scf", dest="scf", action="store_false", help="skip the SCF time-to-solution leg")
    ap.add_argument("--no-solvers", dest="solvers", action="store_false",
                    help="skip the LOBPCG / PPCG / Davidson SCF leg")
    ap.add_argument("--no-dense", dest="dense", action="store_false", help="skip the dense FP64 kernel leg")
    ap.add_argument("--no-exx", dest="exx", action="store_false", help="skip the hybrid-exchange leg")
    ap.add_argument("--no-kpoints", dest="kpoints", action="store_false", help="skip the k-point batch leg")
    ap.add_argument("--no-gspace", dest="gspace", action="store_false", help="skip the sphere-cut (G-space) leg")
    ap.add_argument("--no-cells", dest="cells", action="store_false", help="skip the uneven-cell batch leg")
    ap.add_argument("--no-grams", dest="grams", action="store_false", help="skip the eigensolver Gram leg")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="default band batch and GEMM tiles (profiling runs: no tuning launches in the list)")
    ap.add_argument("--cpu-bands", type=int, default=4, help="CPU baseline: bands per host core")
    ap.add_argument("--ref-bands-per-core", type=int, default=4, help="reference arm: bands per core per step")
    ap.add_argument("--bands", type=int, default=NBAND, help="band block size (profiling runs use a small block)")
    ap.add_argument("--fft-variant", type=int, default=2, choices=[0, 1, 2],
                    help="fine-plane transform form when the autotuner is off (pw_set_fft_variant)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
