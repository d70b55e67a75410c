"""Python host mirror of the reference's Fourier / Spinor / Hamiltonian entry
points for the real (Gamma-point) H*psi path, over the C ABI.

Device buffers are torch CUDA tensors of shape (nband, ntot) -- band-major
rows, i.e. the column-major ntot x nband layout of the reference's
NumTns<Real>(ntot, 1, nband) -- and are passed to the library as raw
pointers.  torch is used only for device memory and streams.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PW_F32, PW_F64, check, lib


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream(stream) -> C.c_void_p:
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Context:
    """One cell + grid + precision.  Mirrors ``Fourier::Initialize /
    InitializeFine`` (src/SCF/fourier.cpp:97-418) and the tables
    ``KohnSham`` owns (ekin_, teter_, vtot_, pseudo_)."""

    def __init__(self, length, numGrid, numGridFine, precision: str = "f64", device: int = 0):
        self.precision = precision
        prec = PW_F64 if precision == "f64" else PW_F32
        L = (C.c_double * 3)(*[float(x) for x in length])
        n = (C.c_int * 3)(*[int(x) for x in numGrid])
        nf = (C.c_int * 3)(*[int(x) for x in numGridFine])
        h = C.c_void_p()
        check(lib.pw_ctx_create(L, n, nf, prec, device, C.byref(h)))
        self._h = h
        nt, ntf = C.c_long(), C.c_long()
        check(lib.pw_ctx_sizes(h, C.byref(nt), C.byref(ntf)))
        self.ntot, self.ntotFine = nt.value, ntf.value
        self.numGrid = tuple(int(x) for x in numGrid)
        self.numGridFine = tuple(int(x) for x in numGridFine)
        self.length = tuple(float(x) for x in length)
        self.device = int(device)

    @classmethod
    def gspace(cls, length, numGrid, ecut: float, precision: str = "f64", device: int = 0) -> "Context":
        """Sphere-cut (G-space) context, the reference's ``Use_Real_Space: 0``
        mode (Fourier::Initialize with spherecut, src/SCF/fourier.cpp:542-640).
        ``numGrid`` is the G-space (= density) grid.  Bands are the half-sphere
        coefficients in idxCoarseCut order with the sqrt(2) convention, passed
        as real tensors of 2 ns numbers (see ``to_real`` / ``to_complex``)."""
        self = cls.__new__(cls)
        self.precision = precision
        prec = PW_F64 if precision == "f64" else PW_F32
        L = (C.c_double * 3)(*[float(x) for x in length])
        n = (C.c_int * 3)(*[int(x) for x in numGrid])
        h = C.c_void_p()
        check(lib.pw_ctx_create_gspace(L, n, float(ecut), prec, device, C.byref(h)))
        self._h = h
        nt, ntf = C.c_long(), C.c_long()
        check(lib.pw_ctx_sizes(h, C.byref(nt), C.byref(ntf)))
        self.ntot, self.ntotFine = nt.value, ntf.value
        self.numGrid = tuple(int(x) // 2 for x in numGrid)
        self.numGridFine = tuple(int(x) for x in numGrid)
        self.length = tuple(float(x) for x in length)
        self.device = int(device)
        self.ecut = float(ecut)
        self.ns = self.ntot // 2
        return self

    def gs_sphere(self):
        """(idxCoarseCut, Miller indices (ns, 3), ekin, teter) of a G-space context."""
        ns = C.c_int()
        check(lib.pw_gs_sphere(self._h, C.byref(ns), None, None, None, None))
        n = ns.value
        idx = np.zeros(n, np.int32)
        mil = np.zeros((n, 3), np.int32)
        ek = np.zeros(n)
        te = np.zeros(n)
        check(lib.pw_gs_sphere(self._h, C.byref(ns), idx.ctypes.data_as(_lib._ip), mil.ctypes.data_as(_lib._ip),
                               ek.ctypes.data_as(_lib._dp), te.ctypes.data_as(_lib._dp)))
        return idx, mil, ek, te

    def gs_set_projectors(self, vnlc: np.ndarray, wgt: np.ndarray):
        """vnlc (ns, nproj) complex, wgt (nproj): EigenSolver::NonlocalMultX's table."""
        v = np.asarray(vnlc, np.complex128)
        flat = np.ascontiguousarray(v.T).view(np.float64).ravel()     # column l: 2 ns interleaved doubles
        w = np.ascontiguousarray(wgt, np.float64)
        check(lib.pw_gs_set_projectors(self._h, v.shape[1], flat.ctypes.data_as(_lib._dp), w.ctypes.data_as(_lib._dp)))

    def gs_get_projectors(self):
        npj = C.c_int()
        check(lib.pw_gs_get_projectors(self._h, C.byref(npj), None, None))
        n = npj.value
        flat = np.zeros(n * self.ntot)
        w = np.zeros(n)
        if n:
            check(lib.pw_gs_get_projectors(self._h, C.byref(npj), flat.ctypes.data_as(_lib._dp),
                                           w.ctypes.data_as(_lib._dp)))
        return flat.view(np.complex128).reshape(n, -1).T, w

    @staticmethod
    def to_real(c):
        """(nb, ns) complex -> (nb, 2 ns) real view (numpy or torch)."""
        if hasattr(c, "is_cuda"):
            import torch
            return torch.view_as_real(c.contiguous()).reshape(c.shape[0], -1)
        return np.ascontiguousarray(c).view(np.float64 if c.dtype == np.complex128 else np.float32).reshape(
            c.shape[0], -1)

    @staticmethod
    def to_complex(x):
        """(nb, 2 ns) real -> (nb, ns) complex view (numpy or torch)."""
        if hasattr(x, "is_cuda"):
            import torch
            return torch.view_as_complex(x.contiguous().reshape(x.shape[0], -1, 2))
        return np.ascontiguousarray(x).view(np.complex128 if x.dtype == np.float64 else np.complex64).reshape(
            x.shape[0], -1)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib.pw_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def np_dtype(self):
        return np.float64 if self.precision == "f64" else np.float32

    @property
    def torch_dtype(self):
        import torch
        return torch.float64 if self.precision == "f64" else torch.float32

    # -- tables ---------------------------------------------------------
    def set_vtot(self, vtot: np.ndarray):
        v = np.ascontiguousarray(vtot, dtype=np.float64).ravel()
        if v.size != self.ntotFine:
            raise ValueError("vtot must have ntotFine entries")
        check(lib.pw_set_vtot(self._h, v.ctypes.data_as(_lib._dp)))

    def set_nonlocal(self, atoms):
        """atoms: list of (idx[npts], beta[nproj, npts], weight[nproj]) --
        one entry per atom, the flat form of PseudoPot::vnlList."""
        natom = len(atoms)
        npts = np.array([len(a[0]) for a in atoms], dtype=np.int32)
        nproj = np.array([len(a[2]) for a in atoms], dtype=np.int32)
        idx = np.ascontiguousarray(np.concatenate([np.asarray(a[0], np.int32) for a in atoms])
                                   if natom else np.zeros(0, np.int32))
        beta = np.ascontiguousarray(np.concatenate([np.asarray(a[1], np.float64).ravel() for a in atoms])
                                    if natom else np.zeros(0))
        wgt = np.ascontiguousarray(np.concatenate([np.asarray(a[2], np.float64) for a in atoms])
                                   if natom else np.zeros(0))
        check(lib.pw_set_nonlocal(self._h, natom, npts.ctypes.data_as(_lib._ip), nproj.ctypes.data_as(_lib._ip),
                                  idx.ctypes.data_as(_lib._ip), beta.ctypes.data_as(_lib._dp),
                                  wgt.ctypes.data_as(_lib._dp)))

    def set_band_batch(self, nb: int):
        check(lib.pw_set_band_batch(self._h, int(nb)))

    # -- operators ------------------------------------------------------
    def hpsi(self, psi, out=None, accumulate: bool = False, stream=None):
        """Spinor::AddMultSpinorFineR2C / KohnSham::MultSpinor on device
        tensors of shape (nband, ntot)."""
        import torch
        assert psi.is_cuda and psi.dtype == self.torch_dtype and psi.is_contiguous()
        nb = psi.shape[0]
        if out is None:
            out = torch.empty_like(psi)
            accumulate = False
        check(lib.pw_hpsi(self._h, _ptr(psi), self.ntot, _ptr(out), self.ntot, nb, int(accumulate), _stream(stream)))
        return out

    def hpsi_host(self, psi: np.ndarray, out: np.ndarray | None = None, accumulate: bool = False):
        psi = np.ascontiguousarray(psi, dtype=self.np_dtype)
        nb = psi.shape[0]
        if out is None:
            out = np.zeros_like(psi)
            accumulate = False
        check(lib.pw_hpsi_host(self._h, psi.ctypes.data_as(C.c_void_p), self.ntot,
                               out.ctypes.data_as(C.c_void_p), self.ntot, nb, int(accumulate)))
        return out

    def teter(self, r, out=None, accumulate: bool = False, stream=None):
        """Spinor::AddTeterPrecond on device tensors (nband, ntot)."""
        import torch
        assert r.is_cuda and r.dtype == self.torch_dtype and r.is_contiguous()
        nb = r.shape[0]
        if out is None:
            out = torch.empty_like(r)
            accumulate = False
        check(lib.pw_teter_precond(self._h, _ptr(r), self.ntot, _ptr(out), self.ntot, nb, int(accumulate),
                                   _stream(stream)))
        return out


# ---------------------------------------------------------------------------
# set-up helpers over the library's own HGH tables
# ---------------------------------------------------------------------------
def hgh_species(znuc: int) -> dict:
    zion, eself, rnl, rrho = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    npj = C.c_int()
    check(lib.pw_hgh_species(int(znuc), C.byref(zion), C.byref(eself), C.byref(rnl), C.byref(rrho), C.byref(npj)))
    return dict(zion=zion.value, eself=eself.value, rcut_nonlocal=rnl.value, rcut_rho=rrho.value, nproj=npj.value)


def hgh_atom_projectors(length, numGridFine, znuc: int, pos):
    """Host-only projector set of one atom: (idx, val4[nproj, npts, 4], wgt)."""
    L = (C.c_double * 3)(*[float(x) for x in length])
    nf = (C.c_int * 3)(*[int(x) for x in numGridFine])
    p = (C.c_double * 3)(*[float(x) for x in pos])
    npts, nproj = C.c_int(), C.c_int()
    check(lib.pw_hgh_atom_projectors(L, nf, int(znuc), p, C.byref(npts), C.byref(nproj), None, None, None))
    idx = np.zeros(npts.value, np.int32)
    val = np.zeros((nproj.value, npts.value, 4))
    wgt = np.zeros(nproj.value)
    check(lib.pw_hgh_atom_projectors(L, nf, int(znuc), p, None, None, idx.ctypes.data_as(_lib._ip),
                                     val.ctypes.data_as(_lib._dp), wgt.ctypes.data_as(_lib._dp)))
    return idx, val, wgt


def hgh_pseudocharge(length, numGridFine, znuc, pos) -> np.ndarray:
    L = (C.c_double * 3)(*[float(x) for x in length])
    nf = (C.c_int * 3)(*[int(x) for x in numGridFine])
    z = np.ascontiguousarray(znuc, np.int32)
    ps = np.ascontiguousarray(pos, np.float64)
    out = np.zeros(int(np.prod(numGridFine)))
    check(lib.pw_hgh_pseudocharge(L, nf, len(z), z.ctypes.data_as(_lib._ip), ps.ctypes.data_as(_lib._dp),
                                  out.ctypes.data_as(_lib._dp)))
    return out


def _ctx_set_atoms(self, znuc, pos):
    z = np.ascontiguousarray(znuc, np.int32)
    ps = np.ascontiguousarray(pos, np.float64)
    check(lib.pw_set_atoms(self._h, len(z), z.ctypes.data_as(_lib._ip), ps.ctypes.data_as(_lib._dp)))
    self._atoms_z = z.copy()


def _ctx_pseudocharge(self) -> np.ndarray:
    out = np.zeros(self.ntotFine)
    check(lib.pw_get_pseudocharge(self._h, out.ctypes.data_as(_lib._dp)))
    return out


def _ctx_launches(self) -> int:
    n, m = C.c_long(), C.c_long()
    check(lib.pw_stats(self._h, C.byref(n), C.byref(m)))
    return n.value


def _ctx_library_calls(self) -> int:
    n, m = C.c_long(), C.c_long()
    check(lib.pw_stats(self._h, C.byref(n), C.byref(m)))
    return m.value


def _ctx_set_nonlocal_mode(self, mode: str):
    check(lib.pw_set_nonlocal_mode(self._h, _lib.PW_NL_DENSE if mode == "dense" else _lib.PW_NL_REALSPACE))


def _ctx_profile(self, enable: bool):
    check(lib.pw_profile(self._h, int(enable)))


def _ctx_profile_read(self, kind: int):
    t, n = C.c_double(), C.c_long()
    check(lib.pw_profile_read(self._h, int(kind), C.byref(t), C.byref(n)))
    return t.value, n.value


def _ctx_gram(self, X, Y=None, stream=None):
    """G = X^T Y (X, Y: (n, ntot) device tensors) as an (nx, ny) FP64 tensor."""
    import torch
    Y = X if Y is None else Y
    G = torch.empty((Y.shape[0], X.shape[0]), dtype=torch.float64, device=X.device)   # column-major nx x ny
    check(lib.pw_gram(self._h, _ptr(X), self.ntot, X.shape[0], _ptr(Y), self.ntot, Y.shape[0], _ptr(G),
                      X.shape[0], _stream(stream)))
    return G.T


def _ctx_set_gemm_mode(self, mode: str = "tc", terms: int = 3):
    """Split-BF16 tensor-core GEMMs with 3 or 4 products per k-step ("tc" is
    the only engine)."""
    if mode != "tc":
        raise ValueError("the split-BF16 tensor-core GEMM is the only engine")
    check(lib.pw_set_gemm_mode(self._h, 0, int(terms)))


def _ctx_set_nl_overlap(self, on: bool = True):
    """Dense projector mode: the projector GEMMs of an H*psi batch on a
    second stream alongside the FFT chain (default on)."""
    check(lib.pw_set_nl_overlap(self._h, int(bool(on))))


def _ctx_set_check_errors(self, on: bool = True):
    check(lib.pw_set_check_errors(self._h, int(on)))


Context.gram = _ctx_gram
Context.set_gemm_mode = _ctx_set_gemm_mode
Context.set_check_errors = _ctx_set_check_errors
Context.set_nl_overlap = _ctx_set_nl_overlap
Context.set_atoms = _ctx_set_atoms
Context.pseudocharge = _ctx_pseudocharge
Context.launches = _ctx_launches
Context.library_calls = _ctx_library_calls
Context.set_nonlocal_mode = _ctx_set_nonlocal_mode
Context.profile = _ctx_profile
Context.profile_read = _ctx_profile_read

KERNEL_KINDS = {0: "coarse_xy_fwd", 1: "z_pad", 2: "fine_plane_gather", 3: "nl_reduce", 4: "fine_plane_apply",
                5: "z_fold", 6: "coarse_xy_inv", 7: "z_teter", 8: "gram", 9: "density", 10: "other",
                11: "library_gemm", 12: "exchange", 13: "rotation"}


# ---------------------------------------------------------------------------
# eigensolvers and SCF
# ---------------------------------------------------------------------------
def _ctx_cholqr(self, X):
    check(lib.pw_cholqr(self._h, _ptr(X), X.shape[0]))
    return X


_SOLVERS = {"lobpcg": _lib.PW_SOLVER_LOBPCG, "chebfsi": _lib.PW_SOLVER_CHEBFSI, "ppcg": _lib.PW_SOLVER_PPCG,
            "davidson": _lib.PW_SOLVER_DAVIDSON}


def _ctx_eigsolve(self, X, solver: str = "lobpcg", maxit: int = 10, tol: float = 1e-8, degree: int = 10):
    """EigenSolver::LOBPCGSolveReal / PPCGSolveReal / DavidsonSolveReal / ChebFSI
    on the device block X (nb, ntot), overwritten by the Ritz vectors.  degree:
    ChebFSI filter degree, PPCG sub-block size or Davidson subspace blocks.
    Returns (eig, resnorm, iterations)."""
    nb = X.shape[0]
    eig = np.zeros(nb)
    res = np.zeros(nb)
    it = C.c_int()
    sid = _SOLVERS[solver]
    check(lib.pw_eigsolve(self._h, sid, _ptr(X), nb, int(maxit), float(tol), int(degree),
                          eig.ctypes.data_as(_lib._dp), res.ctypes.data_as(_lib._dp), C.byref(it)))
    return eig, res, it.value


def _ctx_density(self, psi, occ, nocc_total: int):
    import torch
    rho = torch.empty(self.ntotFine, dtype=torch.float64, device=psi.device)
    occ = np.ascontiguousarray(occ, np.float64)
    check(lib.pw_density(self._h, _ptr(psi), self.ntot, psi.shape[0], occ.ctypes.data_as(_lib._dp),
                         int(nocc_total), _ptr(rho)))
    return rho


def _ctx_scf(self, nocc: int, nextra: int, ecut: float, solver: str = "chebfsi", mixed: bool = False,
             temperature: float = 300.0, cheby_degree: int = 10, cheby_first_cycles: int = 5,
             eig_max_iter: int = 3, eig_tol: float = 1e-10, max_iter: int = 100, mix_dim: int = 8,
             mix_step: float = 0.7, tol_efree: float = 1e-6, refine_threshold: float = 1e-4, seed: int = 1,
             verbose: bool = False, ppcg_sbsize: int = 1, davidson_maxdim: int = 2, graphs: bool = False,
             xc: str = "teter93", mix: str = "anderson", tol_rho: float = 0.0, phi_max_iter: int = 10,
             phi_tol: float = 1e-6, wfn_filter: bool | None = None, smearing: str = "FD"):
    """SCF::Iterate on the device (FP64 context; mixed=True runs the eigensolver in
    an FP32 twin and refines in FP64).  xc: "teter93", "pbe" or "hse06" (nested
    hybrid scheme with ACE).  wfn_filter: ChebFSI's wavefunction cut-off filter
    at ecut (None or True: on, the reference's CheFSI default; False: off).
    smearing: the reference's Smearing_Scheme, "FD" (Fermi-Dirac) or "GB"
    (Gaussian).  Returns (result dict, eigenvalues, rho)."""
    xcs = {"teter93": _lib.PW_XC_TETER93, "pbe": _lib.PW_XC_PBE, "hse06": _lib.PW_XC_HSE06}
    if xc not in xcs:
        raise ValueError(f"unknown exchange-correlation functional {xc!r}")
    if smearing not in ("FD", "GB"):
        raise ValueError(f"unknown smearing scheme {smearing!r}")
    p = _lib.ScfParams(nocc=nocc, nextra=nextra,
                       solver=_SOLVERS[solver], ppcg_sbsize=ppcg_sbsize, davidson_maxdim=davidson_maxdim,
                       graphs=int(graphs), xc=xcs[xc],
                       mix_type=_lib.PW_MIX_BROYDEN if mix == "broyden" else _lib.PW_MIX_ANDERSON,
                       tol_rho=float(tol_rho), phi_max_iter=int(phi_max_iter), phi_tol=float(phi_tol),
                       cheby_degree=cheby_degree, cheby_first_cycles=cheby_first_cycles, eig_max_iter=eig_max_iter,
                       max_iter=max_iter, mix_dim=mix_dim, mixed=int(mixed), verbose=int(verbose), ecut=ecut,
                       temperature=temperature, eig_tol=eig_tol, mix_step=mix_step, tol_efree=tol_efree,
                       refine_threshold=refine_threshold, seed=seed, no_wfn_filter=int(wfn_filter is False),
                       smearing=int(smearing == "GB"))
    r = _lib.ScfResult()
    eig = np.zeros(nocc + nextra)
    rho = np.zeros(self.ntotFine)
    check(lib.pw_scf_run(self._h, C.byref(p), C.byref(r), eig.ctypes.data_as(_lib._dp), rho.ctypes.data_as(_lib._dp)))
    res = {k: getattr(r, k) for k, _ in r._fields_}
    res["phase_s"] = list(r.phase_s)
    res["sub_s"] = list(r.sub_s)
    return res, eig, rho


def _ctx_set_wfn_filter(self, ecut: float | None):
    """KohnSham::MultSpinor's wavefunction cut-off filter: an overwriting hpsi
    returns P H psi (P zeroes the coefficients with |G|^2/2 > ecut); None
    switches it off."""
    check(lib.pw_set_wfn_filter(self._h, 0 if ecut is None else 1, 0.0 if ecut is None else float(ecut)))


def _ctx_wfn_filter(self, X, stream=None):
    """X <- P X in place (the filter's first-call step on psi)."""
    check(lib.pw_wfn_filter(self._h, _ptr(X), self.ntot, X.shape[0], _stream(stream)))
    return X


Context.set_wfn_filter = _ctx_set_wfn_filter
Context.wfn_filter = _ctx_wfn_filter


def _ctx_xc_pbe(self, rho, ecut: float):
    """PBE (eps per particle, V_xc) of a fine-grid density (float64 device tensors)."""
    import torch
    eps = torch.empty_like(rho)
    vxc = torch.empty_like(rho)
    check(lib.pw_xc_pbe(self._h, _ptr(rho), float(ecut), _ptr(eps), _ptr(vxc)))
    return eps, vxc


Context.xc_pbe = _ctx_xc_pbe


def _ctx_xc_hse06(self, rho, ecut: float):
    """Semilocal HSE06 (eps per particle, V_xc) of a fine-grid density: PBE minus
    0.25 times the omega = 0.106 short-range PBE exchange (float64 device tensors)."""
    import torch
    eps = torch.empty_like(rho)
    vxc = torch.empty_like(rho)
    check(lib.pw_xc_hse06(self._h, _ptr(rho), float(ecut), _ptr(eps), _ptr(vxc)))
    return eps, vxc


Context.xc_hse06 = _ctx_xc_hse06


def _ctx_build_twin(self):
    check(lib.pw_ctx_build_twin(self._h))


def _ctx_hartree(self, drho, ecut: float):
    import torch
    vh = torch.empty_like(drho)
    check(lib.pw_hartree(self._h, _ptr(drho), float(ecut), _ptr(vh)))
    return vh


def _ctx_xc(self, rho):
    import torch
    eps, v = torch.empty_like(rho), torch.empty_like(rho)
    check(lib.pw_xc_teter93(self._h, _ptr(rho), _ptr(eps), _ptr(v)))
    return eps, v


def _ctx_forces(self, rho, psi, occ, num_spin: int = 2):
    """KohnSham::CalculateForce (hamiltonian.cpp:2670-3056) for an FP64 context with
    atoms: rho (N_fine) and psi (nband, N_coarse) float64 device tensors, occ the
    occupation rates.  Returns (total, local, nonlocal), each natom x 3."""
    if not hasattr(self, "_atoms_z"):
        raise RuntimeError("atoms not set (set_atoms)")
    natom = len(self._atoms_z)
    occ = np.ascontiguousarray(occ, np.float64)
    nb = 0 if psi is None else psi.shape[0]
    out = [np.zeros((natom, 3)) for _ in range(3)]
    check(lib.pw_forces(self._h, _ptr(rho), _ptr(psi) if nb else None, self.ntot, nb,
                        occ.ctypes.data_as(_lib._dp), int(num_spin), *[o.ctypes.data_as(_lib._dp) for o in out]))
    return tuple(out)


def _ctx_scf_forces(self):
    """Forces from the final state of the last scf() call: (total, local, nonlocal)."""
    natom = len(self._atoms_z)
    out = [np.zeros((natom, 3)) for _ in range(3)]
    check(lib.pw_scf_forces(self._h, *[o.ctypes.data_as(_lib._dp) for o in out]))
    return tuple(out)


def _ctx_band_energy(self, psi, w):
    """E = sum_b w_b <psi_b, H psi_b> (psi: (nband, N_coarse) device tensor)."""
    w = np.ascontiguousarray(w, np.float64)
    e = C.c_double(0.0)
    check(lib.pw_band_energy(self._h, _ptr(psi), self.ntot, psi.shape[0], w.ctypes.data_as(_lib._dp), C.byref(e)))
    return e.value


def _ctx_band_energy_backward(self, psi, w, dv: bool = True, dr: bool = True):
    """(dE/dV_loc on the fine grid as a float64 device tensor or None,
    dE/dR natom x 3 numpy array or None) at fixed psi."""
    import torch
    w = np.ascontiguousarray(w, np.float64)
    g = torch.empty(self.ntotFine, dtype=torch.float64, device=psi.device) if dv else None
    r = np.zeros((len(self._atoms_z), 3)) if dr else None
    check(lib.pw_band_energy_backward(self._h, _ptr(psi), self.ntot, psi.shape[0], w.ctypes.data_as(_lib._dp),
                                      _ptr(g) if dv else None, r.ctypes.data_as(_lib._dp) if dr else None))
    return g, r


def _ctx_scf_state(self):
    """(occupations, bands (nband, N_coarse) float64 device tensor, density) of the last scf()."""
    import torch
    nb = C.c_int(0)
    check(lib.pw_scf_state(self._h, C.byref(nb), None, None, 0, None))
    occ = np.zeros(nb.value)
    psi = torch.empty((nb.value, self.ntot), dtype=torch.float64, device="cuda")
    rho = torch.empty(self.ntotFine, dtype=torch.float64, device="cuda")
    check(lib.pw_scf_state(self._h, C.byref(nb), occ.ctypes.data_as(_lib._dp), _ptr(psi), self.ntot, _ptr(rho)))
    return occ, psi, rho


def _ctx_exx_setup(self, fraction: float = 0.25, screen_mu: float = 0.0, divergence_type: int = 1,
                   ecut: float = 10.0):
    """InitializeEXX: Coulomb kernel (PBE0: fraction 0.25, mu 0)."""
    check(lib.pw_exx_setup(self._h, float(fraction), float(screen_mu), int(divergence_type), float(ecut)))


def _ctx_exx_kernel(self):
    """(exxDiv, kernel on the full coarse spectrum as an (n2, n1, n0) array;
    G-space contexts: on the full G-space grid, zero outside the Fock set)."""
    d = C.c_double(0.0)
    gs = getattr(self, "ns", None) is not None
    grid = self.numGridFine if gs else self.numGrid
    k = np.zeros(int(np.prod(grid)))
    check(lib.pw_exx_get(self._h, C.byref(d), k.ctypes.data_as(_lib._dp)))
    return d.value, k.reshape(grid[2], grid[1], grid[0])


def _ctx_exx_set_phi(self, psi, occ):
    occ = np.ascontiguousarray(occ, np.float64)
    check(lib.pw_exx_set_phi(self._h, _ptr(psi), self.ntot, psi.shape[0], occ.ctypes.data_as(_lib._dp)))


def _ctx_exx_set_mode(self, mode: str):
    m = {"off": _lib.PW_EXX_OFF, "full": _lib.PW_EXX_FULL, "ace": _lib.PW_EXX_ACE}[mode]
    check(lib.pw_exx_set_mode(self._h, m))


def _ctx_exx_apply(self, psi, out=None, accumulate: bool = False, stream=None):
    import torch
    if out is None:
        out = torch.zeros_like(psi)
    check(lib.pw_exx_apply(self._h, _ptr(psi), self.ntot, _ptr(out), self.ntot, psi.shape[0], int(accumulate),
                           _stream(stream)))
    return out


def _ctx_ace_build(self, psi):
    check(lib.pw_ace_build(self._h, _ptr(psi), self.ntot, psi.shape[0]))


def _ctx_ace_apply(self, psi, out=None, stream=None):
    import torch
    if out is None:
        out = torch.zeros_like(psi)
    check(lib.pw_ace_apply(self._h, _ptr(psi), self.ntot, _ptr(out), self.ntot, psi.shape[0], _stream(stream)))
    return out


def _ctx_exx_energy(self, psi, occ, num_spin: int = 2, use_ace: bool = False) -> float:
    occ = np.ascontiguousarray(occ, np.float64)
    e = C.c_double(0.0)
    check(lib.pw_exx_energy(self._h, _ptr(psi), self.ntot, psi.shape[0], occ.ctypes.data_as(_lib._dp),
                            int(num_spin), int(use_ace), C.byref(e)))
    return e.value


def _ctx_set_kpoint(self, k):
    """Bloch vector k (Cartesian, 1/bohr) for pw_hpsi_k."""
    kk = np.ascontiguousarray(k, np.float64)
    check(lib.pw_set_kpoint(self._h, kk.ctypes.data_as(_lib._dp)))


def _ctx_hpsi_k(self, psi, out=None, accumulate: bool = False, stream=None):
    """H(k) psi for complex bands psi (nband, N_coarse) complex128 / complex64 device tensor."""
    import torch
    if out is None:
        out = torch.zeros_like(psi)
    check(lib.pw_hpsi_k(self._h, _ptr(psi), self.ntot, _ptr(out), self.ntot, psi.shape[0], int(accumulate),
                        _stream(stream)))
    return out


def _ctx_kpoint_tables(self):
    ek = np.zeros(self.ntot)
    te = np.zeros(self.ntot)
    check(lib.pw_get_kpoint_tables(self._h, ek.ctypes.data_as(_lib._dp), te.ctypes.data_as(_lib._dp)))
    return ek, te


def _ctx_set_kpoints(self, kpts):
    """A resident batch of Bloch vectors (nk x 3, Cartesian 1/bohr) for hpsi_kbatch."""
    kk = np.ascontiguousarray(kpts, np.float64).reshape(-1, 3)
    check(lib.pw_set_kpoints(self._h, kk.shape[0], kk.ctypes.data_as(_lib._dp)))
    self._nkb = kk.shape[0]


def _ctx_hpsi_kbatch(self, psi, out=None, accumulate: bool = False, stream=None):
    """H(k_i) psi_i for psi of shape (nk, nband, N_coarse) complex on the device."""
    import torch
    if out is None:
        out = torch.zeros_like(psi)
    nb = psi.shape[1]
    check(lib.pw_hpsi_kbatch(self._h, _ptr(psi), self.ntot, _ptr(out), self.ntot, nb, int(accumulate),
                             _stream(stream)))
    return out


class HpsiGraph:
    """A captured pw_hpsi call: replay() applies H to the same buffers again."""

    def __init__(self, ctx, psi, out, accumulate: bool = False):
        self._ctx = ctx
        self._keep = (psi, out)
        h = C.c_void_p()
        check(lib.pw_graph_capture_hpsi(ctx._h, _ptr(psi), ctx.ntot, _ptr(out), ctx.ntot, psi.shape[0],
                                        int(accumulate), C.byref(h)))
        self._g = h

    @property
    def nodes(self) -> int:
        n = C.c_long(0)
        check(lib.pw_graph_nodes(self._g, C.byref(n)))
        return n.value

    def replay(self, stream=None):
        check(lib.pw_graph_launch(self._g, _stream(stream)))

    def close(self):
        if getattr(self, "_g", None):
            lib.pw_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        self.close()


class CellBatch:
    """Independent contexts applied together: hpsi() runs every cell's H*psi
    on forked streams (pw_hpsi_batch); capture() records the whole batch as
    one CUDA graph and returns an object whose replay() launches it."""

    def __init__(self, ctxs, psis, outs):
        n = len(ctxs)
        self._keep = (list(ctxs), list(psis), list(outs))
        self._n = n
        self._c = (C.c_void_p * n)(*[c._h for c in ctxs])
        self._p = (C.c_void_p * n)(*[p.data_ptr() for p in psis])
        self._o = (C.c_void_p * n)(*[o.data_ptr() for o in outs])
        self._ld = (C.c_int * n)(*[c.ntot for c in ctxs])
        self._nb = (C.c_int * n)(*[p.shape[0] for p in psis])

    def hpsi(self, stream=None):
        check(lib.pw_hpsi_batch(self._n, self._c, self._p, self._ld, self._o, self._ld, self._nb, _stream(stream)))

    def capture(self):
        h = C.c_void_p()
        check(lib.pw_graph_capture_batch(self._n, self._c, self._p, self._ld, self._o, self._ld, self._nb,
                                         C.byref(h)))
        g = HpsiGraph.__new__(HpsiGraph)
        g._ctx, g._keep, g._g = None, self._keep, h
        return g


def _ctx_capture_hpsi(self, psi, out, accumulate: bool = False) -> HpsiGraph:
    return HpsiGraph(self, psi, out, accumulate)


def _ctx_autotune(self, nband: int) -> dict:
    """pw_autotune: pick band-batch width, fine-plane FFT radix decomposition
    and projector GEMM tiles by timing."""
    r = _lib.TuneResult()
    check(lib.pw_autotune(self._h, int(nband), C.byref(r)))
    return {k: getattr(r, k) for k, _ in r._fields_}


def _ctx_set_fft_variant(self, variant: int):
    """Radix decomposition of the fused fine-plane transforms (0 default, 1 second)."""
    check(lib.pw_set_fft_variant(self._h, int(variant)))


Context.set_fft_variant = _ctx_set_fft_variant


Context.autotune = _ctx_autotune
Context.capture_hpsi = _ctx_capture_hpsi
Context.set_kpoints = _ctx_set_kpoints
Context.hpsi_kbatch = _ctx_hpsi_kbatch
Context.set_kpoint = _ctx_set_kpoint
Context.hpsi_k = _ctx_hpsi_k
Context.kpoint_tables = _ctx_kpoint_tables
Context.exx_setup = _ctx_exx_setup
Context.exx_kernel = _ctx_exx_kernel
Context.exx_set_phi = _ctx_exx_set_phi
Context.exx_set_mode = _ctx_exx_set_mode
Context.exx_apply = _ctx_exx_apply
Context.ace_build = _ctx_ace_build
Context.ace_apply = _ctx_ace_apply
Context.exx_energy = _ctx_exx_energy
Context.scf_state = _ctx_scf_state
Context.band_energy = _ctx_band_energy
Context.band_energy_backward = _ctx_band_energy_backward
Context.forces = _ctx_forces
Context.scf_forces = _ctx_scf_forces
Context.hartree = _ctx_hartree
Context.xc = _ctx_xc
Context.cholqr = _ctx_cholqr
Context.eigsolve = _ctx_eigsolve
Context.density = _ctx_density
Context.scf = _ctx_scf
Context.build_twin = _ctx_build_twin


# ---------------------------------------------------------------------------
# restart files (DEN, POT, WFN_<rank>, EIG) in the reference's binary layout
# ---------------------------------------------------------------------------
def _ctx_write_density(self, path, rho):
    r = np.ascontiguousarray(rho, np.float64).ravel()
    assert r.size == self.ntotFine
    check(lib.pw_write_density(self._h, str(path).encode(), r.ctypes.data_as(_lib._dp)))


def _ctx_read_density(self, path) -> np.ndarray:
    out = np.zeros(self.ntotFine)
    check(lib.pw_read_density(self._h, str(path).encode(), out.ctypes.data_as(_lib._dp)))
    return out


def _ctx_write_potential(self, path, vtot):
    v = np.ascontiguousarray(vtot, np.float64).ravel()
    assert v.size == self.ntotFine
    check(lib.pw_write_potential(self._h, str(path).encode(), v.ctypes.data_as(_lib._dp)))


def _ctx_write_wfn(self, path, psi, occ):
    """psi: (nband, ntot) host array (each row one band), occ: (nband,)."""
    x = np.ascontiguousarray(psi, np.float64)
    o = np.ascontiguousarray(occ, np.float64)
    check(lib.pw_write_wfn(self._h, str(path).encode(), x.ctypes.data_as(_lib._dp), self.ntot, x.shape[0],
                           o.ctypes.data_as(_lib._dp)))


def _ctx_read_wfn(self, path):
    nb = C.c_int(0)
    check(lib.pw_read_wfn(self._h, str(path).encode(), None, self.ntot, 0, C.byref(nb), None))
    x = np.zeros((nb.value, self.ntot))
    o = np.zeros(nb.value)
    check(lib.pw_read_wfn(self._h, str(path).encode(), x.ctypes.data_as(_lib._dp), self.ntot, nb.value,
                          C.byref(nb), o.ctypes.data_as(_lib._dp)))
    return x, o


def write_eig(path, eig):
    e = np.ascontiguousarray(eig, np.float64)
    check(lib.pw_write_eig(str(path).encode(), e.size, e.ctypes.data_as(_lib._dp)))


def read_eig(path) -> np.ndarray:
    n = C.c_int(0)
    check(lib.pw_read_eig(str(path).encode(), 0, C.byref(n), None))
    e = np.zeros(n.value)
    check(lib.pw_read_eig(str(path).encode(), n.value, C.byref(n), e.ctypes.data_as(_lib._dp)))
    return e


def _ctx_scf_set_initial(self, rho=None, psi=None):
    """Starting density (N_fine) and/or bands (nband, ntot) for the next scf()."""
    r = None if rho is None else np.ascontiguousarray(rho, np.float64).ravel()
    x = None if psi is None else np.ascontiguousarray(psi, np.float64)
    check(lib.pw_scf_set_initial(self._h, None if r is None else r.ctypes.data_as(_lib._dp),
                                 None if x is None else x.ctypes.data_as(_lib._dp), self.ntot,
                                 0 if x is None else x.shape[0]))


Context.write_density = _ctx_write_density
Context.read_density = _ctx_read_density
Context.write_potential = _ctx_write_potential
Context.write_wfn = _ctx_write_wfn
Context.read_wfn = _ctx_read_wfn
Context.scf_set_initial = _ctx_scf_set_initial
