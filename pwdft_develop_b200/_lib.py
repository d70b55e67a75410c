"""ctypes binding of ``libpwdft_b200.so`` (the C ABI in include/pwdft_b200.h).

The library is required: importing this module raises if the shared object
is missing, and every call that returns a non-zero status raises
``PwError`` with the library's message.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpwdft_b200.so"

PW_OK, PW_EINVAL, PW_ECUDA, PW_ENOMEM, PW_EUNSUPPORTED, PW_ETIMEOUT, PW_ENOTREADY, PW_ENUMERIC = \
    0, -1, -2, -3, -4, -5, -6, -7
PW_F64, PW_F32 = 0, 1
PW_NL_DENSE, PW_NL_REALSPACE = 0, 1


class PwError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pwdft_b200 error {code}: {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() or python pwdft_develop_b200/build.py (nvcc, sm_100a)")
    return C.CDLL(str(LIB_PATH))


lib = _load()

_vp, _i, _l, _d = C.c_void_p, C.c_int, C.c_long, C.c_double
_ip, _dp = C.POINTER(C.c_int), C.POINTER(C.c_double)

PW_EXX_OFF, PW_EXX_FULL, PW_EXX_ACE = 0, 1, 2
PW_SOLVER_LOBPCG, PW_SOLVER_CHEBFSI, PW_SOLVER_PPCG, PW_SOLVER_DAVIDSON = 0, 1, 2, 3
PW_XC_TETER93, PW_XC_PBE, PW_XC_HSE06 = 0, 1, 2
PW_MIX_ANDERSON, PW_MIX_BROYDEN = 0, 1


class ScfParams(C.Structure):
    _fields_ = [("nocc", C.c_int), ("nextra", C.c_int), ("solver", C.c_int), ("cheby_degree", C.c_int),
                ("cheby_first_cycles", C.c_int), ("eig_max_iter", C.c_int), ("max_iter", C.c_int),
                ("mix_dim", C.c_int), ("mixed", C.c_int), ("verbose", C.c_int),
                ("ecut", C.c_double), ("temperature", C.c_double), ("eig_tol", C.c_double),
                ("mix_step", C.c_double), ("tol_efree", C.c_double), ("refine_threshold", C.c_double),
                ("seed", C.c_ulonglong), ("ppcg_sbsize", C.c_int), ("davidson_maxdim", C.c_int),
                ("graphs", C.c_int), ("xc", C.c_int), ("mix_type", C.c_int), ("tol_rho", C.c_double),
                ("phi_max_iter", C.c_int), ("phi_tol", C.c_double), ("no_wfn_filter", C.c_int),
                ("smearing", C.c_int)]


class ScfResult(C.Structure):
    _fields_ = [("etot", C.c_double), ("efree", C.c_double), ("eharris", C.c_double), ("exc", C.c_double),
                ("ehart", C.c_double), ("eself", C.c_double), ("fermi", C.c_double), ("time_s", C.c_double),
                ("iterations", C.c_int), ("converged", C.c_int), ("refine_iter", C.c_int),
                ("hpsi_bands", C.c_long), ("phase_s", C.c_double * 6),
                ("sub_s", C.c_double * 4), ("scf_norm", C.c_double), ("efock", C.c_double), ("dexx", C.c_double),
                ("phi_iterations", C.c_int)]


class TuneResult(C.Structure):
    _fields_ = [("band_batch", C.c_int), ("gemm_bn", C.c_int), ("gemm_bn_store", C.c_int), ("tried", C.c_int),
                ("cached", C.c_int), ("ms_default", C.c_double), ("ms_best", C.c_double), ("fft_variant", C.c_int)]


# name -> (restype, argtypes); every name here is declared in include/pwdft_b200.h
SIGNATURES: dict[str, tuple] = {
    "pw_last_error": (C.c_char_p, []),
    "pw_version": (C.c_char_p, []),
    "pw_ctx_create": (_i, [_dp, _ip, _ip, _i, _i, C.POINTER(_vp)]),
    "pw_ctx_destroy": (_i, [_vp]),
    "pw_ctx_sizes": (_i, [_vp, C.POINTER(_l), C.POINTER(_l)]),
    "pw_set_vtot": (_i, [_vp, _dp]),
    "pw_set_nonlocal": (_i, [_vp, _i, _ip, _ip, _ip, _dp, _dp]),
    "pw_hpsi": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_hpsi_host": (_i, [_vp, _vp, _i, _vp, _i, _i, _i]),
    "pw_set_host_chunk": (_i, [_vp, C.c_int]),
    "pw_teter_precond": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_teter_precond_noalloc": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_set_wfn_filter": (_i, [_vp, _i, C.c_double]),
    "pw_set_wait_limit": (_i, [_vp, C.c_double]),
    "pw_set_nl_overlap": (_i, [_vp, _i]),
    "pw_set_fft_variant": (_i, [_vp, _i]),
    "pw_dense_potrf": (_i, [_vp, _i, _vp, _i]),
    "pw_rotate": (_i, [_vp, _vp, _i, _i, _vp, _i, _i, _vp, _i, _i, _vp]),
    "pw_gram_rows": (_i, [_vp, _i, _vp, _i, _i, _vp, _i, _i, _vp, _i, _vp]),
    "pw_rotate_rows": (_i, [_vp, _i, _vp, _i, _i, _vp, _i, _i, _vp, _i, _i, _vp]),
    "pw_dense_trtri": (_i, [_vp, _i, _vp, _i, _vp, _i]),
    "pw_dense_syev": (_i, [_vp, _i, _vp, _i, _vp, _ip]),
    "pw_solve_gen_eig": (_i, [_vp, _i, _i, _i, _vp, _vp, _dp, _ip]),
    "pw_wait_probe": (_i, [_vp, C.c_double]),
    "pw_wfn_filter": (_i, [_vp, _vp, _i, _i, _vp]),
    "pw_set_band_batch": (_i, [_vp, _i]),
    "pw_set_nonlocal_mode": (_i, [_vp, _i]),
    "pw_set_gemm_mode": (_i, [_vp, _i, _i]),
    "pw_set_check_errors": (_i, [_vp, _i]),
    "pw_gram": (_i, [_vp, _vp, _i, _i, _vp, _i, _i, _vp, _i, _vp]),
    "pw_cholqr": (_i, [_vp, _vp, _i]),
    "pw_ctx_build_twin": (_i, [_vp]),
    "pw_hartree": (_i, [_vp, _vp, _d, _vp]),
    "pw_xc_teter93": (_i, [_vp, _vp, _vp, _vp]),
    "pw_xc_pbe": (_i, [_vp, _vp, C.c_double, _vp, _vp]),
    "pw_xc_hse06": (_i, [_vp, _vp, C.c_double, _vp, _vp]),
    "pw_eigsolve": (_i, [_vp, _i, _vp, _i, _i, _d, _i, _dp, _dp, _ip]),
    "pw_density": (_i, [_vp, _vp, _i, _i, _dp, _i, _vp]),
    "pw_scf_run": (_i, [_vp, C.POINTER(ScfParams), C.POINTER(ScfResult), _dp, _dp]),
    "pw_hgh_species": (_i, [_i, _dp, _dp, _dp, _dp, _ip]),
    "pw_set_atoms": (_i, [_vp, _i, _ip, _dp]),
    "pw_get_pseudocharge": (_i, [_vp, _dp]),
    "pw_ctx_natom": (_i, [_vp, _ip]),
    "pw_get_atom_projectors": (_i, [_vp, _i, _ip, _ip, _ip, _dp, _dp]),
    "pw_stats": (_i, [_vp, C.POINTER(_l), C.POINTER(_l)]),
    "pw_hgh_atom_projectors": (_i, [_dp, _ip, _i, _dp, _ip, _ip, _ip, _dp, _dp]),
    "pw_hgh_pseudocharge": (_i, [_dp, _ip, _i, _ip, _dp, _dp]),
    "pw_profile": (_i, [_vp, _i]),
    "pw_profile_read": (_i, [_vp, _i, _dp, C.POINTER(_l)]),
    "pw_forces": (_i, [_vp, _vp, _vp, _i, _i, _dp, _i, _dp, _dp, _dp]),
    "pw_scf_forces": (_i, [_vp, _dp, _dp, _dp]),
    "pw_band_energy": (_i, [_vp, _vp, _i, _i, _dp, _dp]),
    "pw_scf_state": (_i, [_vp, _ip, _dp, _vp, _i, _vp]),
    "pw_exx_setup": (_i, [_vp, _d, _d, _i, _d]),
    "pw_set_kpoint": (_i, [_vp, _dp]),
    "pw_graph_capture_hpsi": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, C.POINTER(_vp)]),
    "pw_graph_launch": (_i, [_vp, _vp]),
    "pw_autotune": (_i, [_vp, _i, C.POINTER(TuneResult)]),
    "pw_hpsi_batch": (_i, [_i, C.POINTER(_vp), C.POINTER(_vp), _ip, C.POINTER(_vp), _ip, _ip, _vp]),
    "pw_graph_capture_batch": (_i, [_i, C.POINTER(_vp), C.POINTER(_vp), _ip, C.POINTER(_vp), _ip, _ip,
                                    C.POINTER(_vp)]),
    "pw_graph_nodes": (_i, [_vp, C.POINTER(_l)]),
    "pw_graph_destroy": (_i, [_vp]),
    "pw_hpsi_k": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_get_kpoint_tables": (_i, [_vp, _dp, _dp]),
    "pw_set_kpoints": (_i, [_vp, _i, _dp]),
    "pw_hpsi_kbatch": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_exx_get": (_i, [_vp, _dp, _dp]),
    "pw_exx_set_phi": (_i, [_vp, _vp, _i, _i, _dp]),
    "pw_exx_set_mode": (_i, [_vp, _i]),
    "pw_exx_set_scratch": (_i, [_vp, C.c_size_t]),
    "pw_exx_apply": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "pw_ace_build": (_i, [_vp, _vp, _i, _i]),
    "pw_ace_apply": (_i, [_vp, _vp, _i, _vp, _i, _i, _vp]),
    "pw_exx_energy": (_i, [_vp, _vp, _i, _i, _dp, _i, _i, _dp]),
    "pw_band_energy_backward": (_i, [_vp, _vp, _i, _i, _dp, _vp, _dp]),
    "pw_write_density": (_i, [_vp, C.c_char_p, _dp]),
    "pw_read_density": (_i, [_vp, C.c_char_p, _dp]),
    "pw_write_potential": (_i, [_vp, C.c_char_p, _dp]),
    "pw_write_wfn": (_i, [_vp, C.c_char_p, _dp, _i, _i, _dp]),
    "pw_read_wfn": (_i, [_vp, C.c_char_p, _dp, _i, _i, _ip, _dp]),
    "pw_write_eig": (_i, [C.c_char_p, _i, _dp]),
    "pw_read_eig": (_i, [C.c_char_p, _i, _ip, _dp]),
    "pw_scf_set_initial": (_i, [_vp, _dp, _dp, _i, _i]),
    "pw_ctx_create_gspace": (_i, [_dp, _ip, C.c_double, _i, _i, C.POINTER(_vp)]),
    "pw_gs_sphere": (_i, [_vp, _ip, _ip, _ip, _dp, _dp]),
    "pw_gs_set_projectors": (_i, [_vp, _i, _dp, _dp]),
    "pw_gs_get_projectors": (_i, [_vp, _ip, _dp, _dp]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def check(rc: int) -> None:
    if rc != PW_OK:
        raise PwError(rc, lib.pw_last_error().decode(errors="replace"))
