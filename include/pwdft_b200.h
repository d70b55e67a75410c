/*
 * pwdft_b200 -- C ABI of the B200-native PWDFT Hamiltonian / eigensolver path.
 *
 * Every entry point returns an int status (PW_OK = 0, negative on error) and
 * never lets a C++ exception cross the boundary; pw_last_error() returns the
 * message of the last failure on the calling thread.  Sizes are 32-bit ints
 * like the reference's `Int` (include/environment.hpp:136).  Wavefunction
 * blocks are column-major N_grid x nband with leading dimension ld, each band
 * contiguous, exactly the layout of the reference's NumTns<Real>(ntot, ncom=1,
 * nband) (include/spinor.hpp:80, src/SCF/spinor.cpp:127-133).  Grid index is
 * i + n0*j + n0*n1*k (x fastest).  A context has one arithmetic precision:
 * PW_F64 (double buffers) or PW_F32 (float buffers); "device" pointers are
 * CUDA device memory, "host" pointers are ordinary host memory.
 */
#ifndef PWDFT_B200_H
#define PWDFT_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define PW_API __attribute__((visibility("default")))
#else
#define PW_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PW_OK = 0,
  PW_EINVAL = -1,        /* bad argument / size mismatch (reference: ErrorHandling) */
  PW_ECUDA = -2,         /* CUDA runtime error */
  PW_ENOMEM = -3,        /* device allocation failed */
  PW_EUNSUPPORTED = -4,  /* grid size or configuration not built into this library */
  PW_ETIMEOUT = -5,      /* a bounded device-side wait gave up */
  PW_ENOTREADY = -6,     /* required tables (potential, projectors) not set */
  PW_ENUMERIC = -7       /* numerical breakdown (e.g. Cholesky of a singular Gram) */
};

enum { PW_F64 = 0, PW_F32 = 1 };

/* Nonlocal apply modes.  PW_NL_DENSE: the fine-grid projector sums of the
 * reference are folded into dense coarse-grid columns q_l = T(beta_l) (T is
 * the fine->coarse map R2C fine, IP_f2c, C2R coarse) and applied as
 * H psi += Q diag(gamma vol/N) Q^T psi on tensor-core GEMMs; exact in exact
 * arithmetic because IP_f2c is the transpose of IP_c2f.  PW_NL_REALSPACE: the
 * reference's gather / scaled-dot / scatter over the index sets on the fine grid. */
enum { PW_NL_DENSE = 0, PW_NL_REALSPACE = 1 };

typedef struct pw_ctx pw_ctx;

/* Message of the last failed call on this thread ("" if none). */
PW_API const char* pw_last_error(void);
/* Library version string. */
PW_API const char* pw_version(void);

/* Create a context for an orthorhombic cell with coarse (wavefunction) grid
 * numGrid and fine (density) grid numGridFine = 2*numGrid.  Replaces
 * Fourier::Initialize / Fourier::InitializeFine (src/SCF/fourier.cpp:97-244,
 * 246-418) and KohnSham::CalculateEkin (src/SCF/hamiltonian.cpp:2630-2667):
 * builds |G|^2/2 and the Teter table on the device. */
PW_API int pw_ctx_create(const double length[3], const int numGrid[3], const int numGridFine[3],
                  int precision, int device, pw_ctx** out);
PW_API int pw_ctx_destroy(pw_ctx* ctx);
/* Query grid totals: ntot (coarse), ntotFine. */
PW_API int pw_ctx_sizes(const pw_ctx* ctx, long* ntot, long* ntotFine);

/* Total local potential on the fine grid (host, double, N_fine values).
 * Replaces the vtot argument of Spinor::AddMultSpinorFineR2C
 * (src/SCF/spinor.cpp:377-378, copied per call at hamiltonian.cpp:3121-3122). */
PW_API int pw_set_vtot(pw_ctx* ctx, const double* vtot_fine_host);

/* Real-space nonlocal projectors, the flat form of std::vector<PseudoPot>
 * with vnlList = vector<pair<SparseVec,Real>> (include/periodtable.hpp:62-63,
 * include/utility.hpp:127-151), as built by PeriodTable::CalculateNonlocalPP
 * (src/SCF/periodtable.cpp:994-1240).  For atom a: atom_npts[a] fine-grid
 * indices (one index set shared by all projectors of the atom), atom_nproj[a]
 * projectors.  idx: concatenation over atoms of the index sets.  beta:
 * concatenation over atoms of nproj x npts VAL columns (projector-major).
 * weight: concatenation over atoms of the nproj vnlList weights (gamma).
 * All host pointers. */
PW_API int pw_set_nonlocal(pw_ctx* ctx, int natom, const int* atom_npts, const int* atom_nproj,
                    const int* idx, const double* beta, const double* weight);

/* Select the nonlocal apply mode (call before pw_set_nonlocal / pw_set_atoms). */
PW_API int pw_set_nonlocal_mode(pw_ctx* ctx, int mode);

/* GEMM settings for FP32 contexts: mode must be 0 (the split-BF16 tcgen05
 * kernels), with `terms` products per k-step (3: hi*hi + hi*lo + lo*hi,
 * 4: + lo*lo); any other mode is PW_EINVAL.  FP64 contexts use FP64 GEMMs. */
PW_API int pw_set_gemm_mode(pw_ctx* ctx, int mode, int terms);
/* When enabled, every H*psi call synchronises and returns PW_ETIMEOUT if a
 * bounded device-side pipeline wait gave up (default off). */
PW_API int pw_set_check_errors(pw_ctx* ctx, int enable);
/* Dense projector mode: run the projector GEMMs of an H*psi batch (Q D Q^T psi
 * depends on psi only) on a second stream of the context while the FFT chain
 * runs, joined before the last coarse transform, which then accumulates
 * into the GEMMs' output (1; the default of FP32 contexts); 0 runs them
 * after the FFT chain on the caller's stream (the default of FP64 contexts,
 * whose FP64 GEMMs gain nothing from the overlap).  Overwriting calls give
 * the same bits either way.  While pw_profile is on the GEMMs run after the
 * FFT chain, so each kernel is timed alone.  No reference counterpart. */
PW_API int pw_set_nl_overlap(pw_ctx* ctx, int on);
/* Limit of every bounded wait inside the tensor-core GEMM pipeline on the
 * context's device (all contexts of that device; default 2 s).  On timeout a
 * kernel records an error code, waits (at least 2 s) for the copies and MMAs it
 * issued itself, frees its tensor memory and returns; the next checked call
 * reports PW_ETIMEOUT.  No reference counterpart (the reference has no device
 * waits). */
PW_API int pw_set_wait_limit(pw_ctx* ctx, double seconds);
/* Exercises that failure path without a fault: one thread waits, with the
 * given limit (at most 10 s), on a barrier that nothing releases, records the
 * timeout and returns; the call returns PW_ETIMEOUT and clears the record, and
 * the context stays usable.  No reference counterpart. */
PW_API int pw_wait_probe(pw_ctx* ctx, double seconds);

/* H*psi for nband bands: hpsi (+)= (-1/2 Laplacian + V_loc + V_nl) psi.
 * Replaces Spinor::AddMultSpinorFineR2C(fft, ekin, vtot, pseudo, a3)
 * (src/SCF/spinor.cpp:377-525; accumulate=1 gives its a3 += semantics) and
 * KohnSham::MultSpinor without hybrid exchange (src/SCF/hamiltonian.cpp:
 * 3059-3268; accumulate=0 overwrites a3).  psi, hpsi: device pointers of the
 * context's precision.  stream: cudaStream_t (NULL = legacy default). */
PW_API int pw_hpsi(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband,
            int accumulate, void* stream);

/* Same as pw_hpsi with host buffers: copies psi in and hpsi out around the
 * device computation (the path a host-side reference caller binds).  With
 * page-locked host buffers the bands move in chunks whose copies in and out
 * overlap the H*psi of the neighbouring chunks; returns when hpsi is written. */
PW_API int pw_hpsi_host(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband,
                 int accumulate);
/* Bands per pw_hpsi_host chunk (rounded up to even; 0: the default 32). */
PW_API int pw_set_host_chunk(pw_ctx* ctx, int nband);

/* Wavefunction cut-off filter of KohnSham::MultSpinor, which the reference
 * switches on for PW_Solver CheFSI with the cut-off Ecut_Wavefunction
 * (set_wfn_filter(PWDFT_Cheby_apply_wfn_ecut_filt, 1, ecutWavefunction),
 * src/SCF/hamiltonian.cpp:316-321; PWDFT_Cheby_apply_wfn_ecut_filt defaults to
 * 1, src/esdf.cpp:2719).  P = C2R o (zero every coefficient with
 * gkkR2C = |G|^2/2 > ecut) o R2C.  While enabled, an overwriting pw_hpsi
 * (accumulate = 0, MultSpinor) returns P H psi -- the exit filter of
 * hamiltonian.cpp:3240-3265, fused into the z-fold kernel and into the
 * store-side projector / ACE matrices (P Q, P xi, built once per geometry); an
 * accumulating call (AddMultSpinorFineR2C) is not filtered, as in the
 * reference.  The reference's first MultSpinor call also replaces psi by
 * P psi in place (hamiltonian.cpp:3090-3116): pw_wfn_filter does that step
 * (pw_eigsolve and pw_scf_run do it on their start blocks; the C++ mirror's
 * Hamiltonian::MultSpinor does it on its first call).  Real-space contexts;
 * enable = 0 switches the filter off. */
PW_API int pw_set_wfn_filter(pw_ctx* ctx, int enable, double ecut);
/* X <- P X in place for nband device columns (needs pw_set_wfn_filter). */
PW_API int pw_wfn_filter(pw_ctx* ctx, void* X, int ld, int nband, void* stream);

/* Teter preconditioner: w (+)= C2R(teter * R2C(r)).  Replaces
 * Spinor::AddTeterPrecond(Fourier*, DblNumVec& teter, NumTns<Real>& a3)
 * (src/SCF/spinor.cpp:310-346). Device pointers. */
PW_API int pw_teter_precond(pw_ctx* ctx, const void* r, int ld, void* w, int ldw, int nband,
                     int accumulate, void* stream);

/* HGH species built into the library (Si: 14, Al: 13; utilities/HGH.m:234-276):
 * valence charge, self energy E_self (HGH.m:995), cut-off radii, number of
 * nonlocal projectors. */
PW_API int pw_hgh_species(int znuc, double* zion, double* eself, double* rcut_nonlocal, double* rcut_rho,
                          int* nproj);

/* Atoms (Cartesian bohr, natom x 3) with the library's HGH tables: builds every
 * atom's projector set as PeriodTable::CalculateNonlocalPP does
 * (src/SCF/periodtable.cpp:994-1240) and the pseudocharge of
 * PeriodTable::CalculatePseudoCharge (periodtable.cpp:282-377, with Cartesian
 * minimum-image distances), the work of KohnSham::CalculatePseudoPotential
 * (src/SCF/hamiltonian.cpp:327-918).  Calls pw_set_nonlocal internally. */
PW_API int pw_set_atoms(pw_ctx* ctx, int natom, const int* znuc, const double* pos);
/* Pseudocharge rho_ps on the fine grid (host, N_fine doubles). */
/* Number of atoms set by pw_set_atoms. */
PW_API int pw_ctx_natom(const pw_ctx* ctx, int* natom);
PW_API int pw_get_pseudocharge(const pw_ctx* ctx, double* rho_fine_host);
/* One atom's projector set: npts, nproj, idx[npts], val4[nproj][npts][4]
 * (VAL, DX, DY, DZ), wgt[nproj].  Output pointers may be NULL. */
PW_API int pw_get_atom_projectors(const pw_ctx* ctx, int atom, int* npts, int* nproj, int* idx, double* val4,
                                  double* wgt);
/* Host-only variants (no context, no GPU): one atom's projector set for a cell
 * and fine grid (call with NULL outputs first to get npts, nproj), and the
 * summed pseudocharge of natom atoms on the fine grid. */
PW_API int pw_hgh_atom_projectors(const double length[3], const int numGridFine[3], int znuc, const double pos[3],
                                  int* npts, int* nproj, int* idx, double* val4, double* wgt);
PW_API int pw_hgh_pseudocharge(const double length[3], const int numGridFine[3], int natom, const int* znuc,
                               const double* pos, double* rho_fine_host);
/* Number of this library's CUDA kernels the context has launched, and of
 * vendor-library (cuBLAS / cuSOLVER) calls it made. */
PW_API int pw_stats(const pw_ctx* ctx, long* kernel_launches, long* library_calls);

/* Per-kernel CUDA-event timing.  pw_profile(ctx, 1) clears the records and
 * brackets every later kernel launch of this context with events on its
 * stream; pw_profile_read returns the summed device time and the number of
 * launches of one kernel kind: 0 coarse-plane FFT, 1 z-pad, 2 fine-plane
 * projector gather, 3 projector reduce, 4 fine-plane apply, 5 z-fold,
 * 6 coarse-plane inverse, 7 Teter z-pencil, 8 Gram, 9 density, 10 other,
 * 11 vendor-library GEMM, 12 exact-exchange pair FFTs, 13 subspace rotation
 * (X C of the eigensolvers). */
PW_API int pw_profile(pw_ctx* ctx, int enable);
PW_API int pw_profile_read(pw_ctx* ctx, int kind, double* total_ms, long* count);

/* Gram block over the coarse grid: G (nx x ny, column-major, leading
 * dimension ldg, FP64, device) = X^T Y for X (ntot x nx, ldx) and Y
 * (ntot x ny, ldy) in the context's precision.  Replaces the
 * blas::Gemm('T','N', ...) + MPI_Allreduce Gram blocks of
 * EigenSolver::Orthogonalize (src/EigenSolver/eigensolver.cpp:301-384) and
 * LOBPCGSolveReal (src/EigenSolver/lobpcg.cpp:683-874).  FP32 contexts run
 * split-BF16 tensor-core GEMMs with FP32 accumulation. */
PW_API int pw_gram(pw_ctx* ctx, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G, int ldg,
                   void* stream);

/* ---------------------------------------------------------------------------
 * Small dense FP64 algebra of the eigensolvers (device pointers, column-major;
 * this library's kernels, where the reference calls LAPACK on rank 0)
 * ------------------------------------------------------------------------- */
/* Upper Cholesky A = U^T U in place (lapack::Potrf('U') of
 * EigenSolver::Orthogonalize, src/EigenSolver/eigensolver.cpp:301-384); the
 * strict lower part is left as it was; PW_ENUMERIC if A is not positive definite. */
PW_API int pw_dense_potrf(pw_ctx* ctx, int n, double* A, int lda);
/* Ui = U^{-1} for an upper-triangular U (the Trsm of Orthogonalize applied to
 * the identity); the strict lower part of Ui is zeroed. */
PW_API int pw_dense_trtri(pw_ctx* ctx, int n, const double* U, int ldu, double* Ui, int ldi);
/* Symmetric eigen-decomposition (lapack::Syevd('V', 'U'), the Rayleigh-Ritz
 * solves of src/EigenSolver/lobpcg.cpp and eigensolver.cpp:133-299): the upper
 * triangle of A is read, A's columns receive the eigenvectors, w (device) the
 * eigenvalues ascending.  Up to n = 160: Householder tridiagonalisation,
 * multisection on Sturm counts and inverse iteration (sweeps = 0); beyond:
 * cyclic Jacobi, and sweeps (host, may be NULL) reports the sweeps it took. */
PW_API int pw_dense_syev(pw_ctx* ctx, int n, double* A, int lda, double* w, int* sweeps);
/* EigenSolver::SolveGenEig (src/EigenSolver/eigensolver.cpp:133-299, serial
 * path): symmetrise A and B from their upper triangles, eig(B) = U sigma U^T,
 * keep the directions with sigma / sigma_max > 1e-8 (numKeep, at least width),
 * A~ = sigma^-1/2 U^T A U sigma^-1/2, eig(A~), C = U sigma^-1/2 Z.  On exit A
 * holds C (numCol x numKeep), eig (host) the lowest `width` values. */
PW_API int pw_solve_gen_eig(pw_ctx* ctx, int lda, int numCol, int width, double* A, double* B, double* eig,
                            int* numKeep);

/* Subspace rotation Out (+)= X C over the coarse grid: X (ntot x k, ldx) and
 * Out (ntot x m, ldo) in the context's precision, C (k x m, ldc) FP64 on the
 * device; the X <- X C updates of Orthogonalize and LOBPCGSolveReal
 * (blas::Gemm('N', 'N'), src/EigenSolver/eigensolver.cpp:301-384,
 * lobpcg.cpp:869-1000).  FP32 contexts: split-BF16 tensor-core GEMM (C rounded
 * to FP32, then split); FP64 contexts: this library's FP64 kernel.  Out must
 * not overlap X. */
PW_API int pw_rotate(pw_ctx* ctx, const void* X, int ldx, int k, const double* C, int ldc, int m, void* Out, int ldo,
                     int accumulate, void* stream);
/* The Gram block and the rotation over the first nrow rows only: a row block
 * of the grid, the local product of the reference's band <-> grid-row
 * transposed eigensolver steps (AlltoallForward, local Gemm, MPI_Allreduce;
 * src/utility.cpp:1159-1197, src/EigenSolver/lobpcg.cpp:683-687).  FP32
 * contexts need nrow and the leading dimensions to be multiples of 8. */
PW_API int pw_gram_rows(pw_ctx* ctx, int nrow, const void* X, int ldx, int nx, const void* Y, int ldy, int ny,
                        double* G, int ldg, void* stream);
PW_API int pw_rotate_rows(pw_ctx* ctx, int nrow, const void* X, int ldx, int k, const double* C, int ldc, int m,
                          void* Out, int ldo, int accumulate, void* stream);

/* ---------------------------------------------------------------------------
 * Block eigensolvers and SCF
 * ------------------------------------------------------------------------- */
enum { PW_SOLVER_LOBPCG = 0, PW_SOLVER_CHEBFSI = 1, PW_SOLVER_PPCG = 2, PW_SOLVER_DAVIDSON = 3 };

/* In-place Cholesky-QR of nb device columns X (ntot x nb): X <- X U^{-1},
 * X^T X = U^T U.  Replaces EigenSolver::Orthogonalize
 * (src/EigenSolver/eigensolver.cpp:301-384). */
PW_API int pw_cholqr(pw_ctx* ctx, void* X, int nb);

/* Lowest nb eigenpairs of H (current potential and projectors) starting from
 * the device block X (overwritten by the Ritz vectors).  solver:
 * PW_SOLVER_LOBPCG restates EigenSolver::LOBPCGSolveReal
 * (src/EigenSolver/lobpcg.cpp:577-1031: maxit = Eig_MaxIter, tol = residual
 * tolerance); PW_SOLVER_CHEBFSI runs Chebyshev-filtered subspace iteration of
 * the given degree (the reference's CheFSI parameters, src/esdf.cpp:2715-2719)
 * for up to maxit cycles; PW_SOLVER_PPCG restates EigenSolver::PPCGSolveReal
 * (src/EigenSolver/ppcg.cpp:670-1243) with sub-block size `degree` (PPCG_sbSize,
 * 1..8); PW_SOLVER_DAVIDSON restates EigenSolver::DavidsonSolveReal
 * (src/EigenSolver/davidson.cpp:60-806) with a subspace of `degree` blocks
 * (maxdim, >= 2) and convergence on the change of each Ritz value.  eig,
 * resnorm: host arrays of nb (may be NULL). */
PW_API int pw_eigsolve(pw_ctx* ctx, int solver, void* X, int nb, int maxit, double tol, int degree, double* eig,
                       double* resnorm, int* iters);

/* Electron density on the fine grid from nband device wavefunctions and host
 * occupation rates (numSpin = 2), renormalised to 2*nocc_total electrons:
 * KohnSham::CalculateDensity (src/SCF/hamiltonian.cpp:2455-2627).  rho_dev:
 * device, N_fine doubles.  nocc_total <= 0: no renormalisation (the raw
 * sum 2 f_k |psi_k|^2 of these bands, a rank's part of a band-distributed
 * density, normalised once after the reduction as the reference does). */
PW_API int pw_density(pw_ctx* ctx, const void* psi, int ld, int nband, const double* occ_host, int nocc_total,
                      double* rho_dev);

/* Hartree potential of a charge on the fine grid (device, N_fine doubles):
 * V_H = IFFT(2 pi / gkk * FFT(drho)) with gkk = |G|^2 / 2, zero for
 * gkk <= 1e-16 or gkk > 4*ecut -- KohnSham::CalculateHartree
 * (src/SCF/hamiltonian.cpp:1990-2026) with drho = rho - pseudocharge.
 * Cubic fine grids. */
PW_API int pw_hartree(pw_ctx* ctx, const double* drho_dev, double ecut, double* vh_dev);
/* LDA Teter93 exchange-correlation energy density and potential on the fine
 * grid (device), points with rho < 1e-10 zeroed -- KohnSham::CalculateXC
 * (src/SCF/hamiltonian.cpp:1278-1308). */
PW_API int pw_xc_teter93(pw_ctx* ctx, const double* rho_dev, double* eps_dev, double* vxc_dev);
/* PBE exchange-correlation on the fine grid (device, N_fine doubles each): the
 * Use_Libxc 0 branch of KohnSham::CalculateXC (src/SCF/hamiltonian.cpp:
 * 1381-1419, 1560-1612, 1680-1760; Slater + PW92 + PBE gradient corrections of
 * src/utility.cpp:3913-4244) with the spectral gradient of
 * KohnSham::CalculateGradDensity (hamiltonian.cpp:1153-1239; components with
 * gkk = 0 or gkk > 4 ecut dropped).  eps: energy per particle (E_xc = sum eps
 * rho vol / N_fine); vxc = d e/d rho - div(2 d e/d|grad rho|^2 grad rho).
 * Cubic cells and fine grids only. */
PW_API int pw_xc_pbe(pw_ctx* ctx, const double* rho_dev, double ecut, double* eps_dev, double* vxc_dev);
/* Semilocal part of HSE06 on the fine grid (same arguments and layout as
 * pw_xc_pbe): PBE minus 0.25 times the erfc-screened (omega = 0.106) PBE
 * exchange where |rho| > 1e-6 and |grad rho|^2 > 1e-10 -- the
 * XC_HYB_GGA_XC_HSE06 branch of KohnSham::CalculateXC (src/SCF/
 * hamiltonian.cpp:1563, 1614-1627) with pbexsr / wpbe_analy_erfc_approx_grad
 * (src/utility.cpp:3340-3846).  The exact-exchange part of the hybrid is
 * pw_exx_setup(ctx, 0.25, 0.106, ...) and the pw_exx_* calls. */
PW_API int pw_xc_hse06(pw_ctx* ctx, const double* rho_dev, double ecut, double* eps_dev, double* vxc_dev);
enum { PW_XC_TETER93 = 0, PW_XC_PBE = 1, PW_XC_HSE06 = 2 };

typedef struct pw_scf_params {
  int nocc;                 /* occupied states (numOccupiedState) */
  int nextra;               /* Extra_States */
  int solver;               /* PW_SOLVER_LOBPCG or PW_SOLVER_CHEBFSI */
  int cheby_degree;         /* ChebFSI filter degree */
  int cheby_first_cycles;   /* filter cycles in the first SCF iteration */
  int eig_max_iter;         /* Eig_MaxIter (LOBPCG) */
  int max_iter;             /* SCF_Outer_MaxIter */
  int mix_dim;              /* Mixing_MaxDim */
  int mixed;                /* 1: FP32 H*psi / split-BF16 Gram eigensolver, FP64 refinement */
  int verbose;              /* 1: a line per SCF iteration (stderr); 2: phase timers (graphs off);
                               3: as 1 plus the synchronised wall time of each step */
  double ecut;              /* Ecut_Wavefunction (Hartree cut-off 4*Ecut) */
  double temperature;       /* Kelvin (the smearing width) */
  double eig_tol;           /* Eig_Tolerance */
  double mix_step;          /* Mixing_StepLength */
  double tol_efree;         /* converged when |E_free - E_Harris| / N_atom < tol_efree */
  double refine_threshold;  /* mixed mode: switch the eigensolver to FP64 below this */
  unsigned long long seed;  /* random start */
  int ppcg_sbsize;          /* PPCG_sbSize (PW_SOLVER_PPCG), 1..8 */
  int davidson_maxdim;      /* subspace size in blocks (PW_SOLVER_DAVIDSON), >= 2 */
  int graphs;               /* 1: replay the Chebyshev filter from a captured CUDA graph */
  int xc;                   /* PW_XC_TETER93 (LDA, default), PW_XC_PBE (XC_Type XC_GGA_XC_PBE, Use_Libxc 0) or
                               PW_XC_HSE06 (XC_HYB_GGA_XC_HSE06: PBE SCF, then nested phi iterations with ACE) */
  int mix_type;             /* PW_MIX_ANDERSON (default) or PW_MIX_BROYDEN (Mixing_Type, potential mixing) */
  double tol_rho;           /* > 0: converged when the density change's scfNorm (SCF::CalculateError) < tol_rho
                               instead of the E_free - E_Harris test */
  int phi_max_iter;         /* PW_XC_HSE06: outer phi (ACE) iterations, Hybrid_Phi_MaxIter (0: 10) */
  double phi_tol;           /* PW_XC_HSE06: converged when dExx = 4 |fock1 - (fock0 + fock2) / 2| < phi_tol */
  int no_wfn_filter;        /* PW_SOLVER_CHEBFSI: 0 (default) runs H*psi with the wavefunction cut-off filter at
                               ecut, as the reference's CheFSI does (PWDFT_Cheby_apply_wfn_ecut_filt 1); 1 runs
                               the unfiltered operator (PWDFT_Cheby_apply_wfn_ecut_filt 0).  Other solvers: no filter */
  int smearing;             /* Smearing_Scheme: 0 "FD" (Fermi-Dirac, default), 1 "GB" (Gaussian, occupation
                               erfc(-x) / 2, -T S term -exp(-x^2) / (2 beta sqrt(pi)), x = beta (E_F - e)) */
} pw_scf_params;
enum { PW_MIX_ANDERSON = 0, PW_MIX_BROYDEN = 1 };

typedef struct pw_scf_result {
  double etot, efree, eharris, exc, ehart, eself, fermi, time_s;
  int iterations, converged, refine_iter;
  long hpsi_bands;          /* single-band H*psi applications performed */
  double phase_s[6];        /* verbose == 2: eigensolver, density, potentials, set-up, mixing, refine switch (s) */
  double sub_s[4];          /* verbose == 2, inside the eigensolver: H*psi, Gram, dense FP64, rotations (s) */
  double scf_norm;          /* last SCF::CalculateError of the output-density change (scf.cpp:2368-2396) */
  double efock;             /* PW_XC_HSE06: exchange energy of the last ACE (Efock, included in etot / efree) */
  double dexx;              /* PW_XC_HSE06: last dExx */
  int phi_iterations;       /* PW_XC_HSE06: outer phi iterations run */
} pw_scf_result;

/* Build (once) the FP32 twin of an FP64 context with the same cell, grids and
 * atoms; the mixed-precision SCF runs its eigensolver there.  Set-up work:
 * call it after pw_set_atoms, before timing an SCF. */
PW_API int pw_ctx_build_twin(pw_ctx* ctx);

/* Self-consistent field iteration for the atoms of an FP64 context
 * (pw_set_atoms): SCF::Iterate / InnerSolve with potential Anderson mixing
 * (src/SCF/scf.cpp:372-591, 1261-1589, 2299-2365), density, Hartree and LDA
 * Teter93 XC (src/SCF/hamiltonian.cpp:1242-1308, 1990-2069, 2455-2627) and the
 * energies of scf.cpp:1834-2140, all on the device.  eig_out: host, nocc+nextra
 * doubles; rho_out: host, N_fine doubles (either may be NULL).
 * xc = PW_XC_HSE06 runs the reference's nested hybrid scheme (scf.cpp:409-
 * 623, 628-925): a PBE SCF, then the semilocal HSE06 potential and phi
 * iterations -- phi <- psi, ACE from the bands (exchange kernel of
 * pw_exx_setup(ctx, 0.25, 0.106, 1, ecut)), an inner SCF with the ACE term in
 * H, Fock energies fock1 (old ACE) / fock2 (new ACE), E += fock2 - 2 fock1,
 * until dExx < phi_tol.  Inner SCF loops restart the mixing history; with
 * tol_rho > 0 their criterion is the scfNorm of the potential change, as the
 * reference's nested loop has it.  The hybrid phase runs in FP64 (a mixed run
 * switches before it); the context keeps the ACE operator afterwards.  Other
 * functionals run without an exchange term whatever pw_exx_set_mode chose
 * (the mode is restored on return). */
PW_API int pw_scf_run(pw_ctx* ctx, const pw_scf_params* p, pw_scf_result* r, double* eig_out, double* rho_out);

/* Autotuner (no reference counterpart): times pw_hpsi on an internal block
 * of nband bands for candidate band-batch widths, the two radix decompositions
 * of the fused fine-plane transforms and, for FP32 contexts with dense
 * projectors, the tile widths of the two projector GEMMs; applies the
 * fastest setting to the context and caches it for later contexts of the
 * same grid, precision, band count and projector count (then cached = 1 and
 * no timing runs).  The local potential must be set. */
typedef struct pw_tune_result {
  int band_batch;           /* bands per internal batch chosen */
  int gemm_bn;              /* Q^T psi GEMM tile width (0: heuristic) */
  int gemm_bn_store;        /* Q W GEMM tile width (0: heuristic) */
  int tried;                /* configurations timed */
  int cached;               /* 1: taken from the cache */
  double ms_default;        /* sweep time with the defaults */
  double ms_best;           /* sweep time with the chosen setting */
  int fft_variant;          /* fused fine-plane transforms: 0 table twiddles, 1 second radix split, 2 (default) register twiddles */
} pw_tune_result;
/* Select the form of the fused fine-plane transforms directly (0: the first
 * radix decomposition N = n1 x n2 of each length with the inter-stage
 * twiddles read from shared-memory tables, 1: the second decomposition, e.g.
 * 96 = 12 x 8 instead of 8 x 12, 2 (the default): the first decomposition
 * with the twiddles of a transform formed in registers from one table entry
 * and the local potential read in the row pass's lane order); pw_autotune
 * times all three.  No reference counterpart. */
PW_API int pw_set_fft_variant(pw_ctx* ctx, int variant);
PW_API int pw_autotune(pw_ctx* ctx, int nband, pw_tune_result* result);

/* CUDA graph of one pw_hpsi call (same pointers, band count and accumulate
 * flag on every replay; the inputs' contents may change between replays).
 * The capture runs one ordinary call first (outside the graph).  Replays
 * issue every kernel and library GEMM of the sweep with one launch. */
typedef struct pw_graph pw_graph;
PW_API int pw_graph_capture_hpsi(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband,
                                 int accumulate, pw_graph** graph);
PW_API int pw_graph_launch(pw_graph* graph, void* stream);
/* H*psi for ncell independent contexts at once (cells of uneven grids, band
 * counts and precisions on one device): cell c applies ctxs[c] to nband[c]
 * bands psi[c] -> out[c] (overwrite), each cell's sweep on its own stream
 * forked from `stream` and joined back into it.  pw_graph_capture_batch
 * captures the whole batch as one CUDA graph (one launch per replay). */
PW_API int pw_hpsi_batch(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld, void* const* out,
                         const int* ldo, const int* nband, void* stream);
PW_API int pw_graph_capture_batch(int ncell, pw_ctx* const* ctxs, const void* const* psi, const int* ld,
                                  void* const* out, const int* ldo, const int* nband, pw_graph** graph);
PW_API int pw_graph_nodes(const pw_graph* graph, long* nodes);
PW_API int pw_graph_destroy(pw_graph* graph);

/* k-point mode (complex bands).  pw_set_kpoint builds, for the Bloch vector
 * k (Cartesian, bohr^-1), the kinetic 1/2 |k+G|^2 and Teter tables
 * (KohnSham::CalculateEkin, complex version, src/SCF/hamiltonian_complex.cpp:
 * 234-277) and the coarse projectors with the phase e^{i k.(r - R_a)}
 * (src/SCF/periodtable.cpp:1104-1121; needs pw_set_atoms).  pw_hpsi_k applies
 * H(k) (Spinor::AddMultSpinorFine, complex, src/SCF/spinor_complex.cpp:292-542)
 * to nband complex bands: device arrays of interleaved (re, im) pairs of the
 * context precision, leading dimensions ld / ldh in complex elements. */
PW_API int pw_set_kpoint(pw_ctx* ctx, const double k[3]);
PW_API int pw_hpsi_k(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate,
                     void* stream);
/* A batch of nk Bloch vectors (kpts: host, nk x 3) kept resident (tables and
 * projectors per k); pw_hpsi_kbatch applies H(k_i) to nband complex bands of
 * every k-point in one pass: psi / hpsi hold nk * nband columns, k-point
 * major (column i * nband + b is band b of k-point i). */
PW_API int pw_set_kpoints(pw_ctx* ctx, int nk, const double* kpts);
PW_API int pw_hpsi_kbatch(pw_ctx* ctx, const void* psi, int ld, void* hpsi, int ldh, int nband, int accumulate,
                          void* stream);
/* The kinetic and Teter tables of the current k on the full coarse grid (host,
 * N_coarse doubles each; either may be NULL). */
PW_API int pw_get_kpoint_tables(const pw_ctx* ctx, double* ekin_host, double* teter_host);

/* Hybrid exact exchange (Gamma point, real bands; sphere-cut FP64 contexts:
 * the complex overload of Spinor::AddMultSpinorEXX, src/SCF/spinor.cpp:
 * 783-945, with pair products on the full G-space grid, the kernel on the
 * Fock set 1/2 |G|^2 < 4 Ecut and phi = sqrt(1 / (vol N)) c).  Modes of the exchange
 * term inside pw_hpsi: off, the full pair-FFT operator
 * (Spinor::AddMultSpinorEXX, src/SCF/spinor.cpp:682-781) or the ACE operator
 * (KohnSham::MultSpinor, src/SCF/hamiltonian.cpp:3135-3218). */
enum { PW_EXX_OFF = 0, PW_EXX_FULL = 1, PW_EXX_ACE = 2 };

/* Coulomb kernel of KohnSham::InitializeEXX (src/SCF/hamiltonian.cpp:3454-3551):
 * v(G) = 4 pi / |G|^2 (times 1 - exp(-|G|^2 / 4 mu^2) when screen_mu > 0),
 * G = 0 set to -exxDiv (+ pi / mu^2), exxDiv from divergence_type 0 (none) or
 * 1 (auxiliary function with alpha = 10 / (2 Ecut)).  exx_fraction is the
 * mixing alpha (0.25 for PBE0). */
PW_API int pw_exx_setup(pw_ctx* ctx, double exx_fraction, double screen_mu, int divergence_type,
                        double ecut_wavefunction);
/* exxDiv and the kernel on the full coarse spectrum (host, N_coarse doubles;
 * sphere-cut contexts: the full G-space grid, N_fine doubles; either pointer
 * may be NULL). */
PW_API int pw_exx_get(const pw_ctx* ctx, double* exx_div, double* kern_host);
/* Exchange orbitals phi = sqrt(N_c / vol) psi with their occupation rates
 * (KohnSham::SetPhiEXX, hamiltonian.cpp:3554-3641).  psi: device, context
 * precision, nphi columns; occ: host, nphi. */
PW_API int pw_exx_set_phi(pw_ctx* ctx, const void* psi, int ld, int nphi, const double* occ);
PW_API int pw_exx_set_mode(pw_ctx* ctx, int mode);
/* Device memory budget for the exchange pair fields (default 1 GiB); V_x psi
 * runs in batches of (band, orbital pair) fields that fit it. */
PW_API int pw_exx_set_scratch(pw_ctx* ctx, size_t bytes);
/* out (+)= V_x psi for nband bands (AddMultSpinorEXX), device pointers. */
PW_API int pw_exx_apply(pw_ctx* ctx, const void* psi, int ld, void* out, int ldo, int nband, int accumulate,
                        void* stream);
/* ACE operator from nband bands (KohnSham::CalculateVexxACE,
 * hamiltonian.cpp:3686-3818): W = V_x psi, M = -psi^T W = L L^T, xi = W L^-T;
 * switches the context to PW_EXX_ACE. */
PW_API int pw_ace_build(pw_ctx* ctx, const void* psi, int ld, int nband);
/* out += -xi (xi^T psi) (the ACE term alone). */
PW_API int pw_ace_apply(pw_ctx* ctx, const void* psi, int ld, void* out, int ldo, int nband, void* stream);
/* Exchange energy num_spin / 2 * sum_j occ_j psi_j^T V_x psi_j
 * (KohnSham::CalculateEXXEnergy, hamiltonian.cpp:3936-4192), with the full
 * operator (use_ace = 0) or the ACE operator (use_ace = 1); e: host. */
PW_API int pw_exx_energy(pw_ctx* ctx, const void* psi, int ld, int nband, const double* occ, int num_spin,
                         int use_ace, double* e);

/* Atomic forces of an FP64 context with atoms (pw_set_atoms),
 * KohnSham::CalculateForce (src/SCF/hamiltonian.cpp:2670-3056), pseudocharge
 * form: local part pseudocharge . grad V_H[rho - rho_ps] (:2716-2800) plus the
 * nonlocal part of :2907-3006.  rho_dev: device, N_fine doubles; psi_dev:
 * device, nband columns of N_coarse doubles (leading dimension ldpsi); occ:
 * host, nband occupation rates in [0, 1]; num_spin: 1 or 2 (numSpin).  force:
 * host, natom x 3 (Hartree / bohr); force_local / force_nonlocal (host, may be
 * NULL) receive the two parts.  The reference's VdW, short-range ion and
 * external terms are not part of this path. */
PW_API int pw_forces(pw_ctx* ctx, const double* rho_dev, const void* psi_dev, int ldpsi, int nband,
                     const double* occ, int num_spin, double* force, double* force_local, double* force_nonlocal);

/* Band energy E = sum_b w_b <psi_b, H psi_b> (the forward half of the
 * adjoint pair; no reference counterpart as an entry point -- the reference
 * forms the same sum inside its energy and force routines).  psi: device,
 * context precision, nband columns (leading dimension ld); w: host, nband
 * weights (numSpin * occupation for a band energy); e: host, one double. */
PW_API int pw_band_energy(pw_ctx* ctx, const void* psi, int ld, int nband, const double* w, double* e);

/* Backward of pw_band_energy at fixed psi.  dE_dV_dev (device, N_fine
 * doubles, may be NULL): dE/dV_loc(r) on the density grid, recomputing the
 * fine-grid bands per batch instead of storing them.  dE_dR (host, natom x 3,
 * may be NULL; FP64 context with pw_set_atoms): dE/dR of every atom through
 * the analytic projector derivatives (the DX/DY/DZ columns of vnlList,
 * src/SCF/periodtable.cpp:994-1240). */
PW_API int pw_band_energy_backward(pw_ctx* ctx, const void* psi, int ld, int nband, const double* w,
                                   double* dE_dV_dev, double* dE_dR);

/* The state the last pw_scf_run left in an FP64 context: band count,
 * occupation rates (host, nband), bands (device, nband columns, leading
 * dimension ldpsi) and output density (device, N_fine); pointers may be NULL. */
PW_API int pw_scf_state(const pw_ctx* ctx, int* nband, double* occ, double* psi_dev, int ldpsi, double* rho_dev);

/* Forces from the state the last pw_scf_run left in the context (its final
 * FP64 bands, occupations and output density), numSpin = 2. */
PW_API int pw_scf_forces(pw_ctx* ctx, double* force, double* force_local, double* force_nonlocal);

/* Teter preconditioner that allocates nothing (no counterpart in the
 * reference).  Same result as pw_teter_precond; for callers that cannot call
 * cudaMalloc where they need it -- code inside CUDA stream capture, hosts that
 * forbid device allocation after start-up, frameworks whose own memory pool
 * must not see the device heap change.  Its working memory is one fixed
 * 16 MiB device array in the library (held by every GPU that loads it until
 * the process exits), so a grid whose single band pair needs more than
 * 16 MiB (ntot * 2 * sizeof(real) bytes) is rejected with PW_EINVAL; larger
 * band counts run in batches that fit.  The first call on a device looks up
 * the array's device address: make that first call before any stream
 * capture.  The address is kept for the life of the process, so calls after a
 * cudaDeviceReset of that device are not supported.  All calls share the array
 * (each call writes every element it reads, so nothing needs clearing between
 * calls); calls that overlap on the same GPU (several streams, or several
 * contexts on one device) race on the array and must be serialised by the
 * caller. */
PW_API int pw_teter_precond_noalloc(pw_ctx* ctx, const void* r, int ld, void* w, int ldw, int nband, int accumulate,
                                    void* stream);

/* Maximum number of bands processed per internal batch (sets scratch size).
 * Default 64. Scratch grows to hold ceil(nband_batch/2) band pairs. */
PW_API int pw_set_band_batch(pw_ctx* ctx, int nband_batch);

/* ---- Restart files in the reference's binary layout ----
 * serialize() layout (include/utility.hpp:1183-1278): a vector is an int32
 * length then that many doubles; a matrix two int32 sizes then the
 * column-major doubles; a 3-tensor three int32 sizes then the doubles; native
 * byte order.  All buffers are host memory.
 *   DEN  (scf.cpp:1070-1088, read at :164-178): the fine-grid fractional
 *        positions i/N_d for d = x, y, z (UniformMeshFine, utility.cpp:405-420),
 *        then the density (N_fine).  pw_read_density checks the grid sizes.
 *   POT  (scf.cpp:1091-1108): the same grid vectors, then Vtot as N_fine x 1.
 *   WFN_<rank> (scf.cpp:1110-1145 via SeparateWrite "name_<rank>", read at
 *        :296-330): the bands as an ntot x 1 x nband tensor, then the
 *        occupations (nband).  Real-space contexts.  pw_read_wfn with
 *        psi = NULL returns the band count in *nband.
 *   EIG  (scf.cpp:1247-1253): the eigenvalues as one vector.
 * pw_scf_set_initial hands the next pw_scf_run a starting density (N_fine,
 * used as given, as isRestartDensity does) and/or starting bands (nband must
 * equal nocc + nextra of that run); either may be NULL.  Consumed by that run. */
PW_API int pw_write_density(const pw_ctx* ctx, const char* path, const double* rho_fine);
PW_API int pw_read_density(const pw_ctx* ctx, const char* path, double* rho_fine);
PW_API int pw_write_potential(const pw_ctx* ctx, const char* path, const double* vtot_fine);
PW_API int pw_write_wfn(const pw_ctx* ctx, const char* path, const double* psi, int ld, int nband, const double* occ);
PW_API int pw_read_wfn(const pw_ctx* ctx, const char* path, double* psi, int ld, int nband_max, int* nband,
                       double* occ);
PW_API int pw_write_eig(const char* path, int n, const double* eig);
PW_API int pw_read_eig(const char* path, int nmax, int* n, double* eig);
PW_API int pw_scf_set_initial(pw_ctx* ctx, const double* rho_fine, const double* psi, int ld, int nband);

/* ---- Sphere-cut (G-space) mode, the reference's Use_Real_Space: 0 ----
 * A band is its Fourier coefficients on the half sphere 1/2 |G|^2 < ecut, in
 * the order of Fourier::idxCoarseCut (ascending R2C index, G_x >= 0 with the
 * G_x = 0 half plane G_y > 0 or G_y = 0, G_z >= 0; src/SCF/fourier.cpp:542-640),
 * complex, with the sqrt(2) convention of Spinor::wavefunG_ (c_0 = psi(0),
 * c_s = sqrt(2) psi(G_s); src/SCF/spinor.cpp:568-590).  The entry points take
 * a band as 2 ns reals (re, im interleaved, `ld` even, in reals), so
 * pw_hpsi / pw_teter_precond / pw_eigsolve / pw_gram / pw_density / pw_scf_run
 * run unchanged on a G-space context; their inner product is the reference's
 * Re(X^H Y) Gram (src/MathLibs/blas.cpp:997-1029).  Im c_0 must be zero.
 * pw_hpsi adds the nonlocal term of EigenSolver::NonlocalMultX
 * (src/EigenSolver/eigensolver.cpp:471-515) to the local + kinetic part of
 * Spinor::AddMultSpinorFineR2C's complex overload (spinor.cpp:528-680), the
 * sum LOBPCGSolveReal forms (src/EigenSolver/lobpcg.cpp:201-211).
 *
 * pw_ctx_create_gspace replaces Fourier::Initialize with spherecut = true
 * (fourier.cpp:542-640) and KohnSham::CalculateEkin's sphere branch
 * (hamiltonian.cpp:2630-2667).  numGrid is the G-space grid N (the density
 * grid: Density_Grid_Factor 1, src/esdf.cpp:2786-2856); N/2 must be a coarse
 * grid built into the library and the sphere must satisfy |m_d| <= N_d / 4.
 * After it, pw_ctx_sizes reports ntot = 2 ns and ntotFine = N.  Exact
 * exchange (pw_exx_*, pw_ace_*) runs on G-space contexts of either precision
 * (FP32: FP32 pair fields and transforms); k-points and forces are not built
 * for them (PW_EUNSUPPORTED). */
PW_API int pw_ctx_create_gspace(const double length[3], const int numGrid[3], double ecut, int precision, int device,
                                pw_ctx** out);
/* Sphere tables of a G-space context (host arrays, any may be NULL):
 * ns, idxCoarseCut (ns), signed Miller indices (3 ns), ekin and Teter (ns). */
PW_API int pw_gs_sphere(const pw_ctx* ctx, int* ns, int* idx_r2c, int* miller, double* ekin, double* teter);
/* Nonlocal projectors of EigenSolver::NonlocalMultX (KohnSham::vnlc_,
 * src/SCF/hamiltonian.cpp:700-797): vnlc (host, column-major ns x nproj
 * complex as interleaved doubles, sqrt(2) convention) and weights wgt (nproj).
 * pw_hpsi then adds vnlc (wgt o Re(vnlc^H c)).  pw_set_atoms on a G-space
 * context builds them from the library's HGH tables
 * (PeriodTable::CalculateNonlocalPP, Fourier space, src/SCF/periodtable.cpp:1599-1849). */
PW_API int pw_gs_set_projectors(pw_ctx* ctx, int nproj, const double* vnlc, const double* wgt);
/* The projector matrix a G-space context holds (host, as pw_gs_set_projectors
 * takes it); nproj may be queried with vnlc = wgt = NULL. */
PW_API int pw_gs_get_projectors(const pw_ctx* ctx, int* nproj, double* vnlc, double* wgt);

#ifdef __cplusplus
}
#endif
#endif /* PWDFT_B200_H */
