// Shared declarations for the pwdft_b200 native library.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/pwdft_b200.h"
#include "pseudo.hpp"

namespace pwb {

// Last error message of the calling thread (returned by pw_last_error()).
void set_error(const std::string& msg);

#define PWB_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      ::pwb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
      return PW_ECUDA;                                                              \
    }                                                                               \
  } while (0)

#define PWB_CHECK(cond, code, msg)                                                  \
  do {                                                                              \
    if (!(cond)) {                                                                  \
      ::pwb::set_error(msg);                                                        \
      return (code);                                                                \
    }                                                                               \
  } while (0)

// A one-time set-up step (kernel attributes) tracked per device: cudaFuncSetAttribute
// applies to the current device only, so a process that drives several GPUs
// repeats the step once on each of them.
struct PerDeviceOnce {
  std::atomic<unsigned long long> bits{0};
  static int dev() {
    int d = 0;
    cudaGetDevice(&d);
    return d & 63;
  }
  bool done() const { return (bits.load(std::memory_order_acquire) >> dev()) & 1ull; }
  void mark() { bits.fetch_or(1ull << dev(), std::memory_order_release); }
};

// Device buffer owned by a context.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int alloc(size_t nbytes);
  void release();
  ~DevBuf() { release(); }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// Nonlocal projector tables in the fine-plane ("tile") sorted layout used by
// the gather / apply kernels.  A tile is one fine z-plane and one chunk of
// CR rows; within a tile entries are grouped by atom ("slots").
struct NonlocalDev {
  int natom = 0, npmax = 0, nent = 0, nslot = 0, ntile = 0, cr = 0, nchunk = 0;
  DevBuf ent_xy;          // int32 [nent]   y*NX + x (fine plane coordinates)
  DevBuf ent_beta;        // T     [npmax][nent] projector values (VAL column)
  DevBuf tile_slot;       // int32 [ntile+1]
  DevBuf slot_atom;       // int32 [nslot]
  DevBuf slot_ent;        // int32 [nslot+1]
  DevBuf atom_slot;       // int32 [natom+1]
  DevBuf atom_slot_list;  // int32 [nslot]
  DevBuf wgt;             // T     [natom*npmax]  gamma * vol / N_fine
};

// Kernel kinds for pw_profile_read.
enum KernelKind {
  KK_CXY_FWD = 0, KK_ZPAD, KK_FPLANE_GATHER, KK_NL_REDUCE, KK_FPLANE_APPLY, KK_ZFOLD, KK_CXY_INV, KK_ZTETER,
  KK_GRAM, KK_DENSITY, KK_MISC, KK_LIBGEMM, KK_EXX, KK_ROT, KK_COUNT
};

// A dense coarse-grid operator Q diag(qd) Q^T: the projector matrix, or the
// ACE vectors with qd = -1.  q: T [np][ntot]; q_bf / qt_bf: split-BF16 copies
// (FP32 contexts) of Q (np x ntot) and Q^T (ntot x npp, npp = np padded to 8).
// q_st is the matrix the accumulating (store) product reads -- Q itself, or
// P Q while the wavefunction cut-off filter is on (qt_bf then holds P Q too).
struct DenseSet {
  const void* q;
  const void* qd;
  const void* q_bf;
  const void* qt_bf;
  int np, npp;
  const void* q_st;
};

}  // namespace pwb

// Opaque context behind the C ABI.
struct pw_ctx {
  int prec = PW_F64;            // PW_F64 or PW_F32 storage / arithmetic
  double L[3] = {0, 0, 0};      // orthorhombic cell lengths (bohr)
  double vol = 0;
  int n[3] = {0, 0, 0};         // coarse (wavefunction) grid
  int nf[3] = {0, 0, 0};        // fine (density) grid
  long ntot = 0, ntotf = 0;
  int device = 0;
  size_t esz = 8;               // bytes per real
  // Fourier tables
  pwb::DevBuf ekin;             // T [n2][n1][n0]  |G|^2/2 on the full coarse spectrum
  pwb::DevBuf teter;            // T [n2][n1][n0]
  pwb::DevBuf vtot;             // T [N_fine]
  pwb::DevBuf vperm;            // T: vtot in the lane order of the fused fine-plane kernel's
                                //    row pass (fft_variant 2), rebuilt whenever vtot is written
  pwb::DevBuf tw[6];            // complex T twiddles for n0,n1,n2,nf0,nf1,nf2
  bool have_vtot = false;
  bool have_nl = false;
  pwb::NonlocalDev nl;
  // nonlocal apply mode: PW_NL_DENSE (coarse-grid projector matrix, GEMMs) or
  // PW_NL_REALSPACE (fine-grid gather / scatter over the projector index sets)
  int nl_mode = PW_NL_DENSE;
  int nproj = 0;                 // total projectors over all atoms
  pwb::DevBuf q;                 // T [nproj][ntot]  coarse projector columns q_l
  pwb::DevBuf qd;                // T [nproj]        gamma_l * vol / ntot
  pwb::DevBuf s_wq;              // T [nproj][band batch] projections
  void* blas = nullptr;          // cublasHandle_t
  // FP32 contexts: bf16 hi/lo copies of Q ([l][g]) and Q^T ([g][l], rows padded
  // to nproj_pad) for the split-BF16 tensor-core GEMMs
  int gemm_terms = 3;            // split products per k-step (3 or 4)
  int gemm_bn = 0, gemm_bn_store = 0;   // projector GEMM tile widths (0: heuristic; set by pw_autotune)
  int fft_variant = 2;           // form of the fused fine-plane transforms (0 / 1 / 2; set by pw_autotune)
  bool check_errors = false;     // read the device error flag after each call (synchronises)
  pw_ctx* twin = nullptr;        // FP32 twin of an FP64 context (mixed-precision SCF), owned
  int nproj_pad = 0;
  pwb::DevBuf q_bf, qt_bf, s_psi_bf, s_w_bf, s_ws, s_gx_bf, s_gy_bf, s_rot, s_rot_x;
  // host copies kept for setup-time work
  std::vector<double> h_vtot;
  // atoms set through pw_set_atoms (HGH species built in this library)
  std::vector<int> atom_z;
  std::vector<double> atom_pos;            // natom x 3, Cartesian bohr
  std::vector<pwb::AtomNL> h_nl;           // per-atom vnlList incl. DX/DY/DZ columns
  std::vector<double> h_rhops;             // pseudocharge on the fine grid
  std::vector<long> h_ps_off;              // natom + 1 offsets into h_ps_idx / h_ps_val
  std::vector<int> h_ps_idx;               // per-atom pseudocharge support (fine-grid index)
  std::vector<double> h_ps_val;            // per-atom pseudocharge values
  // k-point mode: complex bands at Bloch vector kvec (AddMultSpinorFine, complex)
  bool have_k = false;
  double kvec[3] = {0.0, 0.0, 0.0};
  pwb::DevBuf ekin_k, teter_k;      // T [ntot]  1/2 |k+G|^2 and Teter on the full coarse spectrum
  pwb::DevBuf qk;                   // complex T [nproj][ntot]  projectors with the Bloch phase
  pwb::DevBuf qdk;                  // T [nproj]  gamma_l * vol / ntot
  int nkb = 0;                      // k-point batch (pw_set_kpoints)
  std::vector<double> kb_k;         // nkb x 3
  pwb::DevBuf ekin_kb, qkb;         // T [nkb][ntot], complex T [nkb][nproj][ntot]
  // FP32 contexts: the complex projector products as real split-BF16 GEMMs.  Per
  // k-point: A1 = [Q; Q'] as real rows (2 nproj x 2 ntot, Q' = i Q, so that
  // A1 psi = [Re; Im] of Q^H psi) and A2 = its store-side partner (2 ntot x
  // nkp2 rows: (Re, Im) of Q W from [Re W; Im W]), each as bf16 hi / lo
  pwb::DevBuf qk_bf, qkb_bf;        // single k (pw_set_kpoint) / batch (pw_set_kpoints)
  pwb::DevBuf qdk2;                 // float [2 nproj]  the weights twice (rows of A1)
  int nkp2 = 0;                     // 2 nproj rounded up to 8
  // sphere-cut (G-space) mode (Use_Real_Space 0): a band is its half-sphere
  // Fourier coefficients, complex, handled as a real vector of 2 ns numbers
  // (ntot = 2 ns); n = N/2 is the slot box and nf = N the G-space grid
  bool gs = false;
  double gs_ecut = 0.0;
  int gs_ns = 0;
  pwb::DevBuf gs_rows_inv, gs_ent_inv;   // scatter lists: int [n1+2] row offsets, int2 entries
  pwb::DevBuf gs_rows_fwd, gs_ent_fwd;   // gather lists: int [n1/2+2] block offsets, int2 entries
  pwb::DevBuf gs_ekin, gs_teter;    // T [ns]
  std::vector<int> h_gs_idx;        // idxCoarseCut: flat R2C index of each sphere point
  std::vector<int> h_gs_m;          // 3 signed Miller indices per sphere point
  // hybrid exchange (AddMultSpinorEXX / CalculateVexxACE)
  int exx_mode = 0;                 // PW_EXX_OFF / PW_EXX_FULL / PW_EXX_ACE
  double exx_frac = 0.0, exx_mu = 0.0, exx_div = 0.0;
  pwb::DevBuf exx_kern;             // T [ntot]  Coulomb kernel on the full coarse spectrum
  pwb::DevBuf exx_phi;              // T [nphi][ntot]  phi = sqrt(N_c / vol) psi
  pwb::DevBuf exx_w;                // T [nphi]  -exx_frac * occupation
  std::vector<double> exx_occ;      // host copy of the occupations of phi
  int exx_nphi = 0;
  pwb::DevBuf s_exx;                // pair-field scratch
  size_t exx_scratch_bytes = (size_t)1 << 30;
  pwb::DevBuf ace_xi, ace_qd, ace_bf, ace_t_bf;   // ACE vectors xi (T [nace][ntot]) and -1 weights
  int ace_n = 0, ace_npad = 0;
  // wavefunction cut-off filter of KohnSham::MultSpinor (the CheFSI path): while
  // on, an overwriting H*psi returns P H psi, P = C2R o (zero |G|^2/2 > wfn_ecut) o R2C
  bool wfn_filter = false;
  double wfn_ecut = 0.0;
  pwb::DevBuf wmask;                // T [ntot]  1 where |G|^2/2 <= wfn_ecut on the full coarse spectrum, else 0
  long q_version = 0, ace_version = 0;           // bumped when Q / the ACE vectors are rebuilt
  long qf_version = -1, acef_version = -1;       // versions the filtered copies below were made from
  double qf_ecut = -1.0, acef_ecut = -1.0;
  pwb::DevBuf qf, qtf_bf;           // P Q and its split-BF16 transpose (store side of the projector GEMMs)
  pwb::DevBuf acef_xi, acef_t_bf;   // P xi and its split-BF16 transpose (store side of the ACE GEMMs)
  const void* teter_tab = nullptr;  // table of the next Teter-pipeline pass (nullptr: the Teter table)
  // initial guess for the next pw_scf_run (pw_scf_set_initial, e.g. from restart files)
  std::vector<double> init_rho, init_psi;
  int init_nband = 0;
  // converged SCF state kept for pw_scf_forces: FP64 bands, occupations, density
  pwb::DevBuf scf_psi, scf_rho;
  std::vector<double> scf_occ;
  int scf_nband = 0;
  // flattened projector sets as last passed to pw_set_nonlocal (for forces)
  std::vector<int> h_nl_idx, h_pnp, h_patom;
  std::vector<double> h_nl_beta, h_pgamma;
  std::vector<long> h_pio, h_pbo;
  // kernel launch accounting (pw_stats) and optional per-kernel event timing
  long launches = 0;
  long lib_launches = 0;          // cuBLAS / cuSOLVER calls (not this library's kernels)
  bool prof_on = false;
  struct ProfRec { int kind; cudaEvent_t a, b; };
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> ev_pool;
  // scratch for the band-pair pipeline
  int pair_cap = 0;
  pwb::DevBuf s_ad, s_k, s_bc, s_wp, s_w;
  pwb::DevBuf s_host_in, s_host_out;   // device staging for the host-pointer entry points
  pwb::DevBuf gs_full_idx, gs_exx_tw;   // G-space exchange: full-grid index of G_s and -G_s, N-point twiddles
  pwb::DevBuf gsx_psir, gsx_phir, gsx_acc, gsx_fields;   // G-space exchange workspace (real fields, pair fields)
  bool gsx_phi_ready = false;            // gsx_phir holds phi(r) of the current exchange orbitals
  cudaStream_t io_st[3] = {nullptr, nullptr, nullptr};   // host->device, compute, device->host (pw_hpsi_host)
  int host_chunk = 32;                                    // bands per pw_hpsi_host chunk
  // dense projector mode: the projector GEMMs of an H*psi batch on their own
  // stream alongside the FFT chain (pw_set_nl_overlap; set per precision at creation)
  int nl_overlap = 1;
  cudaStream_t nl_st = nullptr;
  cudaEvent_t nl_fork = nullptr, nl_join = nullptr;
  void* scf_cache = nullptr;                              // pw_scf_run workspace kept between runs
  void (*scf_cache_free)(void*) = nullptr;
};

namespace pwb {

// One kernel (or library GEMM) launch: counted for pw_stats and, with
// pw_profile on, bracketed by CUDA events on its stream.
struct Launch {
  pw_ctx* c;
  cudaStream_t st;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  static cudaEvent_t take(pw_ctx* c) {
    if (!c->ev_pool.empty()) {
      cudaEvent_t e = c->ev_pool.back();
      c->ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  Launch(pw_ctx* c_, cudaStream_t st_, int kind_) : c(c_), st(st_), kind(kind_) {
    if (kind == KK_LIBGEMM) c->lib_launches++; else c->launches++;
    if (c->prof_on) {
      a = take(c);
      b = take(c);
      cudaEventRecord(a, st);
    }
  }
  ~Launch() {
    if (a) {
      cudaEventRecord(b, st);
      c->prof.push_back({kind, a, b});
    }
  }
};

// exact exchange of sphere-cut (G-space) FP64 contexts (gs_exx.cu)
int gs_exx_setup(pw_ctx* c, double frac, double mu, int divergence_type, double ecut);
int gs_exx_apply(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int accumulate, cudaStream_t st);

}  // namespace pwb
