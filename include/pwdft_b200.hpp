// C++ host mirror of the reference's Hamiltonian / Spinor / EigenSolver
// interfaces over the C ABI of pwdft_b200.h, for a maintainer who swaps the
// reference's CPU path for this library inside its own C++ code.  Header
// only; link with libpwdft_b200.so.  Errors surface as std::runtime_error,
// the reference's ErrorHandling behaviour (src/global.cpp:71-88).
//
// Mirrored shapes:
//   * NumTns<Real>(ntot, ncom = 1, nband) column-major wavefunction blocks
//     (include/spinor.hpp:80): `BandBlock` is a non-owning view of the same layout.
//   * Hamiltonian::MultSpinor(Spinor&, NumTns<Real>& a3, Fourier&)
//     (include/hamiltonian.hpp:261): `Hamiltonian::MultSpinor` (a3 overwritten),
//     with the wavefunction filter state of KohnSham::set_wfn_filter
//     (include/hamiltonian.hpp:347-356).
//   * Spinor::AddTeterPrecond(Fourier*, teter, a3) (include/spinor.hpp:327):
//     `Hamiltonian::AddTeterPrecond` (a3 accumulated).
//   * EigenSolver::{LOBPCGSolveReal, PPCGSolveReal, DavidsonSolveReal} and
//     ChebFSI (include/eigensolver.hpp:113-191): `EigenSolver::Solve`.
//   * KohnSham::CalculateForce (src/SCF/hamiltonian.cpp:2670-3056): `Hamiltonian::Forces`.
#ifndef PWDFT_B200_HPP
#define PWDFT_B200_HPP

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "pwdft_b200.h"

namespace pwdft_b200 {

inline void check(int rc) {
  if (rc != PW_OK) throw std::runtime_error(std::string("pwdft_b200: ") + pw_last_error());
}

// Non-owning view of an ntot x nband column-major block of real numbers
// (host memory), the layout of the reference's NumTns<Real>(ntot, 1, nband).
struct BandBlock {
  double* data = nullptr;
  int ntot = 0;
  int nband = 0;
  double* VecData(int band) const { return data + (size_t)band * ntot; }
};

// Orthorhombic cell and grids (Domain::length, numGrid, numGridFine).
struct Domain {
  double length[3];
  int numGrid[3];
  int numGridFine[3];
  long NumGridTotal() const { return (long)numGrid[0] * numGrid[1] * numGrid[2]; }
  long NumGridTotalFine() const { return (long)numGridFine[0] * numGridFine[1] * numGridFine[2]; }
};

// Owns device copies of host band blocks for one call.
class DeviceBlock {
 public:
  DeviceBlock(size_t bytes) {
    if (bytes && cudaMalloc(&p_, bytes) != cudaSuccess) throw std::runtime_error("pwdft_b200: cudaMalloc failed");
  }
  ~DeviceBlock() {
    if (p_) cudaFree(p_);
  }
  DeviceBlock(const DeviceBlock&) = delete;
  DeviceBlock& operator=(const DeviceBlock&) = delete;
  void* get() const { return p_; }

 private:
  void* p_ = nullptr;
};

// KohnSham-like owner of one FP64 (or FP32) context: local potential,
// projectors (library HGH tables for Si / Al), H*psi, Teter, forces.
class Hamiltonian {
 public:
  Hamiltonian(const Domain& dm, int precision = PW_F64, int device = 0) : dm_(dm), prec_(precision) {
    check(pw_ctx_create(dm.length, dm.numGrid, dm.numGridFine, precision, device, &ctx_));
  }
  ~Hamiltonian() {
    if (ctx_) pw_ctx_destroy(ctx_);
  }
  Hamiltonian(const Hamiltonian&) = delete;
  Hamiltonian& operator=(const Hamiltonian&) = delete;

  pw_ctx* handle() const { return ctx_; }
  const Domain& domain() const { return dm_; }

  // PeriodTable::CalculateNonlocalPP / CalculatePseudoCharge for every atom
  void SetAtoms(const std::vector<int>& znuc, const std::vector<double>& pos_xyz) {
    check(pw_set_atoms(ctx_, (int)znuc.size(), znuc.data(), pos_xyz.data()));
  }
  // KohnSham::vtot_ (fine grid, host)
  void SetVtot(const double* vtot_fine) { check(pw_set_vtot(ctx_, vtot_fine)); }

  // KohnSham::set_wfn_filter(apply_filter, apply_first, wfn_cutoff)
  // (include/hamiltonian.hpp:347-352): with apply_filter the next MultSpinor
  // call with apply_first set replaces psi by P psi in place, and every
  // MultSpinor call returns a3 = P H psi (hamiltonian.cpp:3090-3116, 3240-3265).
  void set_wfn_filter(int apply_filter, int apply_first, double wfn_cutoff) {
    check(pw_set_wfn_filter(ctx_, apply_filter, wfn_cutoff));
    apply_filter_ = apply_filter != 0;
    apply_first_ = apply_first != 0;
  }
  // KohnSham::set_wfn_filter(apply_first) (include/hamiltonian.hpp:353-356)
  void set_wfn_filter(int apply_first) { apply_first_ = apply_first != 0; }

  // a3 := H psi (host blocks; FP64 contexts).  The view's bands are modified
  // only by the first call of a filtered Hamiltonian (psi <- P psi).
  void MultSpinor(const BandBlock& psi, BandBlock& a3) {
    require_f64();
    if (apply_filter_ && apply_first_) {
      apply_first_ = false;
      const size_t bytes = (size_t)psi.nband * psi.ntot * sizeof(double);
      DeviceBlock dx(bytes);
      cu(cudaMemcpy(dx.get(), psi.data, bytes, cudaMemcpyHostToDevice));
      check(pw_wfn_filter(ctx_, dx.get(), psi.ntot, psi.nband, nullptr));
      cu(cudaMemcpy(psi.data, dx.get(), bytes, cudaMemcpyDeviceToHost));
    }
    check(pw_hpsi_host(ctx_, psi.data, psi.ntot, a3.data, a3.ntot, psi.nband, 0));
  }
  // a3 += T r (host blocks; FP64 contexts)
  void AddTeterPrecond(const BandBlock& r, BandBlock& a3) {
    require_f64();
    const size_t bytes = (size_t)r.nband * r.ntot * sizeof(double);
    DeviceBlock dr(bytes), da(bytes);
    cu(cudaMemcpy(dr.get(), r.data, bytes, cudaMemcpyHostToDevice));
    cu(cudaMemcpy(da.get(), a3.data, bytes, cudaMemcpyHostToDevice));
    check(pw_teter_precond(ctx_, dr.get(), r.ntot, da.get(), a3.ntot, r.nband, 1, nullptr));
    cu(cudaMemcpy(a3.data, da.get(), bytes, cudaMemcpyDeviceToHost));
  }
  // KohnSham::CalculateForce from a host density and host bands (FP64)
  std::vector<double> Forces(const std::vector<double>& rho_fine, const BandBlock& psi, const std::vector<double>& occ,
                             int num_spin = 2) {
    require_f64();
    const size_t bp = (size_t)psi.nband * psi.ntot * sizeof(double), br = rho_fine.size() * sizeof(double);
    DeviceBlock dp(bp), dr(br);
    cu(cudaMemcpy(dp.get(), psi.data, bp, cudaMemcpyHostToDevice));
    cu(cudaMemcpy(dr.get(), rho_fine.data(), br, cudaMemcpyHostToDevice));
    int natom = 0;
    check(pw_ctx_natom(ctx_, &natom));
    std::vector<double> f((size_t)natom * 3);
    check(pw_forces(ctx_, (const double*)dr.get(), dp.get(), psi.ntot, psi.nband, occ.data(), num_spin, f.data(),
                    nullptr, nullptr));
    return f;
  }

 private:
  static void cu(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("pwdft_b200: ") + cudaGetErrorString(e));
  }
  void require_f64() const {
    if (prec_ != PW_F64) throw std::runtime_error("pwdft_b200: host-block entry points take an FP64 context");
  }
  Domain dm_;
  int prec_;
  pw_ctx* ctx_ = nullptr;
  bool apply_filter_ = false, apply_first_ = false;
};

// EigenSolver over a Hamiltonian: the lowest nband eigenpairs from the host
// block psi (overwritten by the Ritz vectors), as LOBPCGSolveReal /
// PPCGSolveReal / DavidsonSolveReal / ChebFSI do on the reference's Spinor.
class EigenSolver {
 public:
  explicit EigenSolver(Hamiltonian& ham) : ham_(ham) {}
  // solver: PW_SOLVER_*; param: ChebFSI degree, PPCG sub-block size or Davidson blocks
  std::vector<double> Solve(BandBlock& psi, int solver, int maxit, double tol, int param = 10,
                            std::vector<double>* resnorm = nullptr) {
    const size_t bytes = (size_t)psi.nband * psi.ntot * sizeof(double);
    DeviceBlock dx(bytes);
    if (cudaMemcpy(dx.get(), psi.data, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("pwdft_b200: copy failed");
    std::vector<double> eig(psi.nband), res(psi.nband);
    int it = 0;
    check(pw_eigsolve(ham_.handle(), solver, dx.get(), psi.nband, maxit, tol, param, eig.data(), res.data(), &it));
    if (cudaMemcpy(psi.data, dx.get(), bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("pwdft_b200: copy failed");
    if (resnorm) *resnorm = res;
    iterations_ = it;
    return eig;
  }
  int iterations() const { return iterations_; }

 private:
  Hamiltonian& ham_;
  int iterations_ = 0;
};

}  // namespace pwdft_b200

#endif  // PWDFT_B200_HPP
