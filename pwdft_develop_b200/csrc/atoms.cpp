// C ABI for atom set-up with the library's own HGH tables: builds the
// nonlocal projector sets (PeriodTable::CalculateNonlocalPP,
// src/SCF/periodtable.cpp:994-1240) and the pseudocharge
// (PeriodTable::CalculatePseudoCharge, periodtable.cpp:282-377) for every atom,
// as KohnSham::CalculatePseudoPotential does (src/SCF/hamiltonian.cpp:327-918).
#include <cstring>

#include "common.hpp"

namespace pwb {
int gs_set_atoms(pw_ctx* c);
}

using namespace pwb;

extern "C" {

int pw_hgh_species(int znuc, double* zion, double* eself, double* rcut_nonlocal, double* rcut_rho, int* nproj) {
  const Species* sp = species(znuc);
  PWB_CHECK(sp, PW_EUNSUPPORTED, "HGH table only built for Si (14) and Al (13)");
  int np = 0;
  for (const auto& p : sp->proj) np += (p.l == 0) ? 1 : 3;
  if (zion) *zion = sp->zion;
  if (eself) *eself = sp->eself;
  if (rcut_nonlocal) *rcut_nonlocal = sp->wavcut;
  if (rcut_rho) *rcut_rho = sp->rhocut;
  if (nproj) *nproj = np;
  return PW_OK;
}

int pw_set_atoms(pw_ctx* ctx, int natom, const int* znuc, const double* pos) {
  PWB_CHECK(ctx && natom >= 0 && (natom == 0 || (znuc && pos)), PW_EINVAL, "bad arguments");
  std::vector<AtomNL> nl(natom);
  std::vector<double> rhops(ctx->ntotf, 0.0);
  std::vector<long> ps_off(1, 0);
  std::vector<int> ps_idx;
  std::vector<double> ps_val;
  for (int a = 0; a < natom; ++a) {
    const Species* sp = species(znuc[a]);
    PWB_CHECK(sp, PW_EUNSUPPORTED, "HGH table only built for Si (14) and Al (13)");
    int rc = ctx->gs ? PW_OK : nonlocal_pp(*sp, pos + 3 * a, ctx->L, ctx->nf, nl[a]);
    if (rc) return rc;
    AtomRho rho;
    rc = pseudo_charge(*sp, pos + 3 * a, ctx->L, ctx->nf, rho);
    if (rc) return rc;
    for (size_t i = 0; i < rho.idx.size(); ++i) {
      rhops[rho.idx[i]] += rho.val[4 * i];
      ps_idx.push_back(rho.idx[i]);
      ps_val.push_back(rho.val[4 * i]);
    }
    ps_off.push_back((long)ps_idx.size());
  }
  if (ctx->gs) {
    // sphere-cut context: Fourier-space projectors (PeriodTable::CalculateNonlocalPP,
    // src/SCF/periodtable.cpp:1599-1849) instead of the real-space sets
    ctx->atom_z.assign(znuc, znuc + natom);
    ctx->atom_pos.assign(pos, pos + 3 * natom);
    int rc = gs_set_atoms(ctx);
    if (rc) return rc;
    ctx->h_nl.clear();
    ctx->h_rhops = std::move(rhops);
    ctx->h_ps_off = std::move(ps_off);
    ctx->h_ps_idx = std::move(ps_idx);
    ctx->h_ps_val = std::move(ps_val);
    return PW_OK;
  }
  std::vector<int> npts(natom), nproj(natom), idx;
  std::vector<double> beta, wgt;
  for (int a = 0; a < natom; ++a) {
    npts[a] = nl[a].npts;
    nproj[a] = (int)nl[a].val.size();
    idx.insert(idx.end(), nl[a].idx.begin(), nl[a].idx.end());
    for (int q = 0; q < nproj[a]; ++q)
      for (int g = 0; g < npts[a]; ++g) beta.push_back(nl[a].val[q][4 * g]);
    wgt.insert(wgt.end(), nl[a].wgt.begin(), nl[a].wgt.end());
  }
  int rc = pw_set_nonlocal(ctx, natom, npts.data(), nproj.data(), idx.data(), beta.data(), wgt.data());
  if (rc) return rc;
  ctx->atom_z.assign(znuc, znuc + natom);
  ctx->atom_pos.assign(pos, pos + 3 * natom);
  ctx->h_nl = std::move(nl);
  ctx->h_rhops = std::move(rhops);
  ctx->h_ps_off = std::move(ps_off);
  ctx->h_ps_idx = std::move(ps_idx);
  ctx->h_ps_val = std::move(ps_val);
  return PW_OK;
}

int pw_ctx_natom(const pw_ctx* ctx, int* natom) {
  PWB_CHECK(ctx && natom, PW_EINVAL, "null argument");
  *natom = (int)ctx->atom_z.size();
  return PW_OK;
}

int pw_get_pseudocharge(const pw_ctx* ctx, double* rho_fine_host) {
  PWB_CHECK(ctx && rho_fine_host, PW_EINVAL, "null argument");
  PWB_CHECK(ctx->h_rhops.size() == (size_t)ctx->ntotf, PW_ENOTREADY, "atoms not set (pw_set_atoms)");
  std::memcpy(rho_fine_host, ctx->h_rhops.data(), ctx->ntotf * sizeof(double));
  return PW_OK;
}

int pw_get_atom_projectors(const pw_ctx* ctx, int atom, int* npts, int* nproj, int* idx, double* val4,
                           double* wgt) {
  PWB_CHECK(ctx && atom >= 0 && atom < (int)ctx->h_nl.size(), PW_EINVAL, "bad atom index");
  const AtomNL& a = ctx->h_nl[atom];
  if (npts) *npts = a.npts;
  if (nproj) *nproj = (int)a.val.size();
  if (idx) std::memcpy(idx, a.idx.data(), a.idx.size() * sizeof(int));
  if (val4)
    for (size_t q = 0; q < a.val.size(); ++q) std::memcpy(val4 + q * 4 * a.npts, a.val[q].data(), 4 * a.npts * sizeof(double));
  if (wgt) std::memcpy(wgt, a.wgt.data(), a.wgt.size() * sizeof(double));
  return PW_OK;
}

int pw_hgh_atom_projectors(const double length[3], const int numGridFine[3], int znuc, const double pos[3],
                           int* npts, int* nproj, int* idx, double* val4, double* wgt) {
  PWB_CHECK(length && numGridFine && pos, PW_EINVAL, "null argument");
  const Species* sp = species(znuc);
  PWB_CHECK(sp, PW_EUNSUPPORTED, "HGH table only built for Si (14) and Al (13)");
  AtomNL a;
  int rc = nonlocal_pp(*sp, pos, length, numGridFine, a);
  if (rc) return rc;
  if (npts) *npts = a.npts;
  if (nproj) *nproj = (int)a.val.size();
  if (idx) std::memcpy(idx, a.idx.data(), a.idx.size() * sizeof(int));
  if (val4)
    for (size_t q = 0; q < a.val.size(); ++q) std::memcpy(val4 + q * 4 * a.npts, a.val[q].data(), 4 * a.npts * sizeof(double));
  if (wgt) std::memcpy(wgt, a.wgt.data(), a.wgt.size() * sizeof(double));
  return PW_OK;
}

int pw_hgh_pseudocharge(const double length[3], const int numGridFine[3], int natom, const int* znuc,
                        const double* pos, double* rho_fine_host) {
  PWB_CHECK(length && numGridFine && rho_fine_host && (natom == 0 || (znuc && pos)), PW_EINVAL, "null argument");
  const long nf = (long)numGridFine[0] * numGridFine[1] * numGridFine[2];
  for (long i = 0; i < nf; ++i) rho_fine_host[i] = 0.0;
  for (int a = 0; a < natom; ++a) {
    const Species* sp = species(znuc[a]);
    PWB_CHECK(sp, PW_EUNSUPPORTED, "HGH table only built for Si (14) and Al (13)");
    AtomRho r;
    int rc = pseudo_charge(*sp, pos + 3 * a, length, numGridFine, r);
    if (rc) return rc;
    for (size_t i = 0; i < r.idx.size(); ++i) rho_fine_host[r.idx[i]] += r.val[4 * i];
  }
  return PW_OK;
}

int pw_stats(const pw_ctx* ctx, long* kernel_launches, long* library_calls) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  if (kernel_launches) *kernel_launches = ctx->launches;
  if (library_calls) *library_calls = ctx->lib_launches;
  return PW_OK;
}

}  // extern "C"
