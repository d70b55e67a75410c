// Restart files in the reference's binary layout and the SCF initial guess.
//
// The reference writes its restart data with serialize() (include/utility.hpp:
// 1183-1278): a vector is an int32 length followed by that many doubles, a
// matrix two int32 sizes then the column-major doubles, a 3-tensor three
// int32 sizes then the doubles, all in the machine's native byte order.
//   DEN   three grid vectors (fractional positions posStart + i / N_d, UniformMeshFine,
//         src/utility.cpp:405-420) then the density vector (src/SCF/scf.cpp:1070-1088;
//         read back at scf.cpp:164-178)
//   POT   the same grid vectors then Vtot as an N_fine x 1 matrix (scf.cpp:1091-1108)
//   WFN_<rank>  the bands as an ntot x 1 x nband tensor, then the occupations
//         (scf.cpp:1110-1145 through SeparateWrite, "name_<rank>", utility.cpp:499-510;
//         read back at scf.cpp:296-330)
//   EIG   the eigenvalues as one vector (scf.cpp:1247-1253)
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "common.hpp"

using namespace pwb;

namespace {

bool put_i32(std::ofstream& f, int v) {
  const int32_t x = v;
  f.write(reinterpret_cast<const char*>(&x), 4);
  return f.good();
}
bool put_vec(std::ofstream& f, const double* v, long n) {
  if (!put_i32(f, (int)n)) return false;
  f.write(reinterpret_cast<const char*>(v), n * 8);
  return f.good();
}
bool get_i32(std::ifstream& f, int& v) {
  int32_t x = 0;
  f.read(reinterpret_cast<char*>(&x), 4);
  v = x;
  return f.good();
}
bool get_vec(std::ifstream& f, std::vector<double>& v) {
  int n = 0;
  if (!get_i32(f, n) || n < 0) return false;
  v.resize(n);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)n * 8);
  return f.good() || (n == 0 && !f.bad());
}

// UniformMeshFine with posStart = 0
void write_grid(std::ofstream& f, const pw_ctx* c) {
  for (int d = 0; d < 3; ++d) {
    std::vector<double> g(c->nf[d]);
    for (int i = 0; i < c->nf[d]; ++i) g[i] = (double)i / c->nf[d];
    put_vec(f, g.data(), (long)g.size());
  }
}
int read_grid(std::ifstream& f, const pw_ctx* c) {
  for (int d = 0; d < 3; ++d) {
    std::vector<double> g;
    PWB_CHECK(get_vec(f, g), PW_EINVAL, "restart file: truncated grid vector");
    PWB_CHECK((int)g.size() == c->nf[d], PW_EINVAL, "restart file: fine grid does not match the context");
  }
  return PW_OK;
}

}  // namespace

extern "C" {

int pw_write_density(const pw_ctx* ctx, const char* path, const double* rho) {
  PWB_CHECK(ctx && path && rho, PW_EINVAL, "null argument");
  std::ofstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("Density file cannot be opened: ") + path);
  write_grid(f, ctx);
  PWB_CHECK(put_vec(f, rho, ctx->ntotf), PW_EINVAL, "writing the density failed");
  return PW_OK;
}

int pw_read_density(const pw_ctx* ctx, const char* path, double* rho) {
  PWB_CHECK(ctx && path && rho, PW_EINVAL, "null argument");
  std::ifstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("File cannot be open: ") + path);
  int rc = read_grid(f, ctx);
  if (rc) return rc;
  std::vector<double> v;
  PWB_CHECK(get_vec(f, v), PW_EINVAL, "restart file: truncated density");
  PWB_CHECK((long)v.size() == ctx->ntotf, PW_EINVAL, "restart file: density size does not match the fine grid");
  std::memcpy(rho, v.data(), v.size() * 8);
  return PW_OK;
}

int pw_write_potential(const pw_ctx* ctx, const char* path, const double* vtot) {
  PWB_CHECK(ctx && path && vtot, PW_EINVAL, "null argument");
  std::ofstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("Potential file cannot be opened: ") + path);
  write_grid(f, ctx);
  put_i32(f, (int)ctx->ntotf);
  put_i32(f, 1);
  f.write(reinterpret_cast<const char*>(vtot), ctx->ntotf * 8);
  PWB_CHECK(f.good(), PW_EINVAL, "writing the potential failed");
  return PW_OK;
}

int pw_write_wfn(const pw_ctx* ctx, const char* path, const double* psi, int ld, int nband, const double* occ) {
  PWB_CHECK(ctx && path && (nband == 0 || (psi && occ)) && nband >= 0 && ld >= ctx->ntot, PW_EINVAL,
            "bad arguments");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "the WFN layout holds real-space bands (real-space contexts only)");
  std::ofstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("File cannot be open: ") + path);
  put_i32(f, (int)ctx->ntot);
  put_i32(f, 1);
  put_i32(f, nband);
  for (int b = 0; b < nband; ++b) f.write(reinterpret_cast<const char*>(psi + (long)b * ld), ctx->ntot * 8);
  PWB_CHECK(put_vec(f, occ, nband), PW_EINVAL, "writing the wavefunctions failed");
  return PW_OK;
}

int pw_read_wfn(const pw_ctx* ctx, const char* path, double* psi, int ld, int nband_max, int* nband, double* occ) {
  PWB_CHECK(ctx && path && nband, PW_EINVAL, "null argument");
  PWB_CHECK(!ctx->gs, PW_EUNSUPPORTED, "the WFN layout holds real-space bands (real-space contexts only)");
  std::ifstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("File cannot be open: ") + path);
  int m = 0, n = 0, p = 0;
  PWB_CHECK(get_i32(f, m) && get_i32(f, n) && get_i32(f, p), PW_EINVAL, "restart file: truncated tensor header");
  PWB_CHECK(m == ctx->ntot && n == 1 && p >= 0, PW_EINVAL, "restart file: band layout does not match the context");
  *nband = p;
  if (!psi) return PW_OK;   // size query
  PWB_CHECK(p <= nband_max && ld >= ctx->ntot, PW_EINVAL, "restart file: more bands than the buffer holds");
  for (int b = 0; b < p; ++b) {
    f.read(reinterpret_cast<char*>(psi + (long)b * ld), (std::streamsize)m * 8);
    PWB_CHECK(f.good(), PW_EINVAL, "restart file: truncated bands");
  }
  std::vector<double> o;
  PWB_CHECK(get_vec(f, o) && (int)o.size() == p, PW_EINVAL, "restart file: occupations do not match the bands");
  if (occ) std::memcpy(occ, o.data(), o.size() * 8);
  return PW_OK;
}

int pw_write_eig(const char* path, int n, const double* eig) {
  PWB_CHECK(path && n >= 0 && (n == 0 || eig), PW_EINVAL, "bad arguments");
  std::ofstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("Eigenvalue file cannot be opened: ") + path);
  PWB_CHECK(put_vec(f, eig, n), PW_EINVAL, "writing the eigenvalues failed");
  return PW_OK;
}

int pw_read_eig(const char* path, int nmax, int* n, double* eig) {
  PWB_CHECK(path && n, PW_EINVAL, "null argument");
  std::ifstream f(path, std::ios::binary);
  PWB_CHECK(f.good(), PW_EINVAL, std::string("File cannot be open: ") + path);
  std::vector<double> v;
  PWB_CHECK(get_vec(f, v), PW_EINVAL, "restart file: truncated eigenvalues");
  *n = (int)v.size();
  if (!eig) return PW_OK;
  PWB_CHECK((int)v.size() <= nmax, PW_EINVAL, "more eigenvalues than the buffer holds");
  std::memcpy(eig, v.data(), v.size() * 8);
  return PW_OK;
}

int pw_scf_set_initial(pw_ctx* ctx, const double* rho, const double* psi, int ld, int nband) {
  PWB_CHECK(ctx, PW_EINVAL, "null context");
  ctx->init_rho.clear();
  ctx->init_psi.clear();
  ctx->init_nband = 0;
  if (rho) ctx->init_rho.assign(rho, rho + ctx->ntotf);
  if (psi) {
    PWB_CHECK(nband > 0 && ld >= ctx->ntot, PW_EINVAL, "bad band block");
    ctx->init_psi.resize((size_t)nband * ctx->ntot);
    for (int b = 0; b < nband; ++b)
      std::memcpy(ctx->init_psi.data() + (size_t)b * ctx->ntot, psi + (long)b * ld, ctx->ntot * 8);
    ctx->init_nband = nband;
  }
  return PW_OK;
}

}  // extern "C"
