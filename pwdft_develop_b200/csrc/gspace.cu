// Sphere-cut (G-space) contexts: the reference's Use_Real_Space: 0 mode.
//
//   * sphere maps        Fourier::Initialize with spherecut (src/SCF/fourier.cpp:542-640)
//   * ekin / Teter        KohnSham::CalculateEkin sphere branch (src/SCF/hamiltonian.cpp:2630-2667)
//   * projector matrix    PeriodTable::CalculateNonlocalPP, Fourier space
//                         (src/SCF/periodtable.cpp:1599-1849) assembled into
//                         KohnSham::vnlc_ (src/SCF/hamiltonian.cpp:700-797)
//   * Teter               Spinor::AddTeterPrecond, complex (src/SCF/spinor.cpp:349-374)
//
// H*psi itself (Spinor::AddMultSpinorFineR2C complex overload plus
// EigenSolver::NonlocalMultX) is Plan::hpsi_gs_batch in pipeline.cuh.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <cmath>
#include <string>
#include <vector>

#include "common.hpp"
#include "fft.cuh"
#include "grid_registry.hpp"

namespace pwb {

int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n);
int upload_twiddles(pw_ctx* c, int slot, int n);
int ensure_scratch(pw_ctx* c, int npair);
int install_dense_q(pw_ctx* ctx, int nproj);

namespace {

// slot of a signed frequency f in [-n/2, n/2]; the fine (G-space grid)
// index of a slot; the slot of the opposite frequency
inline int slot_of(int f, int n) { return f >= 0 ? f : (f == -n / 2 ? n : n + f); }
inline int slot_to_fine(int s, int n, int nf) { return s <= n / 2 ? s : (s < n ? nf - n + s : nf - n / 2); }
inline int mirror_slot(int s, int n) { return s == 0 ? 0 : (s == n / 2 ? n : (s == n ? n / 2 : n - s)); }
inline int kgrid(int i, int n) { return i <= n / 2 ? i : i - n; }

template <typename T>
__global__ void k_gs_teter(const T* __restrict__ r, int ld, T* __restrict__ out, int ldo, long n2s,
                           const T* __restrict__ teter, int accumulate) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n2s) return;
  const long b = blockIdx.y;
  const T v = r[b * ld + i] * teter[i >> 1];
  T* o = out + b * ldo + i;
  *o = accumulate ? *o + v : v;
}

// ---------------------------------------------------------------------------
// Fourier-space HGH projectors (periodtable.cpp:1599-1849)
// ---------------------------------------------------------------------------
constexpr double kRab = 0.01;   // uniform radial mesh of the r*beta(r) samples
constexpr double kDq = 0.01;    // q-table step (periodtable.cpp:1611)

double double_factorial(int n) {
  double r = 1.0;
  for (; n > 1; n -= 2) r *= n;
  return r;
}

// spherical Bessel j_l, l = 0, 1 (src/utility.cpp:4314-4380)
double bessel(int l, double x) {
  const double ax = std::fabs(x);
  if (ax < 1e-16) return l == 0 ? 1.0 : 0.0;
  if (ax <= 0.05) {
    const double x2 = x * x;
    return std::pow(x, l) / double_factorial(2 * l + 1) *
           (1 - x2 / 1.0 / 2.0 / (2.0 * l + 3.0) *
                    (1 - x2 / 2.0 / 2.0 / (2.0 * l + 5.0) *
                             (1 - x2 / 3.0 / 2.0 / (2.0 * l + 7.0) * (1 - x2 / 4.0 / 2.0 / (2.0 * l + 9.0)))));
  }
  if (l == 0) return std::sin(x) / x;
  return (std::sin(x) / x - std::cos(x)) / x;
}

// src/utility.cpp:3329-3338
double simpson(const std::vector<double>& f, double rab) {
  double s = 0.0;
  for (size_t i = 0; i + 2 < f.size(); i += 2) s += (f[i] + 4 * f[i + 1] + f[i + 2]) / 3.0 * rab;
  return s;
}

struct Channel {
  int l;
  double h;
  std::vector<double> tab;
};

// per projector channel: tab(j) = int r^2 beta(r) j_l(j dq r) dr on the
// uniform mesh r <= Rcut (periodtable.cpp:1655-1688)
std::vector<Channel> vq_tables(const Species& sp, double ecut) {
  const int nqxq = (int)std::round(std::sqrt(2 * ecut) / kDq + 4.0);
  const int nr = (int)std::floor(sp.wavcut / kRab + 1e-9) + 1;
  std::vector<double> r(nr), rbeta(nr), aux(nr);
  for (int i = 0; i < nr; ++i) r[i] = kRab * i;
  std::vector<Channel> out;
  for (const auto& p : sp.proj) {
    for (int i = 0; i < nr; ++i) rbeta[i] = r[i] * p.val.eval(r[i]);
    Channel ch{p.l, p.h, std::vector<double>(nqxq)};
    for (int j = 0; j < nqxq; ++j) {
      for (int i = 0; i < nr; ++i) aux[i] = rbeta[i] * bessel(p.l, r[i] * (kDq * j)) * r[i];
      ch.tab[j] = simpson(aux, kRab);
    }
    out.push_back(std::move(ch));
  }
  return out;
}

// four-point Lagrange interpolation of the q table (periodtable.cpp:1703-1714)
double interp(const std::vector<double>& tab, double gk) {
  const double t = gk / kDq;
  const int it0 = (int)t;
  const double px = t - it0, ux = 1.0 - px, vx = 2.0 - px, wx = 3.0 - px;
  return tab[it0] * ux * vx * wx / 6.0 + tab[it0 + 1] * px * vx * wx / 2.0 - tab[it0 + 2] * px * ux * wx / 2.0 +
         tab[it0 + 3] * px * ux * vx / 6.0;
}

// vnlc for all atoms (host, column-major ns x nproj complex as interleaved
// doubles) and the weights h (4 pi)^2 / vol (hamiltonian.cpp:740-797)
int build_gs_projectors(pw_ctx* c, std::vector<double>& vnlc, std::vector<double>& wgt, int& nproj) {
  const int ns = c->gs_ns;
  const int natom = (int)c->atom_z.size();
  std::vector<double> g(3 * (size_t)ns), gk(ns);
  for (int s = 0; s < ns; ++s) {
    double q = 0;
    for (int d = 0; d < 3; ++d) {
      g[3 * s + d] = 2 * M_PI / c->L[d] * c->h_gs_m[3 * s + d];
      q += g[3 * s + d] * g[3 * s + d];
    }
    gk[s] = std::sqrt(q);
  }
  nproj = 0;
  for (int a = 0; a < natom; ++a) {
    const Species* sp = species(c->atom_z[a]);
    PWB_CHECK(sp, PW_EUNSUPPORTED, "HGH table only built for Si (14) and Al (13)");
    for (const auto& p : sp->proj) {
      PWB_CHECK(p.l <= 1, PW_EUNSUPPORTED, "Fourier-space projectors built for l = 0, 1");
      nproj += p.l == 0 ? 1 : 3;
    }
  }
  vnlc.assign((size_t)2 * ns * nproj, 0.0);
  wgt.assign(nproj, 0.0);
  const double sq2 = std::sqrt(2.0);
  const double w4 = std::pow(4 * M_PI, 2) / c->vol;
  std::vector<double> cr(ns), ci(ns), vq(ns);
  int col = 0;
  const Species* last = nullptr;
  std::vector<Channel> chans;
  for (int a = 0; a < natom; ++a) {
    const Species* sp = species(c->atom_z[a]);
    if (sp != last) {
      chans = vq_tables(*sp, c->gs_ecut);
      last = sp;
    }
    const double* R = c->atom_pos.data() + 3 * a;
    for (int s = 0; s < ns; ++s) {
      const double ph = -(g[3 * s] * R[0] + g[3 * s + 1] * R[1] + g[3 * s + 2] * R[2]);
      cr[s] = std::cos(ph);
      ci[s] = std::sin(ph);
    }
    for (const auto& ch : chans) {
      for (int s = 0; s < ns; ++s) vq[s] = interp(ch.tab, gk[s]);
      const int ncomp = ch.l == 0 ? 1 : 3;
      for (int m = 0; m < ncomp; ++m, ++col) {
        double* v = vnlc.data() + (size_t)2 * ns * col;
        wgt[col] = ch.h * w4;
        for (int s = 0; s < ns; ++s) {
          // vkb: s: sqrt(1/4pi) vq; p (z, x, y): -i sqrt(3/4pi) G_d / |G| vq
          double kr = 0, ki = 0;
          if (ch.l == 0) {
            kr = std::sqrt(1.0 / (4 * M_PI)) * vq[s];
          } else if (gk[s] > 1e-10) {
            const int d = m == 0 ? 2 : (m == 1 ? 0 : 1);
            ki = -std::sqrt(3.0 / (4 * M_PI)) * g[3 * s + d] / gk[s] * vq[s];
          }
          const double f = s == 0 ? 1.0 : sq2;
          v[2 * s] = f * (kr * cr[s] - ki * ci[s]);
          v[2 * s + 1] = f * (kr * ci[s] + ki * cr[s]);
        }
      }
    }
  }
  return PW_OK;
}

}  // namespace

int gs_teter(pw_ctx* c, const void* r, int ld, void* out, int ldo, int nband, int band0, int npair, int acc,
             cudaStream_t st) {
  const int nb = std::min(2 * npair, nband - band0);
  if (nb <= 0) return PW_OK;
  const long n2s = 2L * c->gs_ns;
  for (int b0 = band0; b0 < band0 + nb; b0 += 65535) {   // grid.y limit
    const dim3 grid((unsigned)((n2s + 255) / 256), (unsigned)std::min(65535, band0 + nb - b0));
    Launch L_(c, st, KK_ZTETER);
    if (c->prec == PW_F64)
      k_gs_teter<double><<<grid, 256, 0, st>>>((const double*)r + (long)b0 * ld, ld, (double*)out + (long)b0 * ldo,
                                               ldo, n2s, (const double*)c->gs_teter.p, acc);
    else
      k_gs_teter<float><<<grid, 256, 0, st>>>((const float*)r + (long)b0 * ld, ld, (float*)out + (long)b0 * ldo,
                                              ldo, n2s, (const float*)c->gs_teter.p, acc);
    PWB_CUDA(cudaGetLastError());
  }
  return PW_OK;
}

int gs_set_atoms(pw_ctx* c) {
  std::vector<double> vnlc, wgt;
  int nproj = 0;
  int rc = build_gs_projectors(c, vnlc, wgt, nproj);
  if (rc) return rc;
  return pw_gs_set_projectors(c, nproj, vnlc.data(), wgt.data());
}

}  // namespace pwb

using namespace pwb;

extern "C" {

int pw_ctx_create_gspace(const double length[3], const int numGrid[3], double ecut, int precision, int device,
                         pw_ctx** out) {
  PWB_CHECK(out && length && numGrid, PW_EINVAL, "null argument");
  *out = nullptr;
  PWB_CHECK(precision == PW_F64 || precision == PW_F32, PW_EINVAL, "precision must be PW_F64 or PW_F32");
  PWB_CHECK(ecut > 0, PW_EINVAL, "ecut must be positive");
  int box[3];
  for (int d = 0; d < 3; ++d) {
    PWB_CHECK(length[d] > 0, PW_EINVAL, "cell length must be positive");
    PWB_CHECK(numGrid[d] > 0 && numGrid[d] % 4 == 0, PW_EUNSUPPORTED,
              "the G-space grid must be a multiple of 4 (its half is the slot box)");
    PWB_CHECK(fft_len_supported(numGrid[d]), PW_EUNSUPPORTED, "FFT length not supported");
    box[d] = numGrid[d] / 2;
  }
  PWB_CHECK(find_grid(box) != nullptr, PW_EUNSUPPORTED, "grid (G-space grid / 2) not instantiated in this build");
  // sphere points in ascending R2C order (fourier.cpp:554-616)
  const int n0 = numGrid[0], n1 = numGrid[1], n2 = numGrid[2], h0 = n0 / 2 + 1;
  std::vector<int> idx, mil;
  std::vector<double> ek;
  for (int k = 0; k < n2; ++k)
    for (int j = 0; j < n1; ++j)
      for (int i = 0; i < h0; ++i) {
        const int m0 = kgrid(i, n0), m1 = kgrid(j, n1), m2 = kgrid(k, n2);
        const double g0 = 2 * M_PI / length[0] * m0, g1 = 2 * M_PI / length[1] * m1, g2 = 2 * M_PI / length[2] * m2;
        const double gkk = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
        const bool in_grid = m0 > 0 || (m0 == 0 && (m1 > 0 || (m1 == 0 && m2 >= 0)));
        if (!in_grid || !(gkk < ecut)) continue;
        PWB_CHECK(std::abs(m0) <= box[0] / 2 && std::abs(m1) <= box[1] / 2 && std::abs(m2) <= box[2] / 2,
                  PW_EUNSUPPORTED, "the sphere 1/2|G|^2 < ecut needs |m_d| <= N_d/4: raise the grid or lower ecut");
        idx.push_back(i + h0 * (j + n1 * k));
        mil.insert(mil.end(), {m0, m1, m2});
        ek.push_back(gkk);
      }
  const int ns = (int)idx.size();
  PWB_CHECK(ns > 0, PW_EINVAL, "empty sphere");
  PWB_CUDA(cudaSetDevice(device));
  pw_ctx* c = new pw_ctx();
  c->prec = precision;
  c->esz = precision == PW_F64 ? 8 : 4;
  c->device = device;
  for (int d = 0; d < 3; ++d) {
    c->L[d] = length[d];
    c->n[d] = box[d];
    c->nf[d] = numGrid[d];
  }
  c->vol = length[0] * length[1] * length[2];
  c->gs = true;
  c->gs_ecut = ecut;
  c->gs_ns = ns;
  c->ntot = 2L * ns;
  c->ntotf = (long)n0 * n1 * n2;
  c->h_gs_idx = std::move(idx);
  c->h_gs_m = std::move(mil);
  std::vector<double> te(ns);
  for (int s = 0; s < ns; ++s) {
    const double a = ek[s] * 2.0;
    const double b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0));
    te[s] = b / (b + 16.0 * std::pow(a, 4.0));
  }
  // Entry lists of the scatter kernel (one block per slot row, all points
  // G_s and -G_s of the row) and of the gather kernel (one block per slot
  // row r <= n1/2 and its mirror row, the stored points G_s), in the shared
  // memory layouts of k_gs_zinv ([N_z][n0+1]) and k_gs_zfwd ([N_z][2(n0+1)+1])
  const int nsx = box[0] + 1, nsy = box[1] + 1, nsz = box[2] + 1;
  const int pi1 = nsx, pi2 = 2 * nsx + 1, nblk = box[1] / 2 + 1;
  std::vector<char> used((size_t)nsx * nsy * nsz, 0);
  std::vector<std::vector<int>> inv_rows(nsy), fwd_rows(nblk);
  for (int s = 0; s < ns; ++s) {
    const int* m = &c->h_gs_m[3 * s];
    for (int sg = 1; sg >= -1; sg -= 2) {
      if (s == 0 && sg < 0) break;
      const int sx = slot_of(sg * m[0], box[0]), sy = slot_of(sg * m[1], box[1]), sz = slot_of(sg * m[2], box[2]);
      char& u = used[((size_t)sy * nsz + sz) * nsx + sx];
      if (u) { delete c; set_error("sphere slot collision"); return PW_EINVAL; }
      u = 1;
      const int fz = slot_to_fine(sz, box[2], n2);
      inv_rows[sy].insert(inv_rows[sy].end(), {sg * (s + 1), fz * pi1 + sx});
      if (sg < 0) continue;
      const int h = sy <= box[1] / 2 ? 0 : 1;
      const int r = h ? mirror_slot(sy, box[1]) : sy;
      const int nrow = mirror_slot(r, box[1]) == r ? 1 : 2;
      const int fzm = fz == 0 ? 0 : n2 - fz;
      const int off = fz * pi2 + h * nsx + sx;
      const int offm = fzm * pi2 + (nrow == 2 && h == 0 ? nsx : 0) + mirror_slot(sx, box[0]);
      fwd_rows[r].insert(fwd_rows[r].end(), {s, off | (offm << 16)});
    }
  }
  PWB_CHECK((long)n2 * pi2 < 65536, PW_EUNSUPPORTED, "G-space grid too large for the gather offsets");
  // entries of a block in shared-memory offset order: a warp's stores (scatter)
  // and loads (gather) then walk along kx, where consecutive sphere indices sit
  auto flatten = [](const std::vector<std::vector<int>>& rows, std::vector<int>& ptr, std::vector<int>& ent) {
    ptr.assign(1, 0);
    for (const auto& r : rows) {
      std::vector<std::pair<int, int>> e(r.size() / 2);
      for (size_t i = 0; i < e.size(); ++i) e[i] = {r[2 * i], r[2 * i + 1]};
      std::stable_sort(e.begin(), e.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
        return (a.second & 0xffff) < (b.second & 0xffff);
      });
      for (const auto& x : e) ent.insert(ent.end(), {x.first, x.second});
      ptr.push_back((int)(ent.size() / 2));
    }
  };
  std::vector<int> iptr, ient, fptr, fent;
  flatten(inv_rows, iptr, ient);
  flatten(fwd_rows, fptr, fent);
  auto up = [](DevBuf& b, const std::vector<int>& v) -> int {
    int r = b.alloc(std::max<size_t>(v.size(), 2) * 4);
    if (r) return r;
    if (cudaMemcpy(b.p, v.data(), v.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("cudaMemcpy of the sphere lists failed");
      return PW_ECUDA;
    }
    return PW_OK;
  };
  int rc;
  if ((rc = upload_real(c, c->gs_ekin, ek.data(), ns)) || (rc = upload_real(c, c->gs_teter, te.data(), ns)) ||
      (rc = up(c->gs_rows_inv, iptr)) || (rc = up(c->gs_ent_inv, ient)) || (rc = up(c->gs_rows_fwd, fptr)) ||
      (rc = up(c->gs_ent_fwd, fent))) {
    delete c;
    return rc;
  }
  const int lens[6] = {box[0], box[1], box[2], n0, n1, n2};
  for (int s = 0; s < 6; ++s)
    if ((rc = upload_twiddles(c, s, lens[s]))) { delete c; return rc; }
  if ((rc = ensure_scratch(c, 32))) { delete c; return rc; }
  {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) { delete c; set_error("cublasCreate failed"); return PW_ECUDA; }
    cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
    c->blas = h;
  }
  *out = c;
  return PW_OK;
}

int pw_gs_sphere(const pw_ctx* ctx, int* ns, int* idx_r2c, int* miller, double* ekin, double* teter) {
  PWB_CHECK(ctx && ctx->gs, PW_EINVAL, "not a G-space context");
  const int n = ctx->gs_ns;
  if (ns) *ns = n;
  if (idx_r2c) std::copy(ctx->h_gs_idx.begin(), ctx->h_gs_idx.end(), idx_r2c);
  if (miller) std::copy(ctx->h_gs_m.begin(), ctx->h_gs_m.end(), miller);
  if (ekin || teter) {
    for (int s = 0; s < n; ++s) {
      // the same expression as pw_ctx_create_gspace
      const int* m = &ctx->h_gs_m[3 * s];
      const double g0 = 2 * M_PI / ctx->L[0] * m[0], g1 = 2 * M_PI / ctx->L[1] * m[1], g2 = 2 * M_PI / ctx->L[2] * m[2];
      const double e = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
      if (ekin) ekin[s] = e;
      if (teter) {
        const double a = e * 2.0;
        const double b = 27.0 + a * (18.0 + a * (12.0 + a * 8.0));
        teter[s] = b / (b + 16.0 * std::pow(a, 4.0));
      }
    }
  }
  return PW_OK;
}

int pw_gs_set_projectors(pw_ctx* ctx, int nproj, const double* vnlc, const double* wgt) {
  PWB_CHECK(ctx && ctx->gs, PW_EINVAL, "not a G-space context");
  PWB_CHECK(nproj >= 0 && (nproj == 0 || (vnlc && wgt)), PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  ctx->have_nl = false;
  ctx->nproj = nproj;
  if (nproj == 0) return PW_OK;
  int rc;
  // the real view of column l is the projector row l of Q (T [nproj][2 ns])
  if ((rc = upload_real(ctx, ctx->q, vnlc, (size_t)nproj * ctx->ntot))) return rc;
  if ((rc = upload_real(ctx, ctx->qd, wgt, nproj))) return rc;
  if ((rc = install_dense_q(ctx, nproj))) return rc;
  ctx->h_nl_beta.assign(vnlc, vnlc + (size_t)nproj * ctx->ntot);
  ctx->h_pgamma.assign(wgt, wgt + nproj);
  ctx->have_nl = true;
  const int cap = std::max(ctx->pair_cap, 1);
  ctx->pair_cap = 0;
  return ensure_scratch(ctx, cap);
}

int pw_gs_get_projectors(const pw_ctx* ctx, int* nproj, double* vnlc, double* wgt) {
  PWB_CHECK(ctx && ctx->gs, PW_EINVAL, "not a G-space context");
  if (nproj) *nproj = ctx->have_nl ? ctx->nproj : 0;
  if (!ctx->have_nl) return PW_OK;
  if (vnlc) std::copy(ctx->h_nl_beta.begin(), ctx->h_nl_beta.end(), vnlc);
  if (wgt) std::copy(ctx->h_pgamma.begin(), ctx->h_pgamma.end(), wgt);
  return PW_OK;
}

}  // extern "C"
