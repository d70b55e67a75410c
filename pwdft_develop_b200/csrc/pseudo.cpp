// Host-side pseudopotential set-up for the real-space path: HGH tables,
// cubic splines, nonlocal projector index sets and values, and the local
// pseudocharge.  Set-up time only; the results feed pw_set_nonlocal and the
// SCF density/potential kernels.
//
//  * HGH parameters and functional forms: utilities/HGH.m (Si :262-276,
//    Al :234-248, derived h :284-300, forms :303-383, channel
//    diagonalisation :387-432, radial grid :893-894, table columns :1001-1093).
//  * spline / seval: src/utility.cpp:54-225.
//  * projector sets: PeriodTable::CalculateNonlocalPP, src/SCF/periodtable.cpp:994-1240.
//  * pseudocharge: PeriodTable::CalculatePseudoCharge, periodtable.cpp:282-377, with the
//    Cartesian minimum-image distance used by CalculateVLocal (periodtable.cpp:669-703).
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <vector>

#include "common.hpp"
#include "pseudo.hpp"

namespace pwb {

static const double kPi = 3.14159265358979323846;
static const double kMinRadial = 1e-10;   // include/periodtable.hpp:158

void spline_coef(int n, const double* x, const double* y, double* b, double* c, double* d) {
  for (int i = 0; i < n; ++i) b[i] = c[i] = d[i] = 0.0;
  const int nm1 = n - 1;
  if (n < 3) {
    b[0] = (y[1] - y[0]) / (x[1] - x[0]);
    b[1] = b[0];
    return;
  }
  d[0] = x[1] - x[0];
  c[1] = (y[1] - y[0]) / d[0];
  for (int i = 1; i < nm1; ++i) {
    d[i] = x[i + 1] - x[i];
    b[i] = 2. * (d[i - 1] + d[i]);
    c[i + 1] = (y[i + 1] - y[i]) / d[i];
    c[i] = c[i + 1] - c[i];
  }
  b[0] = -d[0];
  b[n - 1] = -d[n - 2];
  c[0] = 0.;
  c[n - 1] = 0.;
  if (n > 3) {
    c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0]);
    c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4]);
    c[0] = c[0] * d[0] * d[0] / (x[3] - x[0]);
    c[n - 1] = -c[n - 1] * d[n - 2] * d[n - 2] / (x[n - 1] - x[n - 4]);
  }
  for (int i = 1; i < n; ++i) {
    const double t = d[i - 1] / b[i - 1];
    b[i] = b[i] - t * d[i - 1];
    c[i] = c[i] - t * c[i - 1];
  }
  c[n - 1] = c[n - 1] / b[n - 1];
  for (int i = n - 2; i >= 0; --i) c[i] = (c[i] - d[i] * c[i + 1]) / b[i];
  b[n - 1] = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2. * c[n - 1]);
  for (int i = 0; i < nm1; ++i) {
    b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2. * c[i]);
    d[i] = (c[i + 1] - c[i]) / d[i];
    c[i] = 3. * c[i];
  }
  c[n - 1] = 3. * c[n - 1];
  d[n - 1] = d[n - 2];
}

double Spline::eval(double u) const {
  const int n = (int)x.size();
  int i;
  if (u < x[0]) {
    i = 0;
  } else if (u > x[n - 1]) {
    i = n - 1;
  } else {
    // binary search as in seval: x[i] <= u < x[i+1]
    i = (int)(std::upper_bound(x.begin(), x.end(), u) - x.begin()) - 1;
    if (i < 0) i = 0;
  }
  const double dx = u - x[i];
  return y[i] + dx * (b[i] + dx * (c[i] + dx * d[i]));
}

void Spline::build(const std::vector<double>& xs, const std::vector<double>& ys) {
  x = xs;
  y = ys;
  const int n = (int)x.size();
  b.assign(n, 0);
  c.assign(n, 0);
  d.assign(n, 0);
  spline_coef(n, x.data(), y.data(), b.data(), c.data(), d.data());
}

namespace {

struct HGHParams {
  double zion, mass, rloc, C[4], r0, h0[3], r1, h1[3], rhocut, wavcut;
};

bool hgh_params(int znuc, HGHParams& p) {
  if (znuc == 14) {
    p = {4.0, 28.0855, 0.44, {-7.336103, 0, 0, 0}, 0.422738, {5.906928, 3.258196, 0}, 0.484278,
         {2.727013, 0, 0}, 3.5, 3.5};
    return true;
  }
  if (znuc == 13) {
    p = {3.0, 26.9815386, 0.45, {-8.491351, 0, 0, 0}, 0.460104, {5.088340, 2.679700, 0}, 0.536744,
         {2.193438, 0, 0}, 3.5, 3.5};
    return true;
  }
  return false;
}

// Jacobi eigen-decomposition of a symmetric 3x3 matrix; columns of V are eigenvectors.
void jacobi3(double A[3][3], double w[3], double V[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = (i == j);
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (std::fabs(A[p][q]) < 1e-300) continue;
        const double theta = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
        for (int k = 0; k < 3; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = cs * akp - sn * akq;
          A[k][q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = cs * apk - sn * aqk;
          A[q][k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = cs * vkp - sn * vkq;
          V[k][q] = sn * vkp + cs * vkq;
        }
      }
  }
  for (int i = 0; i < 3; ++i) w[i] = A[i][i];
}

}  // namespace

const Species* species(int znuc) {
  static std::map<int, std::unique_ptr<Species>> cache;
  auto it = cache.find(znuc);
  if (it != cache.end()) return it->second.get();
  HGHParams p;
  if (!hgh_params(znuc, p)) return nullptr;
  auto sp = std::make_unique<Species>();
  sp->znuc = znuc;
  sp->zion = p.zion;
  sp->mass = p.mass;
  sp->rhocut = p.rhocut;
  sp->wavcut = p.wavcut;
  const double stp = 0.0005;
  const int nr = (int)std::floor((10.0 - (-10.0 + stp / 2)) / stp + 1e-9) + 1;
  std::vector<double> r(nr);
  for (int i = 0; i < nr; ++i) r[i] = -10.0 + stp / 2 + stp * i;
  const double Z = p.zion, rl = p.rloc, C1 = p.C[0], C2 = p.C[1], C3 = p.C[2], C4 = p.C[3];
  std::vector<double> rho(nr), drho(nr);
  double es = 0;
  for (int i = 0; i < nr; ++i) {
    const double x = r[i], e = std::exp(-0.5 * (x / rl) * (x / rl));
    const double r0v = 1.0 / (4 * kPi) *
                       (-std::sqrt(2 / kPi) * Z / std::pow(rl, 3) * e +
                        e * ((-6 * C2 + 3 * C1) / std::pow(rl, 2) + (-20 * C3 + 7 * C2 - C1) * x * x / std::pow(rl, 4) +
                             (-42 * C4 + 11 * C3 - C2) * std::pow(x, 4) / std::pow(rl, 6) +
                             (15 * C4 - C3) * std::pow(x, 6) / std::pow(rl, 8) - C4 * std::pow(x, 8) / std::pow(rl, 10)));
    const double dr0v =
        1.0 / (4 * kPi) *
        (std::sqrt(2 / kPi) * Z * x / std::pow(rl, 5) * e +
         e * ((-40 * C3 + 20 * C2 - 5 * C1) * x / std::pow(rl, 4) +
              (-168 * C4 + 64 * C3 - 11 * C2 + C1) * std::pow(x, 3) / std::pow(rl, 6) +
              (132 * C4 - 17 * C3 + C2) * std::pow(x, 5) / std::pow(rl, 8) +
              (-23 * C4 + C3) * std::pow(x, 7) / std::pow(rl, 10) + C4 * std::pow(x, 9) / std::pow(rl, 12)));
    rho[i] = -r0v;
    drho[i] = -dr0v;
    if (x > 0) {
      const double vl = -Z / x * std::erf(x / (std::sqrt(2.0) * rl)) +
                        e * (C1 + C2 * std::pow(x / rl, 2) + C3 * std::pow(x / rl, 4) + C4 * std::pow(x / rl, 6));
      es += 4 * kPi * x * x * vl * r0v * stp;
    }
  }
  sp->eself = 0.5 * es;   // HGH.m:995
  sp->rho.build(r, rho);
  sp->drho.build(r, drho);
  // channels l = 0, 1
  for (int l = 0; l <= 1; ++l) {
    const double rlp = (l == 0) ? p.r0 : p.r1;
    const double* hd = (l == 0) ? p.h0 : p.h1;
    double h12, h13, h23;
    if (l == 0) {
      h12 = -0.5 * std::sqrt(3.0 / 5.0) * hd[1];
      h13 = 0.5 * std::sqrt(5.0 / 21.0) * hd[2];
      h23 = -0.5 * std::sqrt(100.0 / 63.0) * hd[2];
    } else {
      h12 = -0.5 * std::sqrt(5.0 / 7.0) * hd[1];
      h13 = 1.0 / 6.0 * std::sqrt(35.0 / 11.0) * hd[2];
      h23 = -1.0 / 6.0 * 14.0 / std::sqrt(11.0) * hd[2];
    }
    double A[3][3] = {{hd[0], h12, h13}, {h12, hd[1], h23}, {h13, h23, hd[2]}};
    double w[3], V[3][3];
    jacobi3(A, w, V);
    // eigenvector sign is arbitrary (MATLAB eig); fix it: largest |component| > 0
    for (int a = 0; a < 3; ++a) {
      int im = 0;
      for (int i = 1; i < 3; ++i)
        if (std::fabs(V[i][a]) > std::fabs(V[im][a])) im = i;
      if (V[im][a] < 0)
        for (int i = 0; i < 3; ++i) V[i][a] = -V[i][a];
    }
    int ord[3] = {0, 1, 2};
    std::stable_sort(ord, ord + 3, [&](int a, int b) { return w[a] > w[b]; });
    for (int oi = 0; oi < 3; ++oi) {
      const int a = ord[oi];
      if (std::fabs(w[a]) <= 1e-10) continue;
      std::vector<double> val(nr), der(nr);
      for (int k = 0; k < nr; ++k) {
        double v = 0, dv = 0;
        const double x = r[k];
        for (int i = 1; i <= 3; ++i) {
          const double ex = l + (4 * i - 1) / 2.0;
          const int pw = l + 2 * (i - 1);
          const double nrm = std::sqrt(2.0) / (std::pow(rlp, ex) * std::sqrt(std::tgamma(ex)));
          const double e = std::exp(-x * x / (2 * rlp * rlp));
          const double f = nrm * std::pow(x, pw) * e;
          const double df = (pw == 0) ? nrm * e * (-x / (rlp * rlp))
                                      : nrm * e * (pw * std::pow(x, pw - 1) - std::pow(x, pw + 1) / (rlp * rlp));
          v += V[i - 1][a] * f;
          dv += V[i - 1][a] * df;
        }
        val[k] = v;
        der[k] = dv;
      }
      Species::Proj pj;
      pj.l = l;
      pj.h = w[a];
      pj.val.build(r, val);
      pj.der.build(r, der);
      sp->proj.push_back(std::move(pj));
    }
  }
  const Species* out = sp.get();
  cache[znuc] = std::move(sp);
  return out;
}

static inline double cround(double x) { return x >= 0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5); }

int nonlocal_pp(const Species& sp, const double pos[3], const double L[3], const int nG[3], AtomNL& out) {
  out.idx.clear();
  out.disp.clear();
  out.val.clear();
  out.wgt.clear();
  const double R = sp.wavcut;
  double frac[3];
  for (int d = 0; d < 3; ++d) frac[d] = pos[d] / L[d];
  int nmin[3], nmax[3];
  for (int d = 0; d < 3; ++d) {
    const double w = R / (2 * kPi) * (2 * kPi / L[d]);   // Rzero/(2pi) * |recipcell row|
    nmin[d] = (int)cround((frac[d] - w) * nG[d]);
    nmax[d] = (int)cround((frac[d] + w) * nG[d]);
  }
  std::vector<double> rad, xx, yy, zz;
  for (int k = nmin[2]; k <= nmax[2]; ++k) {
    int kk = k % nG[2];
    if (kk < 0) kk += nG[2];
    for (int j = nmin[1]; j <= nmax[1]; ++j) {
      int jj = j % nG[1];
      if (jj < 0) jj += nG[1];
      for (int i = nmin[0]; i <= nmax[0]; ++i) {
        int ii = i % nG[0];
        if (ii < 0) ii += nG[0];
        const double gx = (i / (double)nG[0] - frac[0]) * L[0];
        const double gy = (j / (double)nG[1] - frac[1]) * L[1];
        const double gz = (k / (double)nG[2] - frac[2]) * L[2];
        const double dist = std::sqrt(gx * gx + gy * gy + gz * gz);
        if (dist < R) {
          out.idx.push_back(ii + jj * nG[0] + kk * nG[0] * nG[1]);
          out.disp.push_back(gx);
          out.disp.push_back(gy);
          out.disp.push_back(gz);
          rad.push_back(dist);
          xx.push_back(gx);
          yy.push_back(gy);
          zz.push_back(gz);
        }
      }
    }
  }
  const int np = (int)out.idx.size();
  out.npts = np;
  for (const auto& pj : sp.proj) {
    if (pj.l == 0) {
      const double coef = std::sqrt(1.0 / (4 * kPi));
      std::vector<double> dv((size_t)np * 4);
      for (int g = 0; g < np; ++g) {
        const double v = pj.val.eval(rad[g]), dr = pj.der.eval(rad[g]);
        dv[4 * g + 0] = coef * v;
        if (rad[g] > kMinRadial) {
          dv[4 * g + 1] = coef * dr * xx[g] / rad[g];
          dv[4 * g + 2] = coef * dr * yy[g] / rad[g];
          dv[4 * g + 3] = coef * dr * zz[g] / rad[g];
        } else {
          dv[4 * g + 1] = dv[4 * g + 2] = dv[4 * g + 3] = 0;
        }
      }
      out.val.push_back(std::move(dv));
      out.wgt.push_back(pj.h);
    } else if (pj.l == 1) {
      const double coef = std::sqrt(3.0 / (4 * kPi));
      // order z, x, y as in periodtable.cpp:1180-1232
      const int dirs[3] = {2, 0, 1};
      for (int m = 0; m < 3; ++m) {
        const int dir = dirs[m];
        std::vector<double> dv((size_t)np * 4);
        for (int g = 0; g < np; ++g) {
          const double v = pj.val.eval(rad[g]), dr = pj.der.eval(rad[g]);
          const double c3[3] = {xx[g], yy[g], zz[g]};
          if (rad[g] > kMinRadial) {
            const double rr = rad[g];
            const double u = c3[dir] / rr;
            dv[4 * g + 0] = coef * (u * v);
            for (int a = 0; a < 3; ++a) {
              double t = coef * ((dr - v / rr) * u * (c3[a] / rr));
              if (a == dir) t += coef * v / rr;
              dv[4 * g + 1 + a] = t;
            }
          } else {
            dv[4 * g + 0] = 0;
            for (int a = 0; a < 3; ++a) dv[4 * g + 1 + a] = (a == dir) ? coef * dr : 0.0;
          }
        }
        out.val.push_back(std::move(dv));
        out.wgt.push_back(pj.h);
      }
    } else {
      set_error("only l = 0, 1 projector channels are built");
      return PW_EUNSUPPORTED;
    }
  }
  return PW_OK;
}

int pseudo_charge(const Species& sp, const double pos[3], const double L[3], const int N[3], AtomRho& out) {
  out.idx.clear();
  out.val.clear();
  const double R = sp.rhocut;
  std::vector<double> dist[3];
  for (int d = 0; d < 3; ++d) {
    dist[d].resize(N[d]);
    for (int i = 0; i < N[d]; ++i) {
      double x = i / (double)N[d] * L[d] - pos[d];
      x -= cround(x / L[d]) * L[d];
      dist[d][i] = x;
    }
  }
  for (int k = 0; k < N[2]; ++k)
    for (int j = 0; j < N[1]; ++j)
      for (int i = 0; i < N[0]; ++i) {
        const double x = dist[0][i], y = dist[1][j], z = dist[2][k];
        const double r = std::sqrt(x * x + y * y + z * z);
        if (r <= R) {
          out.idx.push_back(i + N[0] * (j + N[1] * k));
          const double v = sp.rho.eval(r), dr = sp.drho.eval(r);
          out.val.push_back(v);
          if (r > kMinRadial) {
            out.val.push_back(dr * x / r);
            out.val.push_back(dr * y / r);
            out.val.push_back(dr * z / r);
          } else {
            out.val.push_back(0);
            out.val.push_back(0);
            out.val.push_back(0);
          }
        }
      }
  return PW_OK;
}

}  // namespace pwb
