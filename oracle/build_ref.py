"""Compile standalone reference functions into ``oracle/_ref/libpwref.so``.

Test infrastructure.  The reference's full build needs MPI, FFTW, MKL,
libxc and yaml-cpp, which are absent, so it cannot be built.  Four of its
functions are self-contained and are compiled here directly from the
reference source tree (never copied into this repository): ``spline`` and
``seval`` (src/utility.cpp:54-225), ``IP_c2f`` / ``IP_f2c``
(src/utility.cpp:3148-3275) and the internal PBE pieces ``VExchange_sla``,
``VCorrelation_pw``, ``VGCExchange_pbx``, ``VGCCorrelation_pbc``
(src/utility.cpp:3913-4244, the ``Use_Libxc: 0`` path of KohnSham::CalculateXC)
and the HSE06 short-range PBE exchange ``pbexsr`` with
``wpbe_analy_erfc_approx_grad`` and ``EXPINT`` (src/utility.cpp:3340-3911), and the smearing functions
``wgauss`` and ``getEntropy`` (src/utility.cpp:4404-4444).  The recipe extracts each function body from
``<reference>/src/utility.cpp`` by brace matching into ``oracle/_ref/`` (git
ignored), prepends the headers and typedefs it needs (``<stdlib.h>`` first, as
include/utility.hpp:49 has it: it puts the floating-point ``abs`` overloads
that ``EXPINT`` relies on into the global namespace), adds extern "C" wrappers and
builds a shared object with g++.  Tests use it to pin the NumPy restatement.
"""
from __future__ import annotations

import os
import re
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libpwref.so"
DEFAULT_REF = Path(os.environ.get("PWDFT_REFERENCE", "/root/reference"))

FUNCS = [("void spline(", "spline"), ("void seval(", "seval"),
         ("void IP_c2f(", "IP_c2f"), ("void IP_f2c(", "IP_f2c"),
         ("void VExchange_sla(", "VExchange_sla"), ("void VCorrelation_pw(", "VCorrelation_pw"),
         ("void VGCExchange_pbx(", "VGCExchange_pbx"), ("void VGCCorrelation_pbc(", "VGCCorrelation_pbc"),
         ("void pbexsr(", "pbexsr"), ("void wpbe_analy_erfc_approx_grad(", "wpbe_analy_erfc_approx_grad"),
         ("Real EXPINT(", "EXPINT"), ("Real wgauss(", "wgauss"), ("Real getEntropy(", "getEntropy")]

PRELUDE = """// generated: functions compiled from the reference source tree
#include <stdlib.h>
#include <cmath>
#include <complex>
#include <stdexcept>
#include <string>
#include <algorithm>
typedef std::complex<double> Complex;
typedef double Real;
typedef int Int;
static const double PI = 3.141592653589793;
static void ErrorHandling(const char* m) { throw std::runtime_error(m); }
namespace pwref {
void wpbe_analy_erfc_approx_grad(Real rho, Real s, Real omega, Real& Fx_wpbe, Real& d1rfx, Real& d1sfx);
Real EXPINT(Int n, Real x);
"""

WRAPPERS = """
}  // namespace pwref
extern "C" {
void ref_spline(int n, double* x, double* y, double* b, double* c, double* d) { pwref::spline(n, x, y, b, c, d); }
void ref_seval(double* v, int m, double* u, int n, double* x, double* y, double* b, double* c, double* d) {
  pwref::seval(v, m, u, n, x, y, b, c, d);
}
void ref_ip_c2f(int* Nc, int* Nf, double* tilde, double* tildef) {
  pwref::IP_c2f(Nc, Nf, reinterpret_cast<Complex*>(tilde), reinterpret_cast<Complex*>(tildef));
}
void ref_ip_f2c(int* Nc, int* Nf, double* tilde, double* tildef) {
  pwref::IP_f2c(Nc, Nf, reinterpret_cast<Complex*>(tilde), reinterpret_cast<Complex*>(tildef));
}
// out: ux vx (Slater, at rs) uc vc (PW92, at rs) ugcx v1gcx v2gcx ugcc v1gcc v2gcc (PBE, at rho, grho2)
void ref_pbe_parts(double rs, double rho, double grho2, double* out) {
  pwref::VExchange_sla(rs, out[0], out[1]);
  pwref::VCorrelation_pw(rs, out[2], out[3]);
  pwref::VGCExchange_pbx(rho, grho2, out[4], out[5], out[6]);
  pwref::VGCCorrelation_pbc(rho, grho2, out[7], out[8], out[9]);
}
// out: sx v1x v2x of the short-range PBE exchange at (rho, grho2, omega)
void ref_pbexsr(double rho, double grho2, double omega, double* out) {
  pwref::pbexsr(rho, grho2, omega, out[0], out[1], out[2]);
}
// out: F_x d1rfx d1sfx of the screened enhancement factor at (rho, s, omega)
void ref_wpbe(double rho, double s, double omega, double* out) {
  pwref::wpbe_analy_erfc_approx_grad(rho, s, omega, out[0], out[1], out[2]);
}
double ref_expint(int n, double x) { return pwref::EXPINT(n, x); }
// smearing: 0 "FD", 1 "GB"
double ref_wgauss(double ev, double ef, double tbeta, int gb) { return pwref::wgauss(ev, ef, tbeta, gb ? "GB" : "FD"); }
double ref_entropy(double ev, double ef, double tbeta, int gb) {
  return pwref::getEntropy(ev, ef, tbeta, gb ? "GB" : "FD");
}
}
"""


def _strip_comments(text: str) -> str:
    """Blank out /* */ and // comments (keeping newlines) so that commented-out
    definitions (e.g. the disabled "method I" IP_c2f at src/utility.cpp:2980-3144)
    are not picked up."""
    out, i, n = [], 0, len(text)
    while i < n:
        if text.startswith("/*", i):
            j = text.find("*/", i + 2)
            j = n if j < 0 else j + 2
            out.append("".join(ch if ch == "\n" else " " for ch in text[i:j]))
            i = j
        elif text.startswith("//", i):
            j = text.find("\n", i)
            j = n if j < 0 else j
            out.append(" " * (j - i))
            i = j
        else:
            out.append(text[i])
            i += 1
    return "".join(out)


def _extract(text: str, head: str) -> str:
    i = text.find(head)
    if i < 0:
        raise RuntimeError(f"function {head!r} not found")
    j = text.find("{", i)
    depth = 0
    k = j
    while True:
        ch = text[k]
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                break
        k += 1
    return text[i:k + 1]


def build(ref_root: Path = DEFAULT_REF) -> Path | None:
    src = ref_root / "src" / "utility.cpp"
    if not src.exists():
        return LIB if LIB.exists() else None
    text = _strip_comments(src.read_text(errors="replace"))
    body = [_extract(text, h) for h, _ in FUNCS]
    OUT.mkdir(exist_ok=True)
    cpp = OUT / "ref_funcs.cpp"
    cpp.write_text(PRELUDE + "\n\n".join(body) + WRAPPERS)
    r = subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-o", str(LIB), str(cpp)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    build_hpsi(ref_root)
    return LIB


# ---------------------------------------------------------------------------
# The reference's own H*psi composition: Spinor::AddMultSpinorFineR2C (real
# version, src/SCF/spinor.cpp:377-525), Spinor::AddTeterPrecond (real version,
# spinor.cpp:310-346) and FFTWExecute (src/SCF/fourier.cpp:695-764), compiled
# from the reference tree with IP_c2f / IP_f2c (src/utility.cpp:3148-3275)
# over a small harness written here: the container types these bodies use
# (NumVec / NumMat / NumTns views, SparseVec, PseudoPot::vnlList, Index3,
# Domain), blas::Copy / Axpy / Scal, SetValue, and an FFTW stand-in
# (fftw_plan / fftw_execute: unnormalised 3-D r2c / c2r with FFTW's sign and
# layout conventions, x fastest, computed by a mixed-radix complex FFT).  FFTW
# is a third-party library absent here; the stand-in follows its documented
# definition of the transforms.
# ---------------------------------------------------------------------------
LIB_HPSI = OUT / "libpwref_hpsi.so"

HPSI_FUNCS = ["void FFTWExecute ( Fourier& fft, fftw_plan& plan )"]
HPSI_METHODS = [("Spinor::AddTeterPrecond (Fourier* fftPtr, DblNumVec& teter, NumTns<Real>& a3)", "void "),
                ("Spinor::AddMultSpinorFineR2C ( Fourier& fft, const DblNumVec& ekin,", "void ")]

HPSI_HARNESS = r"""// generated: the reference's H*psi composition over a test harness
#include <cmath>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
typedef int Int;
typedef double Real;
typedef std::complex<double> Complex;
static const Complex Z_ZERO(0.0, 0.0);
enum { VAL, DX, DY, DZ };
static void ErrorHandling(const std::string& m) { throw std::runtime_error(m); }
namespace pwref {
struct Index3 {
  int v[3];
  int& operator[](int i) { return v[i]; }
  const int& operator[](int i) const { return v[i]; }
  int* Data() { return v; }
};
template <class T> struct NumVec {
  std::vector<T> d;
  NumVec() {}
  explicit NumVec(Int n) : d(n) {}
  Int m() const { return (Int)d.size(); }
  // as the reference's NumVec, a const view still hands out a mutable pointer
  T* Data() const { return const_cast<T*>(d.data()); }
  T& operator()(Int i) { return d[i]; }
  const T& operator()(Int i) const { return d[i]; }
  T& operator[](Int i) { return d[i]; }
  const T& operator[](Int i) const { return d[i]; }
};
typedef NumVec<Real> DblNumVec;
typedef NumVec<Complex> CpxNumVec;
typedef NumVec<Int> IntNumVec;
template <class T> struct NumMat {
  Int m_ = 0, n_ = 0;
  std::vector<T> d;
  NumMat() {}
  NumMat(Int m, Int n) : m_(m), n_(n), d((size_t)m * n) {}
  Int m() const { return m_; }
  Int n() const { return n_; }
  T* VecData(Int j) { return d.data() + (size_t)j * m_; }
  const T* VecData(Int j) const { return d.data() + (size_t)j * m_; }
};
typedef NumMat<Real> DblNumMat;
template <class T> struct NumTns {
  Int m_, n_, p_;
  T* data_;
  NumTns(Int m, Int n, Int p, T* data) : m_(m), n_(n), p_(p), data_(data) {}
  Int m() const { return m_; }
  Int n() const { return n_; }
  Int p() const { return p_; }
  T* VecData(Int j, Int k) { return data_ + (size_t)m_ * (j + (size_t)n_ * k); }
  const T* VecData(Int j, Int k) const { return data_ + (size_t)m_ * (j + (size_t)n_ * k); }
};
typedef std::pair<IntNumVec, DblNumMat> SparseVec;
struct PseudoPot {
  std::vector<std::pair<SparseVec, Real>> vnlList;
};
template <class T, class U> void SetValue(NumVec<T>& v, U x) {
  for (auto& e : v.d) e = T(x);
}
namespace blas {
inline void Copy(Int n, const Real* x, Int incx, Real* y, Int incy) {
  for (Int i = 0; i < n; ++i) y[(size_t)i * incy] = x[(size_t)i * incx];
}
inline void Axpy(Int n, Real a, const Real* x, Int incx, Real* y, Int incy) {
  for (Int i = 0; i < n; ++i) y[(size_t)i * incy] += a * x[(size_t)i * incx];
}
inline void Scal(Int n, Real a, Real* x, Int incx) {
  for (Int i = 0; i < n; ++i) x[(size_t)i * incx] *= a;
}
inline void Scal(Int n, Real a, Complex* x, Int incx) {
  for (Int i = 0; i < n; ++i) x[(size_t)i * incx] *= a;
}
}  // namespace blas
struct Domain {
  Index3 numGrid, numGridFine;
  Real length[3];
  Int NumGridTotal() const { return numGrid[0] * numGrid[1] * numGrid[2]; }
  Int NumGridTotalFine() const { return numGridFine[0] * numGridFine[1] * numGridFine[2]; }
  Real Volume() const { return length[0] * length[1] * length[2]; }
};
struct ESDFParam {
  std::string FFTtype;
};
static ESDFParam esdfParam{"even"};

// ---- FFTW stand-in: unnormalised transforms, FFTW_FORWARD = exp(-i ...) ----
struct FFTPlanRec {
  int real_to_complex;      // 1: r2c (in real, out half complex), 0: c2r
  int n[3];                 // x, y, z sizes (x fastest)
  Real* rdata;
  Complex* cdata;
};
typedef FFTPlanRec* fftw_plan;
// One length: the radices (4, 2, 3, 5, then any prime) and, per stage, the
// twiddles w^(j k) of a Stockham autosort pass.
struct FFTLen {
  int n = 0;
  std::vector<int> radix;
  std::vector<std::vector<Complex>> tw[2];   // [sign > 0][stage][j * r + k]
  std::vector<std::vector<Complex>> root[2]; // [sign > 0][stage][s * r + k] = exp(sign 2 pi i k s / r)
  explicit FFTLen(int n_) : n(n_) {
    int m = n;
    for (int r : {4, 2, 3, 5})
      while (m % r == 0) { radix.push_back(r); m /= r; }
    for (int r = 7; m > 1; r += 2)
      while (m % r == 0) { radix.push_back(r); m /= r; }
    for (int sg = 0; sg < 2; ++sg) {
      const double sign = sg ? 1.0 : -1.0;
      int l = 1;
      for (int r : radix) {
        std::vector<Complex> t((size_t)l * r);
        for (int j = 0; j < l; ++j)
          for (int k = 0; k < r; ++k) t[(size_t)j * r + k] = std::polar(1.0, sign * 2.0 * M_PI * j * k / (double)(l * r));
        tw[sg].push_back(t);
        std::vector<Complex> rt((size_t)r * r);
        for (int s2 = 0; s2 < r; ++s2)
          for (int k = 0; k < r; ++k) rt[(size_t)s2 * r + k] = std::polar(1.0, sign * 2.0 * M_PI * ((k * s2) % r) / (double)r);
        root[sg].push_back(rt);
        l *= r;
      }
    }
  }
};
// in place, unnormalised, sign -1 forward / +1 backward; work: n scratch values
static void fft1(const FFTLen& L, Complex* a, Complex* work, int sign) {
  const int n = L.n;
  if (n <= 1) return;
  const int sg = sign > 0 ? 1 : 0;
  Complex* x = a;
  Complex* y = work;
  int l = 1;   // size of the transforms already done
  for (size_t st = 0; st < L.radix.size(); ++st) {
    const int r = L.radix[st];
    const int m = n / (l * r);   // number of interleaved sub-problems left
    const Complex* w = L.tw[sg][st].data();
    const Complex* rt = L.root[sg][st].data();
    if (r == 2) {
      for (int q = 0; q < m; ++q)
        for (int j = 0; j < l; ++j) {
          const Complex v0 = x[(size_t)q * l + j], v1 = x[(size_t)(m + q) * l + j] * w[2 * j + 1];
          y[(size_t)(2 * q) * l + j] = v0 + v1;
          y[(size_t)(2 * q + 1) * l + j] = v0 - v1;
        }
    } else if (r == 4) {
      // exp(sign i pi / 2) = sign i
      const double si = sign > 0 ? 1.0 : -1.0;
      for (int q = 0; q < m; ++q)
        for (int j = 0; j < l; ++j) {
          const Complex v0 = x[(size_t)q * l + j];
          const Complex v1 = x[(size_t)(m + q) * l + j] * w[4 * j + 1];
          const Complex v2 = x[(size_t)(2 * m + q) * l + j] * w[4 * j + 2];
          const Complex v3 = x[(size_t)(3 * m + q) * l + j] * w[4 * j + 3];
          const Complex s02 = v0 + v2, d02 = v0 - v2, s13 = v1 + v3, d13 = v1 - v3;
          const Complex id13(-si * d13.imag(), si * d13.real());
          y[(size_t)(4 * q) * l + j] = s02 + s13;
          y[(size_t)(4 * q + 1) * l + j] = d02 + id13;
          y[(size_t)(4 * q + 2) * l + j] = s02 - s13;
          y[(size_t)(4 * q + 3) * l + j] = d02 - id13;
        }
    } else {
      Complex v[64];
      for (int q = 0; q < m; ++q)
        for (int j = 0; j < l; ++j) {
          v[0] = x[(size_t)q * l + j];
          for (int k = 1; k < r; ++k) v[k] = x[(size_t)(k * m + q) * l + j] * w[(size_t)j * r + k];
          for (int s2 = 0; s2 < r; ++s2) {
            Complex acc = v[0];
            for (int k = 1; k < r; ++k) acc += v[k] * rt[s2 * r + k];
            y[(size_t)(q * r + s2) * l + j] = acc;
          }
        }
    }
    std::swap(x, y);
    l *= r;
  }
  if (x != a)
    for (int i = 0; i < n; ++i) a[i] = x[i];
}
static const FFTLen& fft_len(int n) {
  static std::vector<FFTLen*> cache;
  for (FFTLen* f : cache)
    if (f->n == n) return *f;
  cache.push_back(new FFTLen(n));
  return *cache.back();
}
// complex 3-D transform of an x-fastest (nx, ny, nz) array along one axis;
// along y and z, blocks of up to 8 neighbouring x columns are gathered together
static void fft_axis(Complex* a, int nx, int ny, int nz, int axis, int sign, int xlen) {
  const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
  const FFTLen& L = fft_len(n);
  constexpr int B = 8;
  std::vector<Complex> lines((size_t)B * n), work(n);
  const long sy = xlen, sz = (long)xlen * ny;
  if (axis == 0) {
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) fft1(L, a + j * sy + k * sz, work.data(), sign);
    return;
  }
  const long stride = axis == 1 ? sy : sz;
  const int c1 = axis == 1 ? 1 : ny;
  const int c2 = axis == 2 ? 1 : nz;
  for (int k = 0; k < c2; ++k)
    for (int j = 0; j < c1; ++j)
      for (int i0 = 0; i0 < nx; i0 += B) {
        const int nb = std::min(B, nx - i0);
        Complex* base = a + i0 + j * sy + k * sz;
        for (int t = 0; t < n; ++t)
          for (int b = 0; b < nb; ++b) lines[(size_t)b * n + t] = base[t * stride + b];
        for (int b = 0; b < nb; ++b) fft1(L, lines.data() + (size_t)b * n, work.data(), sign);
        for (int t = 0; t < n; ++t)
          for (int b = 0; b < nb; ++b) base[t * stride + b] = lines[(size_t)b * n + t];
      }
}
// FFTW's r2c / c2r (unnormalised, exp(-i ...) forward), x fastest: x by pairs
// of real lines packed into one complex line, then y and z on the half spectrum
static void fftw_execute(fftw_plan p) {
  const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2], h0 = n0 / 2 + 1;
  const FFTLen& Lx = fft_len(n0);
  std::vector<Complex> line(n0), work(n0);
  const long nlines = (long)n1 * n2;
  Complex* H = p->cdata;                           // half spectrum, rows of h0
  if (p->real_to_complex) {
    for (long r = 0; r < nlines; r += 2) {
      const Real* x0 = p->rdata + r * n0;
      const Real* x1 = (r + 1 < nlines) ? x0 + n0 : nullptr;
      for (int t = 0; t < n0; ++t) line[t] = Complex(x0[t], x1 ? x1[t] : 0.0);
      fft1(Lx, line.data(), work.data(), -1);
      for (int k = 0; k < h0; ++k) {
        const Complex a = line[k], b = std::conj(line[(n0 - k) % n0]);
        H[r * h0 + k] = 0.5 * (a + b);
        if (x1) H[(r + 1) * h0 + k] = Complex(0.0, -0.5) * (a - b);
      }
    }
    fft_axis(H, h0, n1, n2, 1, -1, h0);
    fft_axis(H, h0, n1, n2, 2, -1, h0);
  } else {
    std::vector<Complex> G(H, H + (size_t)h0 * nlines);
    fft_axis(G.data(), h0, n1, n2, 2, +1, h0);
    fft_axis(G.data(), h0, n1, n2, 1, +1, h0);
    for (long r = 0; r < nlines; r += 2) {
      const bool two = r + 1 < nlines;
      // a Hermitian-extended line x0 + i x1 from the two half rows
      for (int k = 0; k < n0; ++k) {
        Complex a, b;
        if (k < h0) {
          a = G[r * h0 + k];
          b = two ? G[(r + 1) * h0 + k] : Complex(0, 0);
        } else {
          a = std::conj(G[r * h0 + (n0 - k)]);
          b = two ? std::conj(G[(r + 1) * h0 + (n0 - k)]) : Complex(0, 0);
        }
        // c2r reads only the real part of the DC and Nyquist entries
        if (k == 0 || 2 * k == n0) {
          a = Complex(a.real(), 0.0);
          b = Complex(b.real(), 0.0);
        }
        line[k] = a + Complex(0.0, 1.0) * b;
      }
      fft1(Lx, line.data(), work.data(), +1);
      for (int t = 0; t < n0; ++t) {
        p->rdata[r * n0 + t] = line[t].real();
        if (two) p->rdata[(r + 1) * n0 + t] = line[t].imag();
      }
    }
  }
}
struct Fourier {
  Domain domain;
  bool isInitialized = true;
  Int numGridTotalR2C = 0, numGridTotalR2CFine = 0;
  DblNumVec inputVecR2C, inputVecR2CFine;
  CpxNumVec outputVecR2C, outputVecR2CFine;
  CpxNumVec inputComplexVec, outputComplexVec, inputComplexVecFine, outputComplexVecFine;
  IntNumVec idxFineGridR2C;
  FFTPlanRec rec[4];
  fftw_plan forwardPlanR2C = nullptr, backwardPlanR2C = nullptr, forwardPlanR2CFine = nullptr,
            backwardPlanR2CFine = nullptr;
  fftw_plan forwardPlan = nullptr, backwardPlan = nullptr, forwardPlanFine = nullptr, backwardPlanFine = nullptr;
  void setup(const int* n, const int* nf, const double* L) {
    for (int d = 0; d < 3; ++d) {
      domain.numGrid[d] = n[d];
      domain.numGridFine[d] = nf[d];
      domain.length[d] = L[d];
    }
    numGridTotalR2C = (n[0] / 2 + 1) * n[1] * n[2];
    numGridTotalR2CFine = (nf[0] / 2 + 1) * nf[1] * nf[2];
    inputVecR2C = DblNumVec(domain.NumGridTotal());
    inputVecR2CFine = DblNumVec(domain.NumGridTotalFine());
    outputVecR2C = CpxNumVec(numGridTotalR2C);
    outputVecR2CFine = CpxNumVec(numGridTotalR2CFine);
    rec[0] = {1, {n[0], n[1], n[2]}, inputVecR2C.Data(), outputVecR2C.Data()};
    rec[1] = {0, {n[0], n[1], n[2]}, inputVecR2C.Data(), outputVecR2C.Data()};
    rec[2] = {1, {nf[0], nf[1], nf[2]}, inputVecR2CFine.Data(), outputVecR2CFine.Data()};
    rec[3] = {0, {nf[0], nf[1], nf[2]}, inputVecR2CFine.Data(), outputVecR2CFine.Data()};
    forwardPlanR2C = &rec[0];
    backwardPlanR2C = &rec[1];
    forwardPlanR2CFine = &rec[2];
    backwardPlanR2CFine = &rec[3];
  }
};
class Spinor {
 public:
  Domain domain_;
  NumTns<Real> wavefun_;
  Spinor(const Domain& d, Real* psi, Int nb) : domain_(d), wavefun_(d.NumGridTotal(), 1, nb, psi) {}
  void AddTeterPrecond(Fourier* fftPtr, DblNumVec& teter, NumTns<Real>& a3);
  void AddMultSpinorFineR2C(Fourier& fft, const DblNumVec& ekin, const DblNumVec& vtot,
                            const std::vector<PseudoPot>& pseudo, NumTns<Real>& a3);
};
void IP_c2f(Int* Nc, Int* Nf, Complex* tilde, Complex* tildef);
void IP_f2c(Int* Nc, Int* Nf, Complex* tilde, Complex* tildef);
"""

HPSI_WRAPPERS = r"""
}  // namespace pwref
extern "C" {
// a3 += (kinetic + V_loc + V_nl) psi for nb bands (psi, a3: nb x ntot), the
// projector sets in the flat form of pw_set_nonlocal (VAL columns)
int ref_add_mult_spinor(const int* n, const int* nf, const double* L, const double* ekin_r2c, const double* vtot,
                        int natom, const int* atom_npts, const int* atom_nproj, const int* idx, const double* beta,
                        const double* wgt, int nb, double* psi, double* a3) {
  using namespace pwref;
  try {
    Fourier fft;
    fft.setup(n, nf, L);
    DblNumVec ekin(fft.numGridTotalR2C), vt(fft.domain.NumGridTotalFine());
    for (Int i = 0; i < fft.numGridTotalR2C; ++i) ekin[i] = ekin_r2c[i];
    for (Int i = 0; i < fft.domain.NumGridTotalFine(); ++i) vt[i] = vtot[i];
    std::vector<PseudoPot> pseudo(natom);
    long io = 0, bo = 0, wo = 0;
    for (int a = 0; a < natom; ++a) {
      for (int l = 0; l < atom_nproj[a]; ++l) {
        SparseVec sv;
        sv.first = IntNumVec(atom_npts[a]);
        sv.second = DblNumMat(atom_npts[a], 4);
        for (int i = 0; i < atom_npts[a]; ++i) {
          sv.first[i] = idx[io + i];
          sv.second.VecData(VAL)[i] = beta[bo + (long)l * atom_npts[a] + i];
        }
        pseudo[a].vnlList.push_back(std::make_pair(sv, wgt[wo + l]));
      }
      io += atom_npts[a];
      bo += (long)atom_nproj[a] * atom_npts[a];
      wo += atom_nproj[a];
    }
    Spinor sp(fft.domain, psi, nb);
    NumTns<Real> out(fft.domain.NumGridTotal(), 1, nb, a3);
    sp.AddMultSpinorFineR2C(fft, ekin, vt, pseudo, out);
  } catch (...) {
    return -1;
  }
  return 0;
}
// ref_add_mult_spinor with the bands split over nthreads OpenMP threads, one
// Fourier per thread (the reference's MPI ranks each hold their own)
int ref_add_mult_spinor_omp(const int* n, const int* nf, const double* L, const double* ekin_r2c, const double* vtot,
                            int natom, const int* atom_npts, const int* atom_nproj, const int* idx, const double* beta,
                            const double* wgt, int nb, double* psi, double* a3, int nthreads) {
  using namespace pwref;
  int bad = 0;
  try {
    Fourier f0;
    f0.setup(n, nf, L);
    for (int d = 0; d < 3; ++d) {   // the length tables are built before the threads start
      fft_len(n[d]);
      fft_len(nf[d]);
    }
    DblNumVec ekin(f0.numGridTotalR2C), vt(f0.domain.NumGridTotalFine());
    for (Int i = 0; i < f0.numGridTotalR2C; ++i) ekin[i] = ekin_r2c[i];
    for (Int i = 0; i < f0.domain.NumGridTotalFine(); ++i) vt[i] = vtot[i];
    std::vector<PseudoPot> pseudo(natom);
    long io = 0, bo = 0, wo = 0;
    for (int a = 0; a < natom; ++a) {
      for (int l = 0; l < atom_nproj[a]; ++l) {
        SparseVec sv;
        sv.first = IntNumVec(atom_npts[a]);
        sv.second = DblNumMat(atom_npts[a], 4);
        for (int i = 0; i < atom_npts[a]; ++i) {
          sv.first[i] = idx[io + i];
          sv.second.VecData(VAL)[i] = beta[bo + (long)l * atom_npts[a] + i];
        }
        pseudo[a].vnlList.push_back(std::make_pair(sv, wgt[wo + l]));
      }
      io += atom_npts[a];
      bo += (long)atom_nproj[a] * atom_npts[a];
      wo += atom_nproj[a];
    }
    const long ntot = f0.domain.NumGridTotal();
#pragma omp parallel num_threads(nthreads)
    {
      Fourier fft;   // per thread, reused over its bands
      fft.setup(n, nf, L);
#pragma omp for schedule(dynamic, 1)
      for (int b = 0; b < nb; ++b) {
        try {
          Spinor sp(fft.domain, psi + b * ntot, 1);
          NumTns<Real> out(ntot, 1, 1, a3 + b * ntot);
          sp.AddMultSpinorFineR2C(fft, ekin, vt, pseudo, out);
        } catch (...) {
#pragma omp atomic write
          bad = 1;
        }
      }
    }
  } catch (...) {
    return -1;
  }
  return bad ? -1 : 0;
}
// a3 += C2R(teter * R2C(r)) for nb bands
int ref_add_teter(const int* n, const int* nf, const double* L, const double* teter_r2c, int nb, double* r,
                  double* a3) {
  using namespace pwref;
  try {
    Fourier fft;
    fft.setup(n, nf, L);
    DblNumVec teter(fft.numGridTotalR2C);
    for (Int i = 0; i < fft.numGridTotalR2C; ++i) teter[i] = teter_r2c[i];
    Spinor sp(fft.domain, r, nb);
    NumTns<Real> out(fft.domain.NumGridTotal(), 1, nb, a3);
    sp.AddTeterPrecond(&fft, teter, out);
  } catch (...) {
    return -1;
  }
  return 0;
}
}
"""


def build_hpsi(ref_root: Path = DEFAULT_REF) -> Path | None:
    """Compile the reference's H*psi composition into oracle/_ref/libpwref_hpsi.so."""
    util = ref_root / "src" / "utility.cpp"
    spinor = ref_root / "src" / "SCF" / "spinor.cpp"
    fourier = ref_root / "src" / "SCF" / "fourier.cpp"
    if not (util.exists() and spinor.exists() and fourier.exists()):
        return LIB_HPSI if LIB_HPSI.exists() else None
    ut = _strip_comments(util.read_text(errors="replace"))
    sp = _strip_comments(spinor.read_text(errors="replace"))
    fo = _strip_comments(fourier.read_text(errors="replace"))
    parts = [_extract(ut, "void IP_c2f("), _extract(ut, "void IP_f2c(")]
    parts += [_extract(fo, h) for h in HPSI_FUNCS]
    parts += [ret + _extract(sp, h) for h, ret in HPSI_METHODS]
    OUT.mkdir(exist_ok=True)
    cpp = OUT / "ref_hpsi.cpp"
    cpp.write_text(HPSI_HARNESS + "\n\n".join(parts) + HPSI_WRAPPERS)
    r = subprocess.run(["g++", "-O3", "-march=x86-64-v2", "-fcx-limited-range", "-fopenmp", "-fPIC", "-shared", "-o", str(LIB_HPSI), str(cpp)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return LIB_HPSI


if __name__ == "__main__":
    print(build())
