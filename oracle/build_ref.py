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
``wpbe_analy_erfc_approx_grad`` and ``EXPINT`` (src/utility.cpp:3340-3911).  The recipe extracts each function body from
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
         ("Real EXPINT(", "EXPINT")]

PRELUDE = """// generated: functions compiled from the reference source tree
#include <stdlib.h>
#include <cmath>
#include <complex>
#include <stdexcept>
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
static void fft1(Complex* a, int n, int sign) {
  if (n <= 1) return;
  int p = 2;
  while (n % p) ++p;
  if (p == n) {
    std::vector<Complex> out(n);
    for (int k = 0; k < n; ++k) {
      Complex s(0, 0);
      for (int j = 0; j < n; ++j) s += a[j] * std::polar(1.0, sign * 2.0 * M_PI * (double)((long)j * k % n) / n);
      out[k] = s;
    }
    for (int k = 0; k < n; ++k) a[k] = out[k];
    return;
  }
  const int m = n / p;
  std::vector<std::vector<Complex>> sub(p, std::vector<Complex>(m));
  for (int r = 0; r < p; ++r)
    for (int j = 0; j < m; ++j) sub[r][j] = a[j * p + r];
  for (int r = 0; r < p; ++r) fft1(sub[r].data(), m, sign);
  for (int k = 0; k < n; ++k) {
    Complex s(0, 0);
    for (int r = 0; r < p; ++r) s += sub[r][k % m] * std::polar(1.0, sign * 2.0 * M_PI * (double)((long)r * k % n) / n);
    a[k] = s;
  }
}
static void fft3(std::vector<Complex>& a, const int* n, int sign) {
  std::vector<Complex> line;
  for (int ax = 0; ax < 3; ++ax) {
    const long stride = ax == 0 ? 1 : ax == 1 ? n[0] : (long)n[0] * n[1];
    const int len = n[ax];
    line.resize(len);
    const long total = (long)n[0] * n[1] * n[2];
    for (long base = 0; base < total; ++base) {
      // base enumerates the lines: skip points that are not the start of a line
      const long pos = (base / stride) % len;
      if (pos != 0) continue;
      for (int t = 0; t < len; ++t) line[t] = a[base + t * stride];
      fft1(line.data(), len, sign);
      for (int t = 0; t < len; ++t) a[base + t * stride] = line[t];
    }
  }
}
static void fftw_execute(fftw_plan p) {
  const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2], h0 = n0 / 2 + 1;
  const long N = (long)n0 * n1 * n2;
  std::vector<Complex> a(N);
  if (p->real_to_complex) {
    for (long i = 0; i < N; ++i) a[i] = Complex(p->rdata[i], 0.0);
    fft3(a, p->n, -1);
    for (int k = 0; k < n2; ++k)
      for (int j = 0; j < n1; ++j)
        for (int i = 0; i < h0; ++i) p->cdata[(k * (long)n1 + j) * h0 + i] = a[(k * (long)n1 + j) * n0 + i];
  } else {
    for (int k = 0; k < n2; ++k)
      for (int j = 0; j < n1; ++j)
        for (int i = 0; i < n0; ++i) {
          Complex v;
          if (i < h0) v = p->cdata[(k * (long)n1 + j) * h0 + i];
          else v = std::conj(p->cdata[(((n2 - k) % n2) * (long)n1 + (n1 - j) % n1) * h0 + (n0 - i)]);
          a[(k * (long)n1 + j) * n0 + i] = v;
        }
    fft3(a, p->n, +1);
    for (long i = 0; i < N; ++i) p->rdata[i] = a[i].real();
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
    r = subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-o", str(LIB_HPSI), str(cpp)], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return LIB_HPSI


if __name__ == "__main__":
    print(build())
