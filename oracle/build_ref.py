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
    return LIB


if __name__ == "__main__":
    print(build())
