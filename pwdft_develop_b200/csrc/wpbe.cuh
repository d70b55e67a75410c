// Short-range PBE exchange of HSE06 on the device (FP64): pbexsr and
// wpbe_analy_erfc_approx_grad of the reference (src/utility.cpp:3340-3846),
// used by KohnSham::CalculateXC for XC_HYB_GGA_XC_HSE06 with omega = 0.106 and
// fraction 0.25 (src/SCF/hamiltonian.cpp:1614-1627).
//
// The screened enhancement factor is the Ernzerhof-Perdew exchange hole
// (J. Chem. Phys. 109, 3313 (1998)) integrated against erfc(w y), w =
// omega / k_F, as in Heyd, Scuseria and Ernzerhof (J. Chem. Phys. 118, 8207
// (2003)): erfc exact in the regular part, the published fit
// (1 + sum_k ea_k x^k) e^{-eb1 x^2} in the singular A / y^2 part.  The
// integrals use closed forms derived for this implementation:
//   regular   int y^{2n+1} e^{-a y^2} erfc(w y) dy
//               = n! / (2 a^{n+1}) [1 - (w / r) sum_{k<=n} binom(2k,k) 4^{-k} (a / r^2)^k],
//             r = sqrt(a + w^2), a = D + s^2 H;
//   singular  A [T_0 + sum_{k=1..8} ea_k w^k T_k],
//             T_0 = (ln q - ln p) / 2 + e^x E1(x) / 2,
//             T_k = M_{k-1}(p) - L_{k-1}(q),
//             p = a + eb1 w^2, q = s^2 H + eb1 w^2, lambda = 4 A / 9, x = q / lambda,
//             M_j(q) = Gamma((j+1)/2) / (2 q^{(j+1)/2}),
//             L_0 = pi / (2 sqrt lambda) erfcx(sqrt x), L_1 = e^x E1(x) / (2 lambda),
//             L_{j+2} = (M_j(q) - L_j) / lambda.
// d F / d s and d F / d w come from forward-mode dual numbers.
#pragma once

#include <cmath>

namespace pwb {
namespace wpbe {

// value and partials with respect to (s, w)
struct D3 {
  double v, s, w;
};
__device__ __forceinline__ D3 mk(double v) { return {v, 0.0, 0.0}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.v + b.v, a.s + b.s, a.w + b.w}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.v - b.v, a.s - b.s, a.w - b.w}; }
__device__ __forceinline__ D3 operator-(D3 a) { return {-a.v, -a.s, -a.w}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) { return {a.v * b.v, a.s * b.v + a.v * b.s, a.w * b.v + a.v * b.w}; }
__device__ __forceinline__ D3 operator+(D3 a, double b) { return {a.v + b, a.s, a.w}; }
__device__ __forceinline__ D3 operator+(double b, D3 a) { return {a.v + b, a.s, a.w}; }
__device__ __forceinline__ D3 operator-(double b, D3 a) { return {b - a.v, -a.s, -a.w}; }
__device__ __forceinline__ D3 operator*(double b, D3 a) { return {b * a.v, b * a.s, b * a.w}; }
__device__ __forceinline__ D3 operator/(D3 a, D3 b) {
  const double q = a.v / b.v;
  return {q, (a.s - q * b.s) / b.v, (a.w - q * b.w) / b.v};
}
__device__ __forceinline__ D3 operator/(D3 a, double b) { return {a.v / b, a.s / b, a.w / b}; }
__device__ __forceinline__ D3 operator/(double b, D3 a) { return mk(b) / a; }
__device__ __forceinline__ D3 chain(D3 a, double f, double df) { return {f, df * a.s, df * a.w}; }
__device__ __forceinline__ D3 dsqrt(D3 a) {
  const double r = sqrt(a.v);
  return chain(a, r, 0.5 / r);
}
__device__ __forceinline__ D3 dlog(D3 a) { return chain(a, log(a.v), 1.0 / a.v); }
// erfcx(y) = e^{y^2} erfc(y), d/dy = 2 y erfcx(y) - 2 / sqrt(pi)
__device__ __forceinline__ D3 derfcx(D3 a) {
  const double f = erfcx(a.v);
  return chain(a, f, 2.0 * a.v * f - 1.1283791670955126);
}

// g(x) = e^x E1(x) for x > 0: the power series of E1 for x <= 1, the
// continued fraction g(x) = 1 / (x + 1 - 1 / (x + 3 - 4 / (x + 5 - ...)))
// (modified Lentz) above.  Relative accuracy ~1e-16.
__device__ __forceinline__ double expe1(double x) {
  if (x <= 1.0) {
    double sum = 0.0, term = 1.0;
    for (int k = 1; k <= 40; ++k) {
      term *= -x / k;
      const double d = term / k;
      sum += d;
      if (fabs(d) < 1e-17 * fabs(sum)) break;
    }
    return exp(x) * (-0.57721566490153286061 - log(x) - sum);
  }
  const double tiny = 1e-300;
  double f = x + 1.0, c = f, dd = 0.0;
  for (int i = 1; i <= 300; ++i) {
    const double an = -(double)i * (double)i, bn = x + 2.0 * i + 1.0;
    dd = bn + an * dd;
    if (fabs(dd) < tiny) dd = tiny;
    c = bn + an / c;
    if (fabs(c) < tiny) c = tiny;
    dd = 1.0 / dd;
    const double del = c * dd;
    f *= del;
    if (fabs(del - 1.0) < 1e-16) break;
  }
  return 1.0 / f;
}
__device__ __forceinline__ D3 dexpe1(D3 a) {
  const double f = expe1(a.v);
  return chain(a, f, f - 1.0 / a.v);
}

// Ernzerhof-Perdew hole and HSE erfc-fit parameters (the published values)
constexpr double kA = 1.0161144, kB = -3.7170836e-1, kC = -7.7215461e-2, kD = 5.7786348e-1, kE = -5.1955731e-2;
constexpr double kHa1 = 9.79681e-3, kHa2 = 4.10834e-2, kHa3 = 1.87440e-1, kHa4 = 1.20824e-3, kHa5 = 3.47188e-2;
constexpr double kFc1 = 6.4753871, kFc2 = 4.7965830e-1;
constexpr double kEGa1 = -2.628417880e-2, kEGa2 = -7.117647788e-2, kEGa3 = 8.534541323e-2, kEGscut = 8.0e-2;
constexpr double kEb1 = 1.455915450052607, kEb1Far = 2.0, kWcut = 14.0;
__device__ __forceinline__ double ea(int k) {
  constexpr double c[8] = {-1.128223946706117, 1.452736265762971, -1.243162299390327, 0.971824836115601,
                           -0.568861079687373, 0.246880514820192, -0.065032363850763, 0.008401793031216};
  return c[k];
}

// F_x(s, w), dF/ds, dF/dw (w > 0)
__device__ inline void fx(double s_, double w_, double& F, double& dFs, double& dFw) {
  const double spi = 1.7724538509055160273, pi = 3.14159265358979323846;
  const D3 s = {s_, 1.0, 0.0}, w = {w_, 0.0, 1.0};
  const D3 s2 = s * s, s4 = s2 * s2;
  const D3 H = (kHa1 * s2 + kHa2 * s4) / (1.0 + kHa3 * s4 + kHa4 * (s4 * s) + kHa5 * (s4 * s2));
  const D3 Fs = kFc1 * H + kFc2;
  const D3 h = s2 * H;
  const D3 a = kD + h;
  D3 EG;
  if (s_ > kEGscut) {
    const D3 sa = dsqrt(a);
    const D3 a72 = a * a * a * sa;
    const D3 ga = spi * (15.0 * kE + 6.0 * kC * (1.0 + Fs * s2) * a + 4.0 * kB * (a * a) + 8.0 * kA * (a * a * a)) /
                      (16.0 * a72) -
                  0.75 * pi * sqrt(kA) * derfcx(1.5 * s * dsqrt(H / kA));
    const D3 gb = (15.0 / 16.0) * spi * s2 / a72;
    EG = -(0.75 * pi + ga) / gb;
  } else {
    EG = kEGa1 + kEGa2 * s2 + kEGa3 * s4;
  }
  // regular part, exact erfc
  const D3 r = dsqrt(a + w * w);
  const D3 t = a / (r * r);
  const D3 wr = w / r;
  const D3 k0 = (1.0 - wr) / (2.0 * a);
  const D3 k1 = (1.0 - wr * (1.0 + 0.5 * t)) / (2.0 * (a * a));
  const D3 k2 = (1.0 - wr * (1.0 + 0.5 * t + 0.375 * (t * t))) / (a * a * a);
  const D3 reg = kB * k0 + kC * (1.0 + s2 * Fs) * k1 + (kE + s2 * EG) * k2;
  // singular part, erfc fit
  const bool far = w_ > kWcut;
  const double eb1 = far ? kEb1Far : kEb1;
  const D3 beta = eb1 * (w * w);
  const D3 p = a + beta, q = h + beta;
  const double lam = 4.0 * kA / 9.0;
  const D3 x = q / lam;
  const D3 g1 = dexpe1(x);
  D3 sing = 0.5 * (dlog(q) - dlog(p)) + 0.5 * g1;
  if (!far) {
    // M_j(y) = Gamma((j+1)/2) / (2 y^{(j+1)/2}), j = 0..7
    constexpr double gam[8] = {1.7724538509055160273, 1.0, 0.88622692545275801365, 1.0,
                               1.3293403881791370205, 2.0, 3.3233509704478425512, 6.0};
    const D3 rq = dsqrt(q), rp = dsqrt(p);
    D3 mq[8], mp[8];
    D3 pq = rq, pp = rp;   // y^{(j+1)/2}
    for (int j = 0; j < 8; ++j) {
      mq[j] = gam[j] / (2.0 * pq);
      mp[j] = gam[j] / (2.0 * pp);
      pq = pq * rq;
      pp = pp * rp;
    }
    D3 L[8];
    L[0] = (0.5 * pi / sqrt(lam)) * derfcx(dsqrt(x));
    L[1] = g1 / (2.0 * lam);
    for (int j = 2; j < 8; ++j) L[j] = (mq[j - 2] - L[j - 2]) / lam;
    D3 wk = mk(1.0), poly = mk(0.0);
    for (int k = 1; k <= 8; ++k) {
      wk = wk * w;
      poly = poly + ea(k - 1) * (wk * (mp[k - 1] - L[k - 1]));
    }
    sing = sing + poly;
  }
  const D3 f = (-8.0 / 9.0) * (kA * sing + reg);
  F = f.v;
  dFs = f.s;
  dFw = f.w;
}

// pbexsr: short-range exchange energy density sx (per volume), v1 = d sx / d rho,
// v2 = (1 / |grad rho|) d sx / d |grad rho|, with the reference's clamp of s > 8.3
__device__ inline void pbexsr(double rho, double grho2, double omega, double& sx, double& v1, double& v2) {
  const double us = 0.161620459673995492, ax = -0.738558766382022406;
  const double rs = cbrt(rho);
  const double vx = (4.0 / 3.0) * ax * rs;
  const double rr = 1.0 / (rho * rs);
  const double ex = ax / rr;
  const double s2 = grho2 * rr * rr * us * us;
  double s = sqrt(s2);
  if (s > 8.3) s = 8.572844 - 18.796223 / s2;
  const double kf = cbrt(3.0 * 9.86960440108935861883 * rho);
  const double w = omega / kf;
  double F, dFs, dFw;
  fx(s, w, F, dFs, dFw);
  const double d1x = dFw * (-w / (3.0 * rho));
  sx = ex * F;
  v1 = vx * F + (-4.0 / 3.0 * s / rho * dFs + d1x) * ex;
  v2 = ex / sqrt(grho2) * (us * rr) * dFs;
}

}  // namespace wpbe
}  // namespace pwb
