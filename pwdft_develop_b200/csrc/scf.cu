// Block eigensolvers and the Gamma-point SCF driver on the device.
//
//  * Cholesky-QR        EigenSolver::Orthogonalize   src/EigenSolver/eigensolver.cpp:301-384
//  * LOBPCG             EigenSolver::LOBPCGSolveReal src/EigenSolver/lobpcg.cpp:577-1031
//    (no locking, first iteration on (X, W), later (X, W, P), residual
//    ||r|| / max(1, |lambda|), SolveGenEig on the 2n or 3n block, final RR)
//  * ChebFSI            Chebyshev-filtered subspace iteration (Zhou, Saad,
//    Tiago, Chelikowsky, J. Comput. Phys. 219, 172 (2006)); the reference only
//    keeps its parameters (src/esdf.cpp:2715-2719) and calls (scf.cpp:1299-1334)
//  * SCF                SCF::Iterate / InnerSolve (scf.cpp:372-591, 1261-1589):
//    density (hamiltonian.cpp:2455-2627), Hartree (:1990-2026), LDA Teter93 XC
//    (:1242-1308), Vtot (:2029-2069), occupations (scf.cpp:1748-1830), energies
//    (:1834-2140), Anderson potential mixing (:2299-2365).
//
// FP64 everywhere except, in mixed mode, the eigensolver's H*psi, block
// updates and Gram products, which run in an FP32 twin context (FP32 FFTs,
// split-BF16 tensor-core Grams with FP32 accumulation).  Small dense problems
// (Cholesky, Rayleigh-Ritz eigenproblems) are FP64 on the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <vector>

#include "blockops.hpp"
#include "common.hpp"
#include "fft.cuh"
#include "fft3d.cuh"
#include "gemm.hpp"
#include "wpbe.cuh"

namespace pwb {

int run_density(pw_ctx* c, const void* psi, int ld, int nband, int band0, int npair, const double* w, double* rho,
                cudaStream_t st);
int gram(pw_ctx* c, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G, int ldg,
         cudaStream_t st, int nrow = -1);
int upload_real(pw_ctx* c, DevBuf& dst, const double* src, size_t n);
int wfn_filter_pass(pw_ctx* c, void* X, int ld, int nb, cudaStream_t st);
int refresh_vperm(pw_ctx* c);

// Hartree on the fine grid: vh = (1/N) IFFT( kern * FFT(rho - rho_ps) ),
// kern = 2 pi / gkk (0 for gkk <= 1e-16 or gkk > 4 Ecut).  Cubic grids only.
template <int N> static int hartree_n(double2* work, const double* rho, const double* rps, const double* kern,
                                      double* vh, const double2* tw, cudaStream_t st) {
  const int nrowtiles = (N * N + AX_TILE - 1) / AX_TILE;
  const int nxt = (N + AX_TILE - 1) / AX_TILE;
  k_fft_axis<N, -1, 0, 1><<<nrowtiles, AX_THREADS, 0, st>>>(work, N, N, N, rho, rps, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, -1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, -1, 2, 2><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, kern, nullptr, 1.0, tw);
  k_fft_axis<N, +1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
  // kern already carries the 1/N normalisation of the unnormalised transforms
  k_fft_axis<N, +1, 0, 3><<<nrowtiles, AX_THREADS, 0, st>>>(work, N, N, N, nullptr, nullptr, nullptr, vh, 1.0, tw);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

static int hartree(pw_ctx* c, double2* work, const double* rho, const double* rps, const double* kern, double* vh,
                   const double2* tw, cudaStream_t st) {
  PWB_CHECK(c->nf[0] == c->nf[1] && c->nf[1] == c->nf[2], PW_EUNSUPPORTED, "SCF Hartree needs a cubic fine grid");
  switch (c->nf[0]) {
    case 24: return hartree_n<24>(work, rho, rps, kern, vh, tw, st);
    case 32: return hartree_n<32>(work, rho, rps, kern, vh, tw, st);
    case 48: return hartree_n<48>(work, rho, rps, kern, vh, tw, st);
    case 96: return hartree_n<96>(work, rho, rps, kern, vh, tw, st);
    case 144: return hartree_n<144>(work, rho, rps, kern, vh, tw, st);
    default: set_error("SCF fine grid size not built"); return PW_EUNSUPPORTED;
  }
}

// LDA Teter93 (Goedecker, Teter, Hutter, PRB 54, 1703 (1996)); bad points zeroed
__global__ void k_xc_teter93(long n, const double* __restrict__ rho, double* __restrict__ eps, double* __restrict__ vxc) {
  const double a0 = 0.4581652932831429, a1 = 2.217058676663745, a2 = 0.7405551735357053, a3 = 0.01968227878617998;
  const double b1 = 1.0, b2 = 4.504130959426697, b3 = 1.110667363742916, b4 = 0.02359291751427506;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double r = rho[i];
    if (r < 1e-10) { eps[i] = 0.0; vxc[i] = 0.0; continue; }
    const double rs = cbrt(3.0 / (4.0 * M_PI * r));
    const double N_ = a0 + rs * (a1 + rs * (a2 + rs * a3));
    const double D = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)));
    const double dN = a1 + rs * (2 * a2 + rs * 3 * a3);
    const double dD = b1 + rs * (2 * b2 + rs * (3 * b3 + rs * 4 * b4));
    const double e = -N_ / D;
    const double de = -(dN * D - N_ * dD) / (D * D);
    eps[i] = e;
    vxc[i] = e - rs / 3.0 * de;
  }
}

// out[k] += sum_i a_k[i] * b_k[i] for K pairs
struct DotSet {
  const double* a[6];
  const double* b[6];
  int k;
};
__global__ void k_dots(long n, DotSet d, double* out) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    for (int k = 0; k < d.k; ++k) s[k] += d.a[k][i] * (d.b[k] ? d.b[k][i] : 1.0);
  __shared__ double red[6][32];
  for (int k = 0; k < d.k; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int k = 0; k < d.k; ++k) {
      double v = (threadIdx.x < (blockDim.x >> 5)) ? red[k][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) atomicAdd(&out[k], v);
    }
  }
}

__global__ void k_lincomb(long n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                          double* __restrict__ z) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = a * x[i] + (y ? b * y[i] : 0.0);
}
__global__ void k_init_rho(long n, const double* __restrict__ rps, double* __restrict__ rho) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    rho[i] = rps[i] > 1e-6 ? rps[i] : 1e-6;
}

static inline int nblk(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 8); }

// ---------------------------------------------------------------------------
// PBE (unpolarised): the Use_Libxc 0 branch of KohnSham::CalculateXC
// (src/SCF/hamiltonian.cpp:1381-1419, 1560-1612, 1680-1760) with the
// gradient of KohnSham::CalculateGradDensity (hamiltonian.cpp:1153-1239).
// Point functions: Slater exchange, Perdew-Wang 1992 correlation and the PBE
// gradient corrections (Perdew, Burke, Ernzerhof, PRL 77, 3865 (1996)) in the
// constants of the reference's VExchange_sla / VCorrelation_pw /
// VGCExchange_pbx / VGCCorrelation_pbc (src/utility.cpp:3913-4244).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pw92_point(double rs, double& ec, double& vc) {
  const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
  const double q = sqrt(rs);
  const double om = 2.0 * a * (b1 * q + b2 * rs + b3 * rs * q + b4 * rs * rs);
  const double rdom = 2.0 * a * (0.5 * b1 * q + b2 * rs + 1.5 * b3 * rs * q + 2.0 * b4 * rs * rs);   // rs d om/d rs
  const double lg = log(1.0 + 1.0 / om);
  ec = -2.0 * a * (1.0 + a1 * rs) * lg;
  vc = -2.0 * a * (1.0 + 2.0 / 3.0 * a1 * rs) * lg - 2.0 / 3.0 * a * (1.0 + a1 * rs) * rdom / (om * (om + 1.0));
}

// eps (per particle), v1 = d(rho eps)/d rho, v2 = 2 d(rho eps)/d sigma at one point
__device__ __forceinline__ void pbe_point(double rho, double sigma, double& eps, double& v1, double& v2) {
  const double third = 1.0 / 3.0;
  const double ar = fabs(rho);
  eps = 0.0;
  v1 = 0.0;
  v2 = 0.0;
  if (ar > 1e-10) {
    const double rs = pow(3.0 / 4.0 / M_PI / ar, third);
    const double ux = -0.458165293283143 / rs;   // Slater, -(3/4pi)(9pi/4)^(1/3) / rs
    double uc, vc;
    pw92_point(rs, uc, vc);
    eps = ux + uc;
    v1 = 4.0 / 3.0 * ux + vc;
  }
  if (ar > 1e-6 && sigma > 1e-10) {
    // exchange: F_x - 1 = kappa - kappa / (1 + mu s^2 / kappa), s = |grad rho| / (2 k_F rho)
    const double kappa = 0.804, mu = 0.2195149727645171;
    const double g = sqrt(sigma);
    const double kf = 3.093667726280136 * pow(ar, third);
    const double dsg = 0.5 / kf;
    const double s = g * dsg / ar;
    const double den = 1.0 + s * s * mu / kappa;
    const double fx = kappa - kappa / den;
    const double exu = -0.75 / M_PI * kf;
    const double dfx = 2.0 * mu * s / (den * den);
    const double ex = exu * fx;
    // correlation: H = gamma ln(1 + beta/gamma t^2 (1 + A t^2) / (1 + A t^2 + A^2 t^4))
    const double gam = 0.03109069086965, bet = 0.06672455060314922;
    const double rs = 0.6203504908994 / pow(ar, third);
    double ec0, vc0;
    pw92_point(rs, ec0, vc0);
    const double ks = 1.128379167095513 * sqrt(1.919158292677513 / rs);
    const double t2 = sigma / ((2.0 * ks * ar) * (2.0 * ks * ar));
    const double ee = exp(-ec0 / gam);
    const double A = bet / gam * (1.0 / (ee - 1.0));
    const double y = A * t2;
    const double d = 1.0 + y + y * y;
    const double xy = (1.0 + y) / d;
    const double qy = y * y * (2.0 + y) / (d * d);
    const double s1 = 1.0 + bet / gam * t2 * xy;
    const double H = gam * log(s1);
    const double rdh = bet * t2 / s1 * (-7.0 / 3.0 * xy - qy * (A * ee * (vc0 - ec0) / bet - 7.0 / 3.0));
    eps += ex + H;
    v1 += ex + exu / 3.0 * fx - exu * dfx * (4.0 / 3.0) * s + H + rdh;
    v2 = exu * dfx * dsg / g + bet / (2.0 * ks * ks * ar) * (xy - qy) / s1;
  }
}

// gradient components g0..g2 in, h_d = v2 g_d out (in place); eps, v1 out.
// hse_frac > 0: semilocal HSE06, minus hse_frac times the short-range PBE
// exchange of screening omega where |rho| > 1e-6 and sigma > 1e-10
// (hamiltonian.cpp:1614-1627; |rho| is passed where the reference passes rho,
// which differs only for rho < -1e-6, where its cube root is not a number)
__global__ void k_pbe(long n, const double* __restrict__ rho, double* __restrict__ g0, double* __restrict__ g1,
                      double* __restrict__ g2, double* __restrict__ eps, double* __restrict__ v1, double hse_frac,
                      double omega) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double a = g0[i], b = g1[i], c = g2[i];
    const double r = rho[i], sigma = a * a + b * b + c * c;
    double e, u, w;
    pbe_point(r, sigma, e, u, w);
    if (hse_frac != 0.0 && fabs(r) > 1e-6 && sigma > 1e-10) {
      double sx, v1x, v2x;
      wpbe::pbexsr(fabs(r), sigma, omega, sx, v1x, v2x);
      e -= hse_frac * sx / r;
      u -= hse_frac * v1x;
      w -= hse_frac * v2x;
    }
    eps[i] = e;
    v1[i] = u;
    g0[i] = w * a;
    g1[i] = w * b;
    g2[i] = w * c;
  }
}

// dst (+)= src * i G_d / N, zero where gkk = 0 or gkk > 4 Ecut (ikFine and the
// cut of hamiltonian.cpp:1196-1201); full cubic fine spectrum, x fastest
__global__ void k_spec_deriv(int N, double g, double gmax2, int d, const double2* __restrict__ src,
                             double2* __restrict__ dst, int accumulate) {
  const long n = (long)N * N * N;
  const double inv = 1.0 / (double)n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / ((long)N * N));
    const double mx = x <= N / 2 ? x : x - N, my = y <= N / 2 ? y : y - N, mz = z <= N / 2 ? z : z - N;
    const double gx = g * mx, gy = g * my, gz = g * mz;
    const double gkk = (gx * gx + gy * gy + gz * gz) / 2;
    const double gd = d == 0 ? gx : (d == 1 ? gy : gz);
    const double k = (gkk == 0.0 || gkk > gmax2) ? 0.0 : gd * inv;
    const double2 v = src[i];
    const double2 r = make_double2(-k * v.y, k * v.x);
    if (accumulate) dst[i] = make_double2(dst[i].x + r.x, dst[i].y + r.y);
    else dst[i] = r;
  }
}

// unnormalised forward 3-D FFT of a real field, and inverse to a real field
template <int N> static void fft3_fwd_real(double2* w, const double* rin, const double2* tw, cudaStream_t st) {
  const int nrowtiles = (N * N + AX_TILE - 1) / AX_TILE, nxt = (N + AX_TILE - 1) / AX_TILE;
  k_fft_axis<N, -1, 0, 1><<<nrowtiles, AX_THREADS, 0, st>>>(w, N, N, N, rin, nullptr, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, -1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(w, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, -1, 2, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(w, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
}
template <int N>
static void fft3_inv_real(double2* w, double* rout, const double2* tw, cudaStream_t st, double scale = 1.0) {
  const int nrowtiles = (N * N + AX_TILE - 1) / AX_TILE, nxt = (N + AX_TILE - 1) / AX_TILE;
  k_fft_axis<N, +1, 2, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(w, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, +1, 1, 0><<<dim3(nxt, N), AX_THREADS, 0, st>>>(w, N, N, N, nullptr, nullptr, nullptr, nullptr, 1.0, tw);
  k_fft_axis<N, +1, 0, 3><<<nrowtiles, AX_THREADS, 0, st>>>(w, N, N, N, nullptr, nullptr, nullptr, rout, scale, tw);
}

// unnormalised 3-D FFT of a real cubic fine-grid field (forward) or to one (inverse, times scale)
static int fft3_real(int N, bool inverse, double2* w, const double* rin, double* rout, double scale,
                     const double2* tw, cudaStream_t st) {
  switch (N) {
#define PWB_FFT3(n)                                       \
    case n:                                               \
      if (inverse) fft3_inv_real<n>(w, rout, tw, st, scale); \
      else fft3_fwd_real<n>(w, rin, tw, st);              \
      break;
    PWB_FFT3(24) PWB_FFT3(32) PWB_FFT3(48) PWB_FFT3(96) PWB_FFT3(144)
#undef PWB_FFT3
    default: set_error("SCF fine grid size not built"); return PW_EUNSUPPORTED;
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// sum_i w_i Re(conj(a_i) b_i) (RhoDdot with the weights pi vol / gkk)
__global__ void k_wdot(long n, const double* __restrict__ w, const double2* __restrict__ a,
                       const double2* __restrict__ b, double* out) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += w[i] * (a[i].x * b[i].x + a[i].y * b[i].y);
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(out, v);
  }
}
// z = a x + b y (complex arrays, real coefficients; y may be null); optional mask
__global__ void k_clin(long n, double a, const double2* __restrict__ x, double b, const double2* __restrict__ y,
                       const double* __restrict__ mask, double2* __restrict__ z) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 v = make_double2(a * x[i].x, a * x[i].y);
    if (y) { v.x += b * y[i].x; v.y += b * y[i].y; }
    if (mask) { v.x *= mask[i]; v.y *= mask[i]; }
    z[i] = v;
  }
}

// eps (per particle) and V_xc = v1 - sum_d d_d(v2 d_d rho) of PBE on the
// cubic fine grid; scratch: two complex and three real fine fields
template <int N>
static int pbe_n(pw_ctx* c, const double* rho, double ecut, double* eps, double* vxc, double2* S, double2* T,
                 double* g, const double2* tw, cudaStream_t st, double hse_frac) {
  const long n = (long)N * N * N;
  const double gs = 2 * M_PI / c->L[0];
  fft3_fwd_real<N>(S, rho, tw, st);
  for (int d = 0; d < 3; ++d) {
    k_spec_deriv<<<nblk(n), 256, 0, st>>>(N, gs, 4.0 * ecut, d, S, T, 0);
    fft3_inv_real<N>(T, g + d * n, tw, st);
  }
  k_pbe<<<nblk(n), 256, 0, st>>>(n, rho, g, g + n, g + 2 * n, eps, vxc, hse_frac, 0.106);
  for (int d = 0; d < 3; ++d) {
    fft3_fwd_real<N>(S, g + d * n, tw, st);
    k_spec_deriv<<<nblk(n), 256, 0, st>>>(N, gs, 4.0 * ecut, d, S, T, d > 0);
  }
  fft3_inv_real<N>(T, g, tw, st);
  k_lincomb<<<nblk(n), 256, 0, st>>>(n, 1.0, vxc, -1.0, g, vxc);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

static int xc_pbe(pw_ctx* c, const double* rho, double ecut, double* eps, double* vxc, double2* S, double2* T,
                  double* g, const double2* tw, cudaStream_t st, double hse_frac = 0.0) {
  PWB_CHECK(c->nf[0] == c->nf[1] && c->nf[1] == c->nf[2] && c->L[0] == c->L[1] && c->L[1] == c->L[2],
            PW_EUNSUPPORTED, "PBE gradients need a cubic cell and fine grid");
  switch (c->nf[0]) {
    case 24: return pbe_n<24>(c, rho, ecut, eps, vxc, S, T, g, tw, st, hse_frac);
    case 32: return pbe_n<32>(c, rho, ecut, eps, vxc, S, T, g, tw, st, hse_frac);
    case 48: return pbe_n<48>(c, rho, ecut, eps, vxc, S, T, g, tw, st, hse_frac);
    case 96: return pbe_n<96>(c, rho, ecut, eps, vxc, S, T, g, tw, st, hse_frac);
    case 144: return pbe_n<144>(c, rho, ecut, eps, vxc, S, T, g, tw, st, hse_frac);
    default: set_error("SCF fine grid size not built"); return PW_EUNSUPPORTED;
  }
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11)
// and Box-Muller: out[i] ~ N(0,1) for the key `seed`, counter = i / 4.
__device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += W0; k1 += W1;
  }
}
template <typename T>
__global__ void k_gaussian(long n, unsigned long long seed, T* __restrict__ out) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; 4 * q < n; q += (long)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), 0u, 0u};
    philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double two32 = 4294967296.0;
    for (int h = 0; h < 2; ++h) {
      const double u1 = ((double)c[2 * h] + 0.5) / two32, u2 = ((double)c[2 * h + 1] + 0.5) / two32;
      const double rr = sqrt(-2.0 * log(u1));
      double sn, cs;
      sincospi(2.0 * u2, &sn, &cs);
      const long i = 4 * q + 2 * h;
      if (i < n) out[i] = (T)(rr * cs);
      if (i + 1 < n) out[i + 1] = (T)(rr * sn);
    }
  }
}

// ---------------------------------------------------------------------------
// SCF / eigensolver state
// ---------------------------------------------------------------------------
struct Solver {
  pw_ctx* c = nullptr;   // context doing the eigensolve (FP64 or FP32 twin)
  int nb = 0;            // block width
  long nt = 0;
  size_t esz = 8;
  DevBuf X, HX, W, HW, P, HP, Y, HY, Z;   // [nb][nt] blocks
  DevBuf S, HS;                            // LOBPCG [3nb][nt] (X,W,P contiguous)
  DevBuf G1, G2, wbuf;                     // dense FP64 work (3nb x 3nb)
  std::vector<double> eig, res;
  void* ptr(DevBuf& b, long col = 0) { return (char*)b.p + (size_t)col * nt * esz; }
  // Chebyshev filter replayed from a CUDA graph (coefficients in fcoef)
  bool use_graph = false;
  cudaStream_t st = nullptr;
  cudaGraph_t fgraph = nullptr;
  cudaGraphExec_t fexec = nullptr;
  int f_nb = 0, f_m = 0, f_calls = 0;
  void* f_res = nullptr;
  DevBuf fcoef;
  // the whole ChebFSI step (coefficients from the device Ritz values, filter,
  // cut-off filter pass, Cholesky-QR, H*psi, Rayleigh-Ritz) as one graph
  cudaGraph_t sgraph = nullptr;
  cudaGraphExec_t sexec = nullptr;
  int s_nb = 0, s_m = 0, s_calls = 0;
  bool s_off = false;       // capture failed once: the step runs directly
  DevBuf bup;               // upper bound of the spectrum (device scalar)
  DevBuf x32;               // the FP32 block at the switch to FP64 (mixed precision)
  double bup_host = 0.0;
  void drop_graphs() {
    if (fexec) cudaGraphExecDestroy(fexec);
    if (fgraph) cudaGraphDestroy(fgraph);
    if (sexec) cudaGraphExecDestroy(sexec);
    if (sgraph) cudaGraphDestroy(sgraph);
    fexec = nullptr;
    fgraph = nullptr;
    sexec = nullptr;
    sgraph = nullptr;
    f_calls = 0;
    s_calls = 0;
  }
  ~Solver() {
    drop_graphs();
    if (st) cudaStreamDestroy(st);
  }
};

// eigensolver sub-phase timers (H*psi, Gram, dense FP64, rotations), seconds
static bool g_sub_on = false;
static double g_sub[4] = {0, 0, 0, 0};
struct SubTimer {
  int k;
  std::chrono::steady_clock::time_point t0;
  explicit SubTimer(int k_) : k(k_) {
    if (g_sub_on) { cudaDeviceSynchronize(); t0 = std::chrono::steady_clock::now(); }
  }
  ~SubTimer() {
    if (g_sub_on) {
      cudaDeviceSynchronize();
      g_sub[k] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
  }
};

static int hpsi(pw_ctx* c, const void* x, void* y, int nb, cudaStream_t st) {
  SubTimer t_(0);
  return pw_hpsi(c, x, (int)c->ntot, y, (int)c->ntot, nb, 0, st);
}

template <typename T> static int t_axpby(Solver& s, int n, int nb, double a, const void* X, double b, void* Y) {
  return axpby<T>(n, nb, a, (const T*)X, s.nt, b, (T*)Y, s.nt, nullptr);
}
static int v_axpby(Solver& s, int nb, double a, const void* X, double b, void* Y) {
  return s.c->prec == PW_F64 ? t_axpby<double>(s, (int)s.nt, nb, a, X, b, Y) : t_axpby<float>(s, (int)s.nt, nb, a, X, b, Y);
}
static int v_colnorm2(Solver& s, int nb, const void* X, double* out_dev) {
  return s.c->prec == PW_F64 ? colnorm2<double>((int)s.nt, nb, (const double*)X, s.nt, out_dev, nullptr)
                             : colnorm2<float>((int)s.nt, nb, (const float*)X, s.nt, out_dev, nullptr);
}
static int v_colscale(Solver& s, int nb, void* X, const double* sc) {
  return s.c->prec == PW_F64 ? colscale<double>((int)s.nt, nb, (double*)X, s.nt, sc, nullptr)
                             : colscale<float>((int)s.nt, nb, (float*)X, s.nt, sc, nullptr);
}

static int alloc_block(Solver& s, DevBuf& b, int ncol) { return b.alloc((size_t)ncol * s.nt * s.esz); }

// Cholesky-QR: X <- X U^{-1}, S = X^T X = U^T U (Orthogonalize, eigensolver.cpp:301-384).
// On stream st; defer_check: the factorisation's status stays in d.info (no
// host round trip, for a captured step) instead of being checked here
static int cholqr(Solver& s, Dense& d, void* X, int nb, void* tmp, cudaStream_t st = nullptr,
                  bool defer_check = false) {
  int rc;
  if ((rc = s.G1.alloc((size_t)nb * nb * 8))) return rc;
  double* G = (double*)s.G1.p;
  { SubTimer t_(1); if ((rc = gram(s.c, X, (int)s.nt, nb, X, (int)s.nt, nb, G, nb, st))) return rc; }
  SubTimer td_(2);
  if (defer_check) rc = dense_potrf_upper(nb, G, nb, (int*)d.info.p, st);
  else rc = d.potrf_upper(nb, G, nb, st);
  if (rc) return rc;
  // Uinv = U^{-1} (upper): U * Uinv = I
  if ((rc = s.G2.alloc((size_t)nb * nb * 8))) return rc;
  double* Ui = (double*)s.G2.p;
  if ((rc = dense_trtri_upper(nb, G, nb, Ui, nb, st))) return rc;
  RotBlock rb{X, s.nt, nb, Ui, nb};
  { SubTimer t_(3); if ((rc = rotate(s.c, (int)s.nt, nb, &rb, 1, tmp, s.nt, 0.0, st))) return rc; }
  PWB_CUDA(cudaMemcpyAsync(X, tmp, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice, st));
  return PW_OK;
}

// Rayleigh-Ritz on an orthonormal block Y with HY: eig(Y^T HY) = V diag(l),
// X = Y V, HX = HY V; the eigenvalues in s.wbuf and, unless deferred, s.eig
static int rayleigh_ritz(Solver& s, Dense& d, void* Y, void* HY, void* X, void* HX, int nb, cudaStream_t st = nullptr,
                         bool defer_eig = false) {
  int rc;
  if ((rc = s.G1.alloc((size_t)nb * nb * 8)) || (rc = s.wbuf.alloc((size_t)nb * 8 * 2))) return rc;
  double* A = (double*)s.G1.p;
  { SubTimer t_(1); if ((rc = gram(s.c, Y, (int)s.nt, nb, HY, (int)s.nt, nb, A, nb, st))) return rc; }
  // symmetrise from the upper triangle
  if ((rc = dense_sym_upper(nb, A, nb, st))) return rc;
  double* w = (double*)s.wbuf.p;
  { SubTimer t_(2); if ((rc = d.syevd(nb, A, nb, w, st))) return rc; }
  if (!defer_eig) {
    s.eig.resize(nb);
    PWB_CUDA(cudaMemcpyAsync(s.eig.data(), w, nb * 8, cudaMemcpyDeviceToHost, st));
    PWB_CUDA(cudaStreamSynchronize(st));
  }
  SubTimer t_(3);
  RotBlock r1{Y, s.nt, nb, A, nb};
  if ((rc = rotate(s.c, (int)s.nt, nb, &r1, 1, X, s.nt, 0.0, st))) return rc;
  RotBlock r2{HY, s.nt, nb, A, nb};
  return rotate(s.c, (int)s.nt, nb, &r2, 1, HX, s.nt, 0.0, st);
}

// Chebyshev filter of degree m on [a, b] scaled at a0 (Zhou et al. 2006,
// Algorithm 3.2): on exit Y = p_m(H) X.  X is overwritten.

// k-step Lanczos on a random vector: upper bound of the spectrum
static int lanczos_upper(Solver& s, int k, double* upper, double* lower) {
  DevBuf v, w, v0;
  int rc;
  if ((rc = v.alloc(s.nt * s.esz)) || (rc = w.alloc(s.nt * s.esz)) || (rc = v0.alloc(s.nt * s.esz))) return rc;
  std::mt19937_64 gen(12345);
  std::normal_distribution<double> nd;
  std::vector<double> hv(s.nt);
  double nrm = 0;
  for (auto& x : hv) { x = nd(gen); nrm += x * x; }
  if (s.c->gs) {
    // sphere-cut bands: Im c_0 is not a degree of freedom (H maps it to zero)
    nrm -= hv[1] * hv[1];
    hv[1] = 0;
  }
  nrm = std::sqrt(nrm);
  for (auto& x : hv) x /= nrm;
  if (s.c->prec == PW_F64) PWB_CUDA(cudaMemcpy(v.p, hv.data(), s.nt * 8, cudaMemcpyHostToDevice));
  else {
    std::vector<float> hf(hv.begin(), hv.end());
    PWB_CUDA(cudaMemcpy(v.p, hf.data(), s.nt * 4, cudaMemcpyHostToDevice));
  }
  PWB_CUDA(cudaMemset(v0.p, 0, s.nt * s.esz));
  std::vector<double> al, be;
  DevBuf dot;
  if ((rc = dot.alloc(16))) return rc;
  if (s.c->wfn_filter) {
    // with the cut-off filter the Krylov space must start inside the span of P
    // (where P H is the symmetric P H P): filter and renormalise the start vector
    if ((rc = wfn_filter_pass(s.c, v.p, (int)s.nt, 1, nullptr))) return rc;
    if ((rc = v_colnorm2(s, 1, v.p, (double*)dot.p))) return rc;
    double n2;
    PWB_CUDA(cudaMemcpy(&n2, dot.p, 8, cudaMemcpyDeviceToHost));
    if ((rc = v_axpby(s, 1, 0.0, v.p, 1.0 / std::sqrt(n2), v.p))) return rc;
  }
  double beta = 0;
  for (int j = 0; j < k; ++j) {
    if ((rc = hpsi(s.c, v.p, w.p, 1, nullptr))) return rc;
    // alpha = v . w
    double* G = (double*)dot.p;
    if ((rc = gram(s.c, v.p, (int)s.nt, 1, w.p, (int)s.nt, 1, G, 1, nullptr))) return rc;
    double alpha;
    PWB_CUDA(cudaMemcpy(&alpha, G, 8, cudaMemcpyDeviceToHost));
    al.push_back(alpha);
    // w = w - alpha v - beta v0
    if ((rc = v_axpby(s, 1, -alpha, v.p, 1.0, w.p))) return rc;
    if (j > 0 && (rc = v_axpby(s, 1, -beta, v0.p, 1.0, w.p))) return rc;
    if ((rc = v_colnorm2(s, 1, w.p, G))) return rc;
    double b2;
    PWB_CUDA(cudaMemcpy(&b2, G, 8, cudaMemcpyDeviceToHost));
    beta = std::sqrt(b2);
    be.push_back(beta);
    PWB_CUDA(cudaMemcpy(v0.p, v.p, s.nt * s.esz, cudaMemcpyDeviceToDevice));
    PWB_CUDA(cudaMemcpy(v.p, w.p, s.nt * s.esz, cudaMemcpyDeviceToDevice));
    const double inv = 1.0 / beta;
    if ((rc = v_axpby(s, 1, 0.0, w.p, inv, v.p))) return rc;
  }
  // eigenvalues of the tridiagonal T (host, Jacobi on a k x k matrix)
  const int n = (int)al.size();
  std::vector<double> T((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) {
    T[(size_t)i * n + i] = al[i];
    if (i + 1 < n) T[(size_t)i * n + i + 1] = T[(size_t)(i + 1) * n + i] = be[i];
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += T[(size_t)p * n + q] * T[(size_t)p * n + q];
    if (off < 1e-24) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = T[(size_t)p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (T[(size_t)q * n + q] - T[(size_t)p * n + p]) / (2 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
        for (int r = 0; r < n; ++r) {
          const double a1 = T[(size_t)r * n + p], a2 = T[(size_t)r * n + q];
          T[(size_t)r * n + p] = cs * a1 - sn * a2;
          T[(size_t)r * n + q] = sn * a1 + cs * a2;
        }
        for (int r = 0; r < n; ++r) {
          const double a1 = T[(size_t)p * n + r], a2 = T[(size_t)q * n + r];
          T[(size_t)p * n + r] = cs * a1 - sn * a2;
          T[(size_t)q * n + r] = sn * a1 + cs * a2;
        }
      }
  }
  double mx = -1e300, mn = 1e300;
  for (int i = 0; i < n; ++i) {
    mx = std::max(mx, T[(size_t)i * n + i]);
    mn = std::min(mn, T[(size_t)i * n + i]);
  }
  *upper = mx + beta;
  *lower = mn;
  return PW_OK;
}

// one ChebFSI step on the block X (orthonormal on entry and exit); eigenvalues in s.eig
// The same filter with device-resident coefficients on stream st (capturable):
// coef[0..1] for the first step, coef[3 (i - 1) ..] for step i
static int cheby_filter_dev(Solver& s, int nb, int m, const double* coef, void* X, void* Y, void* Z, void* HY,
                            void** result, cudaStream_t st) {
  int rc;
  const bool f64 = s.c->prec == PW_F64;
  auto lin = [&](const double* c, void* hy, void* y, void* x, void* z) {
    return f64 ? cheb_lin<double>((int)s.nt, nb, c, (const double*)hy, (const double*)y, (const double*)x, (double*)z,
                                  s.nt, st)
               : cheb_lin<float>((int)s.nt, nb, c, (const float*)hy, (const float*)y, (const float*)x, (float*)z,
                                 s.nt, st);
  };
  if ((rc = pw_hpsi(s.c, X, (int)s.nt, HY, (int)s.nt, nb, 0, st))) return rc;
  if ((rc = lin(coef, HY, X, nullptr, Y))) return rc;
  void* xp = X;
  void* yp = Y;
  void* zp = Z;
  for (int i = 2; i <= m; ++i) {
    if ((rc = pw_hpsi(s.c, yp, (int)s.nt, HY, (int)s.nt, nb, 0, st))) return rc;
    if ((rc = lin(coef + 3 * (i - 1), HY, yp, xp, zp))) return rc;
    void* t = xp;
    xp = yp;
    yp = zp;
    zp = t;
  }
  *result = yp;
  return PW_OK;
}

// Chebyshev filter (Zhou-Saad recurrence on [a, b], scaled by the lower bound
// a0).  With s.use_graph the first call runs directly (allocations, library
// handles), the second captures a CUDA graph, later calls only upload the new
// coefficients and replay it; without it every call launches directly.  Both
// run the same kernels in the same order.
static int cheby_filter_run(Solver& s, int nb, int m, double a, double b, double a0, void** result) {
  int rc;
  if (!s.st) PWB_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  {
    // order after the work already queued on the default stream (X, bounds)
    cudaEvent_t ev;
    PWB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    PWB_CUDA(cudaEventRecord(ev, 0));
    PWB_CUDA(cudaStreamWaitEvent(s.st, ev, 0));
    cudaEventDestroy(ev);
  }
  const double e = (b - a) / 2.0, cc = (b + a) / 2.0;
  double sigma = e / (a0 - cc);
  const double sigma1 = sigma, gamma = 2.0 / sigma1;
  std::vector<double> coef(3 * std::max(m, 1), 0.0);
  coef[0] = sigma1 / e;
  coef[1] = -cc * sigma1 / e;
  for (int i = 2; i <= m; ++i) {
    const double sigma2 = 1.0 / (gamma - sigma);
    coef[3 * (i - 1) + 0] = 2 * sigma2 / e;
    coef[3 * (i - 1) + 1] = -2 * sigma2 * cc / e;
    coef[3 * (i - 1) + 2] = -sigma * sigma2;
    sigma = sigma2;
  }
  if ((rc = s.fcoef.alloc(coef.size() * 8))) return rc;
  PWB_CUDA(cudaMemcpyAsync(s.fcoef.p, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice, s.st));
  const double* cd = (const double*)s.fcoef.p;
  if (s.fexec && (s.f_nb != nb || s.f_m != m)) {
    cudaGraphExecDestroy(s.fexec);
    cudaGraphDestroy(s.fgraph);
    s.fexec = nullptr;
    s.fgraph = nullptr;
    s.f_calls = 0;
  }
  if (!s.use_graph || (!s.fexec && s.f_calls == 0)) {
    rc = cheby_filter_dev(s, nb, m, cd, s.X.p, s.Y.p, s.Z.p, s.HY.p, result, s.st);
    s.f_calls = 1;
    s.f_nb = nb;
    s.f_m = m;
  } else {
    if (!s.fexec) {
      PWB_CUDA(cudaStreamSynchronize(s.st));
      PWB_CUDA(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
      rc = cheby_filter_dev(s, nb, m, cd, s.X.p, s.Y.p, s.Z.p, s.HY.p, &s.f_res, s.st);
      cudaError_t e1 = cudaStreamEndCapture(s.st, &s.fgraph);
      if (rc) return rc;
      PWB_CUDA(e1);
      PWB_CUDA(cudaGraphInstantiate(&s.fexec, s.fgraph, 0));
    }
    PWB_CUDA(cudaGraphLaunch(s.fexec, s.st));
    *result = s.f_res;
  }
  PWB_CUDA(cudaStreamSynchronize(s.st));
  return rc;
}

static int chebfsi_step(Solver& s, Dense& d, int nb, int degree, double a, double b, double a0) {
  int rc;
  void* res = nullptr;
  if ((rc = cheby_filter_run(s, nb, degree, a, b, a0, &res))) return rc;
  // With the wavefunction cut-off filter, P H is P H P on the span of P and
  // zero on its complement; the shifted recurrence amplifies whatever part of
  // the block lies in the complement (rounding of the transforms) at the
  // eigenvalue 0, which sits inside the wanted part of the spectrum.  One P
  // pass over the filtered block keeps the iteration in the span of P.
  if (s.c->wfn_filter && (rc = wfn_filter_pass(s.c, res, (int)s.nt, nb, nullptr))) return rc;
  // res is one of X, Y, Z; orthonormalise it, then Rayleigh-Ritz into X / HX
  void* tmp = (res == s.Z.p) ? s.Y.p : s.Z.p;
  if ((rc = cholqr(s, d, res, nb, tmp))) return rc;
  if ((rc = hpsi(s.c, res, s.HY.p, nb, nullptr))) return rc;
  void* outX = (res == s.X.p) ? tmp : s.X.p;
  if ((rc = rayleigh_ritz(s, d, res, s.HY.p, outX, s.HX.p, nb))) return rc;
  if (outX != s.X.p) PWB_CUDA(cudaMemcpy(s.X.p, outX, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice));
  return PW_OK;
}

// Chebyshev coefficients of cheby_filter_run's recurrence from the previous
// step's Ritz values on the device: a = w[nb-1], a0 = w[0], b = *bup
__global__ void k_cheb_coef(const double* w, int nb, const double* bup, int m, double* coef) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double a = w[nb - 1], a0 = w[0], b = *bup;
  const double e = (b - a) / 2.0, cc = (b + a) / 2.0;
  double sigma = e / (a0 - cc);
  const double sigma1 = sigma, gamma = 2.0 / sigma1;
  coef[0] = sigma1 / e;
  coef[1] = -cc * sigma1 / e;
  coef[2] = 0.0;
  for (int i = 2; i <= m; ++i) {
    const double sigma2 = 1.0 / (gamma - sigma);
    coef[3 * (i - 1) + 0] = 2 * sigma2 / e;
    coef[3 * (i - 1) + 1] = -2 * sigma2 * cc / e;
    coef[3 * (i - 1) + 2] = -sigma * sigma2;
    sigma = sigma2;
  }
}

// the ChebFSI step with the bounds of the previous Rayleigh-Ritz (a =
// eig[nb-1], a0 = eig[0]) and the Lanczos upper bound b_up, all on s.st with
// no host round trip inside: with s.use_graph the first call runs directly,
// the second captures it as one CUDA graph, later calls replay it; the host
// then reads the Cholesky status and the new Ritz values once
static int chebfsi_step_dev(Solver& s, Dense& d, int nb, int m, cudaStream_t st) {
  int rc;
  k_cheb_coef<<<1, 32, 0, st>>>((const double*)s.wbuf.p, nb, (const double*)s.bup.p, m, (double*)s.fcoef.p);
  PWB_CUDA(cudaGetLastError());
  void* res = nullptr;
  if ((rc = cheby_filter_dev(s, nb, m, (const double*)s.fcoef.p, s.X.p, s.Y.p, s.Z.p, s.HY.p, &res, st))) return rc;
  if (s.c->wfn_filter && (rc = wfn_filter_pass(s.c, res, (int)s.nt, nb, st))) return rc;
  void* tmp = (res == s.Z.p) ? s.Y.p : s.Z.p;
  if ((rc = cholqr(s, d, res, nb, tmp, st, true))) return rc;
  if ((rc = pw_hpsi(s.c, res, (int)s.nt, s.HY.p, (int)s.nt, nb, 0, st))) return rc;
  void* outX = (res == s.X.p) ? tmp : s.X.p;
  if ((rc = rayleigh_ritz(s, d, res, s.HY.p, outX, s.HX.p, nb, st, true))) return rc;
  if (outX != s.X.p) PWB_CUDA(cudaMemcpyAsync(s.X.p, outX, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice, st));
  return PW_OK;
}

static int chebfsi_step_graph(Solver& s, Dense& d, int nb, int m, double b_up) {
  if (!s.use_graph || s.s_off || s.eig.size() < (size_t)nb || !s.wbuf.p)
    return chebfsi_step(s, d, nb, m, s.eig[nb - 1], b_up, s.eig[0]);
  int rc;
  if (!s.st) PWB_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  {
    cudaEvent_t ev;
    PWB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    PWB_CUDA(cudaEventRecord(ev, 0));
    PWB_CUDA(cudaStreamWaitEvent(s.st, ev, 0));
    cudaEventDestroy(ev);
  }
  if ((rc = s.fcoef.alloc((size_t)3 * std::max(m, 1) * 8)) || (rc = s.bup.alloc(8))) return rc;
  s.bup_host = b_up;
  PWB_CUDA(cudaMemcpyAsync(s.bup.p, &s.bup_host, 8, cudaMemcpyHostToDevice, s.st));
  if (s.sexec && (s.s_nb != nb || s.s_m != m)) {
    cudaGraphExecDestroy(s.sexec);
    cudaGraphDestroy(s.sgraph);
    s.sexec = nullptr;
    s.sgraph = nullptr;
    s.s_calls = 0;
  }
  if (!s.sexec && s.s_calls == 0) {
    if ((rc = chebfsi_step_dev(s, d, nb, m, s.st))) return rc;
    s.s_calls = 1;
    s.s_nb = nb;
    s.s_m = m;
  } else {
    if (!s.sexec) {
      PWB_CUDA(cudaStreamSynchronize(s.st));
      PWB_CUDA(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
      rc = chebfsi_step_dev(s, d, nb, m, s.st);
      cudaError_t e1 = cudaStreamEndCapture(s.st, &s.sgraph);
      cudaError_t e2 = (rc == PW_OK && e1 == cudaSuccess) ? cudaGraphInstantiate(&s.sexec, s.sgraph, 0) : e1;
      if (rc != PW_OK || e2 != cudaSuccess) {
        // a step that cannot be captured runs directly from now on
        cudaGetLastError();
        if (s.sgraph) cudaGraphDestroy(s.sgraph);
        s.sgraph = nullptr;
        s.sexec = nullptr;
        s.s_off = true;
        PWB_CUDA(cudaStreamSynchronize(s.st));
        return chebfsi_step(s, d, nb, m, s.eig[nb - 1], b_up, s.eig[0]);
      }
    }
    PWB_CUDA(cudaGraphLaunch(s.sexec, s.st));
  }
  int info = 0;
  s.eig.resize(nb);
  PWB_CUDA(cudaMemcpyAsync(&info, d.info.p, sizeof(int), cudaMemcpyDeviceToHost, s.st));
  PWB_CUDA(cudaMemcpyAsync(s.eig.data(), s.wbuf.p, (size_t)nb * 8, cudaMemcpyDeviceToHost, s.st));
  PWB_CUDA(cudaStreamSynchronize(s.st));
  PWB_CHECK(info == 0, PW_ENUMERIC, "Cholesky factorisation of the Gram matrix failed");
  return PW_OK;
}

// residual norms ||HX - X diag(l)|| / max(1, |l|) (lobpcg.cpp:697-709)
static int residuals(Solver& s, int nb) {
  int rc;
  if ((rc = alloc_block(s, s.Z, nb))) return rc;
  PWB_CUDA(cudaMemcpy(s.Z.p, s.HX.p, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice));
  std::vector<double> ml(nb);
  for (int i = 0; i < nb; ++i) ml[i] = -s.eig[i];
  DevBuf dl;
  if ((rc = dl.alloc(nb * 8 * 2))) return rc;
  PWB_CUDA(cudaMemcpy(dl.p, ml.data(), nb * 8, cudaMemcpyHostToDevice));
  // Z = HX - X diag(l): scale a copy of X then add
  if ((rc = alloc_block(s, s.Y, nb))) return rc;
  PWB_CUDA(cudaMemcpy(s.Y.p, s.X.p, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice));
  if ((rc = v_colscale(s, nb, s.Y.p, (double*)dl.p))) return rc;
  if ((rc = v_axpby(s, nb, 1.0, s.Y.p, 1.0, s.Z.p))) return rc;
  double* nr = (double*)dl.p + nb;
  if ((rc = v_colnorm2(s, nb, s.Z.p, nr))) return rc;
  std::vector<double> h(nb);
  PWB_CUDA(cudaMemcpy(h.data(), nr, nb * 8, cudaMemcpyDeviceToHost));
  s.res.resize(nb);
  for (int i = 0; i < nb; ++i) s.res[i] = std::sqrt(h[i]) / std::max(1.0, std::fabs(s.eig[i]));
  return PW_OK;
}

// LOBPCG restated from EigenSolver::LOBPCGSolveReal (real-space branch).
static int lobpcg(Solver& s, Dense& d, int width, int maxit, double tol, bool first_scf, int* iters) {
  int rc;
  const long nt = s.nt;
  const size_t esz = s.esz;
  const int lda = 3 * width;
  if ((rc = alloc_block(s, s.S, 3 * width)) || (rc = alloc_block(s, s.HS, 3 * width)) || (rc = alloc_block(s, s.Y, width)))
    return rc;
  void* X = s.ptr(s.S, 0);
  void* W = s.ptr(s.S, width);
  void* P = s.ptr(s.S, 2 * width);
  void* AX = s.ptr(s.HS, 0);
  void* AW = s.ptr(s.HS, width);
  void* AP = s.ptr(s.HS, 2 * width);
  PWB_CUDA(cudaMemcpy(X, s.X.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
  if (first_scf && (rc = cholqr(s, d, X, width, s.Y.p))) return rc;
  if ((rc = hpsi(s.c, X, AX, width, nullptr))) return rc;
  if ((rc = s.G1.alloc((size_t)lda * lda * 8)) || (rc = s.G2.alloc((size_t)lda * lda * 8))) return rc;
  DevBuf xtx, dvec, rvec;
  if ((rc = xtx.alloc((size_t)width * width * 8)) || (rc = dvec.alloc((size_t)3 * width * 8)) ||
      (rc = rvec.alloc((size_t)(width + 1) * 8)))
    return rc;
  std::vector<double> eigS(lda);
  double resMax = 0;
  int iter = 0;
  std::vector<double> resNorm(width);
  do {
    ++iter;
    const int numSet = (iter == 1) ? 2 : 3;
    // XTX = X^T AX;  R = AX - X XTX  (all on the device; only the largest
    // residual norm, the convergence test, comes back to the host)
    double* XTX = (double*)xtx.p;
    if ((rc = gram(s.c, X, (int)nt, width, AX, (int)nt, width, XTX, width, nullptr))) return rc;
    PWB_CUDA(cudaMemcpyAsync(s.Y.p, AX, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice, nullptr));
    if ((rc = dense_scale(width, width, -1.0, XTX, width, (double*)s.G2.p, width, nullptr))) return rc;
    RotBlock rb{X, nt, width, (double*)s.G2.p, width};
    if ((rc = rotate(s.c, (int)nt, width, &rb, 1, s.Y.p, nt, 1.0, nullptr, true))) return rc;
    double* nrm = (double*)dvec.p;
    double* rn = (double*)rvec.p;
    if ((rc = v_colnorm2(s, width, s.Y.p, nrm))) return rc;
    if ((rc = resnorms(width, nrm, XTX, width, rn, nullptr))) return rc;
    PWB_CUDA(cudaMemcpy(&resMax, rn + width, 8, cudaMemcpyDeviceToHost));
    // W = Teter * R, normalised
    if ((rc = pw_teter_precond(s.c, s.Y.p, (int)nt, W, (int)nt, width, 0, nullptr))) return rc;
    if ((rc = v_colnorm2(s, width, W, nrm)) || (rc = vec_rsqrt(width, nrm, nullptr)) ||
        (rc = v_colscale(s, width, W, nrm)))
      return rc;
    if (numSet == 3) {
      if ((rc = v_colnorm2(s, width, P, nrm)) || (rc = vec_rsqrt(width, nrm, nullptr)) ||
          (rc = v_colscale(s, width, P, nrm)) || (rc = v_colscale(s, width, AP, nrm)))
        return rc;
    }
    if ((rc = hpsi(s.c, W, AW, width, nullptr))) return rc;
    // AMat = S^T AS, BMat = S^T S over the active sets (upper blocks used)
    const int numCol = numSet * width;
    double* A = (double*)s.G1.p;
    double* B = (double*)s.G2.p;
    if ((rc = gram(s.c, s.S.p, (int)nt, numCol, s.HS.p, (int)nt, numCol, A, lda, nullptr))) return rc;
    if ((rc = gram(s.c, s.S.p, (int)nt, numCol, s.S.p, (int)nt, numCol, B, lda, nullptr))) return rc;
    int numKeep = 0;
    if ((rc = solve_gen_eig(d, lda, numCol, width, A, B, eigS.data(), &numKeep, nullptr))) return rc;
    // X_new = X Cx + W Cw (+ P Cp);  P_new = W Cw (+ P Cp); same for AX, AP
    const double* Cx = A;
    const double* Cw = A + width;
    const double* Cp = A + 2 * width;
    RotBlock pb[2] = {{W, nt, width, Cw, lda}, {P, nt, width, Cp, lda}};
    if ((rc = rotate(s.c, (int)nt, width, pb, numSet - 1, s.Y.p, nt, 0.0, nullptr))) return rc;
    RotBlock xb{X, nt, width, Cx, lda};
    if ((rc = rotate(s.c, (int)nt, width, &xb, 1, s.Z.p, nt, 0.0, nullptr))) return rc;
    // Z = X Cx ; X = Z + Y ; P = Y
    if ((rc = v_axpby(s, width, 1.0, s.Z.p, 0.0, X))) return rc;
    if ((rc = v_axpby(s, width, 1.0, s.Y.p, 1.0, X))) return rc;
    PWB_CUDA(cudaMemcpy(P, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
    RotBlock apb[2] = {{AW, nt, width, Cw, lda}, {AP, nt, width, Cp, lda}};
    if ((rc = rotate(s.c, (int)nt, width, apb, numSet - 1, s.Y.p, nt, 0.0, nullptr))) return rc;
    RotBlock axb{AX, nt, width, Cx, lda};
    if ((rc = rotate(s.c, (int)nt, width, &axb, 1, s.Z.p, nt, 0.0, nullptr))) return rc;
    if ((rc = v_axpby(s, width, 1.0, s.Z.p, 0.0, AX))) return rc;
    if ((rc = v_axpby(s, width, 1.0, s.Y.p, 1.0, AX))) return rc;
    PWB_CUDA(cudaMemcpy(AP, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
  } while (iter < maxit && resMax > tol);
  PWB_CUDA(cudaMemcpy(resNorm.data(), rvec.p, width * 8, cudaMemcpyDeviceToHost));
  // final Rayleigh-Ritz with X^T AX (lobpcg.cpp:991-1003)
  if ((rc = rayleigh_ritz(s, d, X, AX, s.X.p, s.HX.p, width))) return rc;
  s.res = resNorm;
  if (iters) *iters = iter;
  return PW_OK;
}

static int v_bdiag_dots_dev(Solver& s, int width, int sb, const void* U, const void* V, DevBuf& part, double* out) {
  return s.c->prec == PW_F64
             ? bdiag_dots_dev<double>((int)s.nt, width, sb, (const double*)U, (const double*)V, s.nt, part, out, nullptr)
             : bdiag_dots_dev<float>((int)s.nt, width, sb, (const float*)U, (const float*)V, s.nt, part, out, nullptr);
}
static int v_bdiag_rotate(Solver& s, int width, int sb, const void* X, const double* C, void* Y, double beta) {
  return s.c->prec == PW_F64
             ? bdiag_rotate<double>((int)s.nt, width, sb, (const double*)X, s.nt, C, (double*)Y, s.nt, beta, nullptr)
             : bdiag_rotate<float>((int)s.nt, width, sb, (const float*)X, s.nt, C, (float*)Y, s.nt, beta, nullptr);
}

// V -= X (X^T V), AV -= AX (X^T V)
static int project_out(Solver& s, int width, void* X, void* AX, void* V, void* AV, DevBuf& G) {
  int rc;
  if ((rc = G.alloc((size_t)width * width * 8))) return rc;
  double* g = (double*)G.p;
  if ((rc = gram(s.c, X, (int)s.nt, width, V, (int)s.nt, width, g, width, nullptr))) return rc;
  if ((rc = dense_scale(width, width, -1.0, g, width, g, width, nullptr))) return rc;
  RotBlock rb{X, s.nt, width, g, width};
  if ((rc = rotate(s.c, (int)s.nt, width, &rb, 1, V, s.nt, 1.0, nullptr, true))) return rc;
  RotBlock ra{AX, s.nt, width, g, width};
  return rotate(s.c, (int)s.nt, width, &ra, 1, AV, s.nt, 1.0, nullptr, true);
}

// V, AV /= ||V|| column-wise
static int normalize_pair(Solver& s, int width, void* V, void* AV, DevBuf& tmp) {
  int rc;
  if ((rc = tmp.alloc((size_t)width * 8))) return rc;
  double* d = (double*)tmp.p;
  // 1 / ||v|| on the device; a vanishing direction (an exactly converged
  // column) stays zero instead of 0/0
  if ((rc = v_colnorm2(s, width, V, d)) || (rc = vec_rsqrt(width, d, nullptr))) return rc;
  if ((rc = v_colscale(s, width, V, d))) return rc;
  return AV ? v_colscale(s, width, AV, d) : PW_OK;
}

// Cholesky-QR of X with AX transformed alongside: X <- X U^-1, AX <- AX U^-1
static int cholqr_pair(Solver& s, Dense& d, void* X, void* AX, int nb, void* tmp) {
  const cudaStream_t st = nullptr;
  int rc;
  if ((rc = s.G1.alloc((size_t)nb * nb * 8)) || (rc = s.G2.alloc((size_t)nb * nb * 8))) return rc;
  double* G = (double*)s.G1.p;
  if ((rc = gram(s.c, X, (int)s.nt, nb, X, (int)s.nt, nb, G, nb, st))) return rc;
  if ((rc = d.potrf_upper(nb, G, nb, st))) return rc;
  double* Ui = (double*)s.G2.p;
  if ((rc = dense_trtri_upper(nb, G, nb, Ui, nb, st))) return rc;
  RotBlock rb{X, s.nt, nb, Ui, nb};
  if ((rc = rotate(s.c, (int)s.nt, nb, &rb, 1, tmp, s.nt, 0.0, st))) return rc;
  PWB_CUDA(cudaMemcpy(X, tmp, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice));
  RotBlock ra{AX, s.nt, nb, Ui, nb};
  if ((rc = rotate(s.c, (int)s.nt, nb, &ra, 1, tmp, s.nt, 0.0, st))) return rc;
  PWB_CUDA(cudaMemcpy(AX, tmp, (size_t)nb * s.nt * s.esz, cudaMemcpyDeviceToDevice));
  return PW_OK;
}

// PPCG restated from EigenSolver::PPCGSolveReal, real-space branch
// (src/EigenSolver/ppcg.cpp:670-1243): residual R = AX - X (X^T AX), W = T R,
// W and P made orthogonal to X, per sub-block of sb columns a 2sb / 3sb
// generalized Rayleigh-Ritz (Sygvd) giving x <- x cx + p, p <- w cw + p cp,
// Cholesky-QR of X every iteration, final Rayleigh-Ritz.  No locking.
static int ppcg(Solver& s, Dense& d, int width, int sb, int maxit, double tol, bool first_scf, int* iters) {
  int rc;
  const long nt = s.nt;
  const size_t esz = s.esz;
  sb = std::max(1, std::min(sb, std::min(8, width)));
  const int nsb = (width + sb - 1) / sb;
  if ((rc = alloc_block(s, s.S, 3 * width)) || (rc = alloc_block(s, s.HS, 3 * width)) || (rc = alloc_block(s, s.Y, width)))
    return rc;
  void* X = s.ptr(s.S, 0);
  void* W = s.ptr(s.S, width);
  void* P = s.ptr(s.S, 2 * width);
  void* AX = s.ptr(s.HS, 0);
  void* AW = s.ptr(s.HS, width);
  void* AP = s.ptr(s.HS, 2 * width);
  PWB_CUDA(cudaMemcpy(X, s.X.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
  if (first_scf && (rc = cholqr(s, d, X, width, s.Y.p))) return rc;
  if ((rc = hpsi(s.c, X, AX, width, nullptr))) return rc;
  DevBuf G, G2, tmpv, part, Cd, Gs, rvec;
  if ((rc = Cd.alloc((size_t)3 * nsb * sb * sb * 8))) return rc;
  double* Cx = (double*)Cd.p;
  double* Cw = Cx + (size_t)nsb * sb * sb;
  double* Cp = Cw + (size_t)nsb * sb * sb;
  const size_t bs = (size_t)nsb * sb * sb;
  // the twelve sub-block Gram arrays, device-resident
  if ((rc = Gs.alloc(12 * bs * 8)) || (rc = rvec.alloc((size_t)(width + 1) * 8))) return rc;
  double* gp[12];
  for (int i = 0; i < 12; ++i) gp[i] = (double*)Gs.p + i * bs;
  double *xax = gp[0], *waw = gp[1], *xaw = gp[2], *xx = gp[3], *ww = gp[4], *xw = gp[5], *pap = gp[6],
         *xap = gp[7], *wap = gp[8], *pp = gp[9], *xp = gp[10], *wp = gp[11];
  std::vector<double> resNorm(width);
  double resMax = 0;
  int iter = 0;
  do {
    ++iter;
    const int numSet = (iter == 1) ? 2 : 3;
    // R = AX - X (X^T AX) into Y, on the device; only the largest residual
    // norm (the convergence test) comes back to the host
    if ((rc = G.alloc((size_t)width * width * 8)) || (rc = G2.alloc((size_t)width * width * 8))) return rc;
    double* g = (double*)G.p;
    if ((rc = gram(s.c, X, (int)nt, width, AX, (int)nt, width, g, width, nullptr))) return rc;
    if ((rc = dense_scale(width, width, -1.0, g, width, (double*)G2.p, width, nullptr))) return rc;
    PWB_CUDA(cudaMemcpyAsync(s.Y.p, AX, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice, nullptr));
    RotBlock rb{X, nt, width, (double*)G2.p, width};
    if ((rc = rotate(s.c, (int)nt, width, &rb, 1, s.Y.p, nt, 1.0, nullptr, true))) return rc;
    if ((rc = tmpv.alloc((size_t)width * 8))) return rc;
    if ((rc = v_colnorm2(s, width, s.Y.p, (double*)tmpv.p))) return rc;
    if ((rc = resnorms(width, (const double*)tmpv.p, g, width, (double*)rvec.p, nullptr))) return rc;
    PWB_CUDA(cudaMemcpy(&resMax, (double*)rvec.p + width, 8, cudaMemcpyDeviceToHost));
    // W = T R, AW = H W, orthogonal to X, normalised
    if ((rc = pw_teter_precond(s.c, s.Y.p, (int)nt, W, (int)nt, width, 0, nullptr))) return rc;
    if ((rc = hpsi(s.c, W, AW, width, nullptr))) return rc;
    if ((rc = project_out(s, width, X, AX, W, AW, G))) return rc;
    if ((rc = normalize_pair(s, width, W, AW, tmpv))) return rc;
    if (numSet == 3) {
      if ((rc = project_out(s, width, X, AX, P, AP, G))) return rc;
      if ((rc = normalize_pair(s, width, P, AP, tmpv))) return rc;
    }
    // sub-block Gram blocks (device)
    {
      SubTimer t_(1);
      if ((rc = v_bdiag_dots_dev(s, width, sb, X, AX, part, xax)) ||
          (rc = v_bdiag_dots_dev(s, width, sb, W, AW, part, waw)) ||
          (rc = v_bdiag_dots_dev(s, width, sb, X, AW, part, xaw)) ||
          (rc = v_bdiag_dots_dev(s, width, sb, X, X, part, xx)) ||
          (rc = v_bdiag_dots_dev(s, width, sb, W, W, part, ww)) ||
          (rc = v_bdiag_dots_dev(s, width, sb, X, W, part, xw)))
        return rc;
      if (numSet == 3 &&
          ((rc = v_bdiag_dots_dev(s, width, sb, P, AP, part, pap)) ||
           (rc = v_bdiag_dots_dev(s, width, sb, X, AP, part, xap)) ||
           (rc = v_bdiag_dots_dev(s, width, sb, W, AP, part, wap)) ||
           (rc = v_bdiag_dots_dev(s, width, sb, P, P, part, pp)) ||
           (rc = v_bdiag_dots_dev(s, width, sb, X, P, part, xp)) ||
           (rc = v_bdiag_dots_dev(s, width, sb, W, P, part, wp))))
        return rc;
    }
    // nsb small generalized eigenproblems (Sygvd), one warp each on the device
    {
      const double* grams[12] = {xax, waw, xaw, xx, ww, xw, pap, xap, wap, pp, xp, wp};
      if ((rc = ppcg_subblock_solve(width, sb, numSet, grams, Cx, Cw, Cp, nullptr))) return rc;
    }
    {
      SubTimer t_(3);
      // p = w cw (+ p cp); ap = aw cw (+ ap cp)
      if (numSet == 3) {
        if ((rc = v_bdiag_rotate(s, width, sb, P, Cp, s.Y.p, 0.0)) ||
            (rc = v_bdiag_rotate(s, width, sb, W, Cw, s.Y.p, 1.0)))
          return rc;
        PWB_CUDA(cudaMemcpy(P, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
        if ((rc = v_bdiag_rotate(s, width, sb, AP, Cp, s.Y.p, 0.0)) ||
            (rc = v_bdiag_rotate(s, width, sb, AW, Cw, s.Y.p, 1.0)))
          return rc;
        PWB_CUDA(cudaMemcpy(AP, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
      } else {
        if ((rc = v_bdiag_rotate(s, width, sb, W, Cw, P, 0.0)) || (rc = v_bdiag_rotate(s, width, sb, AW, Cw, AP, 0.0)))
          return rc;
      }
      // x = x cx + p; ax = ax cx + ap
      PWB_CUDA(cudaMemcpy(s.Y.p, P, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
      if ((rc = v_bdiag_rotate(s, width, sb, X, Cx, s.Y.p, 1.0))) return rc;
      PWB_CUDA(cudaMemcpy(X, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
      PWB_CUDA(cudaMemcpy(s.Y.p, AP, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
      if ((rc = v_bdiag_rotate(s, width, sb, AX, Cx, s.Y.p, 1.0))) return rc;
      PWB_CUDA(cudaMemcpy(AX, s.Y.p, (size_t)width * nt * esz, cudaMemcpyDeviceToDevice));
    }
    // Cholesky-QR of X, AX transformed alongside
    if ((rc = cholqr_pair(s, d, X, AX, width, s.Y.p))) return rc;
  } while (iter < maxit && resMax > tol);
  PWB_CUDA(cudaMemcpy(resNorm.data(), rvec.p, width * 8, cudaMemcpyDeviceToHost));
  // final Rayleigh-Ritz (ppcg.cpp:1112-1166)
  if ((rc = rayleigh_ritz(s, d, X, AX, s.X.p, s.HX.p, width))) return rc;
  if (iters) *iters = iter;
  return residuals(s, width);
}

// Block Davidson restated from EigenSolver::DavidsonSolveReal
// (src/EigenSolver/davidson.cpp:60-806): subspace S = (X | W_1 | ...) of at
// most maxdim * width columns; residuals of the unconverged Ritz pairs,
// Teter-preconditioned and normalised, are appended; generalized
// Rayleigh-Ritz on S (SolveGenEig); convergence on the change of each Ritz
// value; restart from the Ritz vectors when the subspace is full.
static int davidson(Solver& s, Dense& d, int width, int maxdim, int maxit, double tol, bool first_scf, int* iters) {
  int rc;
  const long nt = s.nt;
  const size_t esz = s.esz;
  maxdim = std::max(2, maxdim);
  const int w = width, lda = maxdim * w;
  if ((rc = alloc_block(s, s.S, lda)) || (rc = alloc_block(s, s.HS, lda)) || (rc = alloc_block(s, s.Y, w)))
    return rc;
  void* X = s.ptr(s.S, 0);
  void* AX = s.ptr(s.HS, 0);
  PWB_CUDA(cudaMemcpy(X, s.X.p, (size_t)w * nt * esz, cudaMemcpyDeviceToDevice));
  if (first_scf && (rc = cholqr(s, d, X, w, s.Y.p))) return rc;
  if ((rc = hpsi(s.c, X, AX, w, nullptr))) return rc;
  if ((rc = s.G1.alloc((size_t)lda * lda * 8)) || (rc = s.G2.alloc((size_t)lda * lda * 8))) return rc;
  double* A = (double*)s.G1.p;
  double* B = (double*)s.G2.p;
  std::vector<double> Asave((size_t)lda * lda, 0.0), Bsave((size_t)lda * lda, 0.0), hC((size_t)lda * lda);
  DevBuf G, Cd, tmpv;
  if ((rc = G.alloc((size_t)lda * w * 8)) || (rc = Cd.alloc((size_t)lda * w * 8)) || (rc = tmpv.alloc((size_t)w * 8)))
    return rc;
  auto fetch = [&](int nrow, int ncol, std::vector<double>& dst, int r0, int c0) -> int {
    std::vector<double> h((size_t)nrow * ncol);
    PWB_CUDA(cudaMemcpy(h.data(), G.p, h.size() * 8, cudaMemcpyDeviceToHost));
    for (int j = 0; j < ncol; ++j)
      for (int i = 0; i < nrow; ++i) dst[(r0 + i) + (size_t)(c0 + j) * lda] = h[i + (size_t)j * nrow];
    return PW_OK;
  };
  if ((rc = gram(s.c, X, (int)nt, w, AX, (int)nt, w, (double*)G.p, w, nullptr)) || (rc = fetch(w, w, Asave, 0, 0)))
    return rc;
  if ((rc = gram(s.c, X, (int)nt, w, X, (int)nt, w, (double*)G.p, w, nullptr)) || (rc = fetch(w, w, Bsave, 0, 0)))
    return rc;
  PWB_CUDA(cudaMemcpy(A, Asave.data(), Asave.size() * 8, cudaMemcpyHostToDevice));
  PWB_CUDA(cudaMemcpy(B, Bsave.data(), Bsave.size() * 8, cudaMemcpyHostToDevice));
  std::vector<double> eigS(w), eigT(lda), res(w, 0.0);
  int keep = 0;
  if ((rc = solve_gen_eig(d, lda, w, w, A, B, eigT.data(), &keep, nullptr))) return rc;
  std::copy(eigT.begin(), eigT.begin() + w, eigS.begin());
  std::vector<int> conv(w, 0);
  int nb = w, na = w, iter = 0;
  for (iter = 1; iter <= maxit; ++iter) {
    // compact the Ritz coefficients of the unconverged pairs
    PWB_CUDA(cudaMemcpy(hC.data(), A, hC.size() * 8, cudaMemcpyDeviceToHost));
    std::vector<double> cc((size_t)nb * na), lam(na);
    for (int i = 0, j = 0; i < w; ++i)
      if (!conv[i]) {
        for (int r = 0; r < nb; ++r) cc[r + (size_t)j * nb] = hC[r + (size_t)i * lda];
        lam[j] = -eigS[i];
        ++j;
      }
    PWB_CUDA(cudaMemcpy(Cd.p, cc.data(), cc.size() * 8, cudaMemcpyHostToDevice));
    // Wn = AS C - S C diag(lambda), appended at column nb
    void* Wn = s.ptr(s.S, nb);
    void* AWn = s.ptr(s.HS, nb);
    RotBlock r1{s.S.p, nt, nb, (const double*)Cd.p, nb};
    if ((rc = rotate(s.c, (int)nt, na, &r1, 1, s.Y.p, nt, 0.0, nullptr))) return rc;
    PWB_CUDA(cudaMemcpy(tmpv.p, lam.data(), na * 8, cudaMemcpyHostToDevice));
    if ((rc = v_colscale(s, na, s.Y.p, (const double*)tmpv.p))) return rc;
    RotBlock r2{s.HS.p, nt, nb, (const double*)Cd.p, nb};
    if ((rc = rotate(s.c, (int)nt, na, &r2, 1, Wn, nt, 0.0, nullptr))) return rc;
    if ((rc = v_axpby(s, na, 1.0, s.Y.p, 1.0, Wn))) return rc;
    // precondition, normalise, apply H
    if ((rc = pw_teter_precond(s.c, Wn, (int)nt, s.Y.p, (int)nt, na, 0, nullptr))) return rc;
    PWB_CUDA(cudaMemcpy(Wn, s.Y.p, (size_t)na * nt * esz, cudaMemcpyDeviceToDevice));
    if ((rc = normalize_pair(s, na, Wn, nullptr, tmpv))) return rc;
    if ((rc = hpsi(s.c, Wn, AWn, na, nullptr))) return rc;
    // extend the projected pencil by the new columns
    if ((rc = gram(s.c, s.S.p, (int)nt, nb + na, AWn, (int)nt, na, (double*)G.p, nb + na, nullptr)) ||
        (rc = fetch(nb + na, na, Asave, 0, nb)))
      return rc;
    if ((rc = gram(s.c, s.S.p, (int)nt, nb + na, Wn, (int)nt, na, (double*)G.p, nb + na, nullptr)) ||
        (rc = fetch(nb + na, na, Bsave, 0, nb)))
      return rc;
    nb += na;
    PWB_CUDA(cudaMemcpy(A, Asave.data(), Asave.size() * 8, cudaMemcpyHostToDevice));
    PWB_CUDA(cudaMemcpy(B, Bsave.data(), Bsave.size() * 8, cudaMemcpyHostToDevice));
    if ((rc = solve_gen_eig(d, lda, nb, w, A, B, eigT.data(), &keep, nullptr))) return rc;
    na = 0;
    for (int i = 0; i < w; ++i) {
      res[i] = std::fabs(eigS[i] - eigT[i]);
      conv[i] = res[i] < tol ? 1 : 0;
      if (!conv[i]) ++na;
    }
    std::copy(eigT.begin(), eigT.begin() + w, eigS.begin());
    const bool done = (na == 0) || iter == maxit;
    if (done || nb + na > lda) {
      // X = S C, AX = AS C (Ritz vectors)
      RotBlock rx{s.S.p, nt, nb, A, lda};
      if ((rc = rotate(s.c, (int)nt, w, &rx, 1, s.Y.p, nt, 0.0, nullptr))) return rc;
      PWB_CUDA(cudaMemcpy(X, s.Y.p, (size_t)w * nt * esz, cudaMemcpyDeviceToDevice));
      RotBlock ra{s.HS.p, nt, nb, A, lda};
      if ((rc = rotate(s.c, (int)nt, w, &ra, 1, s.Y.p, nt, 0.0, nullptr))) return rc;
      PWB_CUDA(cudaMemcpy(AX, s.Y.p, (size_t)w * nt * esz, cudaMemcpyDeviceToDevice));
      if (done) break;
      // restart from the Ritz vectors
      nb = w;
      std::fill(Asave.begin(), Asave.end(), 0.0);
      std::fill(Bsave.begin(), Bsave.end(), 0.0);
      std::vector<double> I((size_t)lda * lda, 0.0);
      for (int i = 0; i < w; ++i) {
        Asave[i + (size_t)i * lda] = eigS[i];
        Bsave[i + (size_t)i * lda] = 1.0;
        I[i + (size_t)i * lda] = 1.0;
      }
      PWB_CUDA(cudaMemcpy(A, I.data(), I.size() * 8, cudaMemcpyHostToDevice));
    }
  }
  PWB_CUDA(cudaMemcpy(s.X.p, X, (size_t)w * nt * esz, cudaMemcpyDeviceToDevice));
  PWB_CUDA(cudaMemcpy(s.HX.p, AX, (size_t)w * nt * esz, cudaMemcpyDeviceToDevice));
  s.eig = eigS;
  s.res = res;
  if (iters) *iters = std::min(iter, maxit);
  return PW_OK;
}

}  // namespace pwb

using namespace pwb;

namespace {

struct ScfState {
  pw_ctx* c64 = nullptr;
  pw_ctx* c32 = nullptr;
  DevBuf rho, rho_out, rps, vtot, vtot_new, vxc, eps, vh, kern, work, tw, dots, wocc;
  DevBuf work2, grad;              // PBE: second complex field, three real gradient fields
  // density-sphere weights pi vol / gkk (G != 0, gkk < 4 Ecut) and mask (RhoDdot,
  // CalculateError, BroydenMix); density change; Broyden spectra and history
  DevBuf bw, bmask, dr, bA, bB, bdf, bdv, bcdf, bdots;
  DevBuf dvh, dfh, dif_v, dif_f;   // Anderson history [mixdim][nf] and differences
  int nhist = 0, hpos = 0;
};

// pw_scf_run's device workspace, eigensolver blocks, dense-solver handle and
// the grid tables of the last cut-off, kept in the context between runs (the
// buffers are reused when large enough; the tables depend on the cell, the
// fine grid and Ecut only)
struct ScfCache {
  ScfState S;
  Solver sv;
  Dense dn;
  double ecut = -1.0;   // cut-off of the tables in S (Hartree kernel, density-sphere weights)
  ~ScfCache() { dn.release(); }
};
void* scf_cache_new() { return new ScfCache(); }
void scf_cache_free(void* p) { delete static_cast<ScfCache*>(p); }
ScfState& cache_state(ScfCache& c) { return c.S; }
Solver& cache_solver(ScfCache& c) { return c.sv; }
Dense& cache_dense(ScfCache& c) { return c.dn; }
double& cache_ecut(ScfCache& c) { return c.ecut; }

struct PhaseTimer {
  bool on;
  std::chrono::steady_clock::time_point t0;
  double* acc;
  PhaseTimer(bool on_, double* acc_) : on(on_), acc(acc_) {
    if (on) { cudaDeviceSynchronize(); t0 = std::chrono::steady_clock::now(); }
  }
  ~PhaseTimer() {
    if (on) {
      cudaDeviceSynchronize();
      *acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
  }
};

int dots(ScfState& S, long n, std::initializer_list<std::pair<const double*, const double*>> pr, double* out) {
  DotSet ds{};
  ds.k = 0;
  for (auto& p : pr) {
    ds.a[ds.k] = p.first;
    ds.b[ds.k] = p.second;
    ds.k++;
  }
  PWB_CUDA(cudaMemset(S.dots.p, 0, 64));
  k_dots<<<nblk(n), 256>>>(n, ds, (double*)S.dots.p);
  PWB_CUDA(cudaMemcpy(out, S.dots.p, ds.k * 8, cudaMemcpyDeviceToHost));
  return PW_OK;
}

int set_vtot_dev(pw_ctx* c, const double* vtot_dev) {
  int rc = c->vtot.alloc(c->ntotf * c->esz);
  if (rc) return rc;
  if (c->prec == PW_F64) PWB_CUDA(cudaMemcpy(c->vtot.p, vtot_dev, c->ntotf * 8, cudaMemcpyDeviceToDevice));
  else if ((rc = copy_d2f(c->ntotf, vtot_dev, (float*)c->vtot.p, nullptr))) return rc;
  if ((rc = refresh_vperm(c))) return rc;
  c->have_vtot = true;
  return PW_OK;
}

// occupation rate and the -T S term of one state (wgauss / getEntropy,
// src/utility.cpp:4404-4444): gb = 0 Fermi-Dirac ("FD"), 1 Gaussian ("GB")
double wgauss(double ev, double ef, double tbeta, int gb) {
  const double x = tbeta * (ef - ev);
  return gb ? 0.5 * std::erfc(-x) : 1.0 / (1.0 + std::exp(-x));
}
double smear_entropy(double ev, double ef, double tbeta, int gb) {
  const double x = tbeta * (ef - ev);
  if (gb) return -0.5 / tbeta * std::exp(-std::min(200.0, x * x)) / std::sqrt(M_PI);
  if (std::fabs(x) > 36.0) return 0.0;
  const double occ = 1.0 / (1.0 + std::exp(-x));
  return (occ * std::log(occ) + (1.0 - occ) * std::log(1.0 - occ)) / tbeta;
}

void occupations(const std::vector<double>& eig, int nocc, double tbeta, int gb, std::vector<double>& occ,
                 double& ef) {
  std::vector<double> ev(eig);
  std::sort(ev.begin(), ev.end());
  const int npsi = (int)ev.size();
  occ.assign(npsi, 1.0);
  if (npsi == nocc) { ef = ev[npsi - 1]; return; }
  double lb = ev[0], ub = ev[npsi - 1];
  ef = 0.5 * (lb + ub);
  auto sum = [&](double f) { double s = 0; for (double e : ev) s += wgauss(e, f, tbeta, gb); return s; };
  double os = sum(ef);
  int it = 1;
  while (std::fabs(os - nocc) > 1e-16 && it < 200) {
    if (os < nocc) lb = ef; else ub = ef;
    ef = 0.5 * (lb + ub);
    os = sum(ef);
    ++it;
  }
  for (int j = 0; j < npsi; ++j) occ[j] = wgauss(eig[j], ef, tbeta, gb);
}

}  // namespace

extern "C" {

int pw_scf_run(pw_ctx* ctx, const pw_scf_params* p, pw_scf_result* r, double* eig_out, double* rho_out) {
  PWB_CHECK(ctx && p && r, PW_EINVAL, "null argument");
  PWB_CHECK(ctx->prec == PW_F64, PW_EINVAL, "pw_scf_run takes the FP64 context (mixed mode builds an FP32 twin)");
  PWB_CHECK(!ctx->atom_z.empty(), PW_ENOTREADY, "atoms not set (pw_set_atoms)");
  PWB_CHECK(p->nocc > 0 && p->nextra >= 0 && p->ecut > 0, PW_EINVAL, "bad SCF parameters");
  PWB_CHECK(p->solver >= PW_SOLVER_LOBPCG && p->solver <= PW_SOLVER_DAVIDSON, PW_EINVAL, "unknown eigensolver");
  PWB_CHECK(p->smearing == 0 || p->smearing == 1, PW_EINVAL, "unknown smearing scheme");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const auto t_start = std::chrono::steady_clock::now();
  if (!ctx->scf_cache) {
    ctx->scf_cache = scf_cache_new();
    ctx->scf_cache_free = scf_cache_free;
  }
  ScfCache& cache = *(ScfCache*)ctx->scf_cache;
  ScfState& S = cache_state(cache);
  S.c64 = ctx;
  S.c32 = nullptr;
  S.nhist = 0;
  S.hpos = 0;
  const long nf = ctx->ntotf, nt = ctx->ntot;
  const int nb = p->nocc + p->nextra;
  const int natom = (int)ctx->atom_z.size();
  int rc;
  if (p->mixed) {
    if (!ctx->twin && (rc = pw_ctx_build_twin(ctx))) return rc;
    S.c32 = ctx->twin;
    if ((rc = pw_set_band_batch(S.c32, nb))) return rc;
  }
  // CheFSI runs H*psi with the wavefunction cut-off filter at Ecut unless the
  // caller turns it off (KohnSham::Setup, hamiltonian.cpp:316-321); the
  // contexts' own filter settings are restored on return
  struct FilterGuard {
    pw_ctx* c[2];
    bool on[2];
    double ecut[2];
    ~FilterGuard() {
      for (int i = 0; i < 2; ++i) {
        if (!c[i]) continue;
        if (on[i]) pw_set_wfn_filter(c[i], 1, ecut[i]);
        else c[i]->wfn_filter = false;
      }
    }
  } fguard{{ctx, S.c32}, {ctx->wfn_filter, S.c32 ? S.c32->wfn_filter : false},
           {ctx->wfn_ecut, S.c32 ? S.c32->wfn_ecut : 0.0}};
  const bool use_filter = p->solver == PW_SOLVER_CHEBFSI && !p->no_wfn_filter && !ctx->gs;
  for (pw_ctx* c : {ctx, S.c32}) {
    if (!c) continue;
    if (use_filter) {
      if ((rc = pw_set_wfn_filter(c, 1, p->ecut))) return rc;
    } else {
      c->wfn_filter = false;
    }
  }
  const bool prof = p->verbose == 2;
  g_sub_on = prof;
  for (double& x : g_sub) x = 0;
  double tph[6] = {0, 0, 0, 0, 0, 0};   // eigensolver, density, potentials, set-up, mixing, refine switch
  auto t_setup0 = std::chrono::steady_clock::now();
  if ((rc = pw_set_band_batch(ctx, nb))) return rc;
  // device arrays
  for (DevBuf* b : {&S.rho, &S.rho_out, &S.rps, &S.vtot, &S.vtot_new, &S.vxc, &S.eps, &S.vh, &S.kern})
    if ((rc = b->alloc(nf * 8))) return rc;
  if ((rc = S.work.alloc(nf * 16)) || (rc = S.dots.alloc(64)) || (rc = S.wocc.alloc((nb + 2) * 8))) return rc;
  const int mixdim = std::max(1, p->mix_dim);
  if ((rc = S.dvh.alloc((size_t)mixdim * nf * 8)) || (rc = S.dfh.alloc((size_t)mixdim * nf * 8)) ||
      (rc = S.dif_v.alloc((size_t)mixdim * nf * 8)) || (rc = S.dif_f.alloc((size_t)mixdim * nf * 8)))
    return rc;
  PWB_CUDA(cudaMemcpy(S.rps.p, ctx->h_rhops.data(), nf * 8, cudaMemcpyHostToDevice));
  if (cache_ecut(cache) != p->ecut || !S.kern.p || !S.bw.p) {
    // Hartree kernel 2 pi / gkk / N on the fine grid (fourier.cpp:323-344 gkkFine)
    std::vector<double> k(nf);
    const int N0 = ctx->nf[0], N1 = ctx->nf[1], N2 = ctx->nf[2];
    for (int z = 0; z < N2; ++z)
      for (int y = 0; y < N1; ++y)
        for (int x = 0; x < N0; ++x) {
          const double m0 = x <= N0 / 2 ? x : x - N0, m1 = y <= N1 / 2 ? y : y - N1, m2 = z <= N2 / 2 ? z : z - N2;
          const double g0 = 2 * M_PI / ctx->L[0] * m0, g1 = 2 * M_PI / ctx->L[1] * m1, g2 = 2 * M_PI / ctx->L[2] * m2;
          const double gkk = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
          k[x + (size_t)N0 * (y + (size_t)N1 * z)] =
              (gkk <= 1e-16 || gkk > 4.0 * p->ecut) ? 0.0 : 2.0 * M_PI / gkk / (double)nf;
        }
    PWB_CUDA(cudaMemcpy(S.kern.p, k.data(), nf * 8, cudaMemcpyHostToDevice));
    // density-sphere weights and mask (idxFineCutDensity, RhoDdot: scf.cpp:2263-2296)
    std::vector<double> bw(nf), bm(nf);
    for (int z = 0; z < N2; ++z)
      for (int y = 0; y < N1; ++y)
        for (int x = 0; x < N0; ++x) {
          const double m0 = x <= N0 / 2 ? x : x - N0, m1 = y <= N1 / 2 ? y : y - N1, m2 = z <= N2 / 2 ? z : z - N2;
          const double g0 = 2 * M_PI / ctx->L[0] * m0, g1 = 2 * M_PI / ctx->L[1] * m1, g2 = 2 * M_PI / ctx->L[2] * m2;
          const double gkk = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
          const size_t i = x + (size_t)N0 * (y + (size_t)N1 * z);
          bm[i] = gkk < 4.0 * p->ecut ? 1.0 : 0.0;
          bw[i] = (gkk != 0.0 && gkk < 4.0 * p->ecut) ? M_PI * ctx->vol / gkk : 0.0;
        }
    if ((rc = S.bw.alloc(nf * 8)) || (rc = S.bmask.alloc(nf * 8)) || (rc = S.dr.alloc(nf * 8)) ||
        (rc = S.bdots.alloc((size_t)(std::max(1, p->mix_dim) + 1) * (std::max(1, p->mix_dim) + 1) * 8)))
      return rc;
    PWB_CUDA(cudaMemcpy(S.bw.p, bw.data(), nf * 8, cudaMemcpyHostToDevice));
    PWB_CUDA(cudaMemcpy(S.bmask.p, bm.data(), nf * 8, cudaMemcpyHostToDevice));
    std::vector<double> t(2 * N0);
    for (int m = 0; m < N0; ++m) {
      t[2 * m] = std::cos(2 * M_PI * m / N0);
      t[2 * m + 1] = -std::sin(2 * M_PI * m / N0);
    }
    if ((rc = S.tw.alloc(N0 * 16))) return rc;
    PWB_CUDA(cudaMemcpy(S.tw.p, t.data(), N0 * 16, cudaMemcpyHostToDevice));
    cache_ecut(cache) = p->ecut;
  } else if ((rc = S.dr.alloc(nf * 8)) ||
             (rc = S.bdots.alloc((size_t)(std::max(1, p->mix_dim) + 1) * (std::max(1, p->mix_dim) + 1) * 8))) {
    return rc;
  }
  const double w = ctx->vol / (double)nf;
  double eself = 0;
  for (int z : ctx->atom_z) {
    double es;
    pw_hgh_species(z, nullptr, &es, nullptr, nullptr, nullptr);
    eself += es;
  }
  // initial density from the pseudocharge (scf.cpp:232-255)
  double* rho = (double*)S.rho.p;
  double* rps = (double*)S.rps.p;
  if (!ctx->init_rho.empty()) {
    // restart density (isRestartDensity, scf.cpp:164-178), used as given
    PWB_CUDA(cudaMemcpy(rho, ctx->init_rho.data(), nf * 8, cudaMemcpyHostToDevice));
  } else {
    k_init_rho<<<nblk(nf), 256>>>(nf, rps, rho);
    double sums[2];
    if ((rc = dots(S, nf, {{rho, nullptr}, {rps, nullptr}}, sums))) return rc;
    k_lincomb<<<nblk(nf), 256>>>(nf, sums[1] / sums[0], rho, 0.0, nullptr, rho);
  }
  const bool broyden = p->mix_type == PW_MIX_BROYDEN;
  PWB_CHECK(p->mix_type == PW_MIX_ANDERSON || broyden, PW_EINVAL, "unknown mixing scheme");
  PWB_CHECK(!broyden || (ctx->nf[0] == ctx->nf[1] && ctx->nf[1] == ctx->nf[2]), PW_EUNSUPPORTED,
            "Broyden mixing needs a cubic fine grid");
  if (broyden && ((rc = S.bA.alloc(nf * 16)) || (rc = S.bB.alloc(nf * 16)) ||
                  (rc = S.bdf.alloc((size_t)mixdim * nf * 16)) || (rc = S.bdv.alloc((size_t)mixdim * nf * 16)) ||
                  (rc = S.bcdf.alloc((size_t)2 * nf * 16))))
    return rc;
  // HSE06: the reference's nested hybrid scheme runs a PBE SCF first
  // (Setup_XC("XC_GGA_XC_PBE"), scf.cpp:409-425) and switches to the
  // semilocal HSE06 for the phi iterations (scf.cpp:628-640)
  const bool hse = p->xc == PW_XC_HSE06;
  const bool pbe = p->xc == PW_XC_PBE || hse;
  PWB_CHECK(p->xc == PW_XC_TETER93 || pbe, PW_EINVAL, "unknown exchange-correlation functional");
  if (pbe && ((rc = S.work2.alloc(nf * 16)) || (rc = S.grad.alloc(3 * nf * 8)))) return rc;
  // H*psi of a non-hybrid SCF carries no exchange term, whatever mode the
  // context was left in (restored on return); the hybrid SCF starts without it
  struct ExxModeGuard {
    pw_ctx* c;
    int mode;
    ~ExxModeGuard() { c->exx_mode = mode; }
  } exx_guard{ctx, ctx->exx_mode};
  ctx->exx_mode = PW_EXX_OFF;
  double hse_frac = 0.0;
  auto potentials = [&](const double* rh, double* exc_out) -> int {
    int q = PW_OK;
    if (pbe)
      q = xc_pbe(ctx, rh, p->ecut, (double*)S.eps.p, (double*)S.vxc.p, (double2*)S.work.p, (double2*)S.work2.p,
                 (double*)S.grad.p, (const double2*)S.tw.p, nullptr, hse_frac);
    else
      k_xc_teter93<<<nblk(nf), 256>>>(nf, rh, (double*)S.eps.p, (double*)S.vxc.p);
    if (q) return q;
    q = hartree(ctx, (double2*)S.work.p, rh, rps, (const double*)S.kern.p, (double*)S.vh.p, (const double2*)S.tw.p,
                    nullptr);
    if (q) return q;
    if (!exc_out) return PW_OK;   // the caller reduces eps rho with its own sums
    double e;
    if ((q = dots(S, nf, {{(const double*)S.eps.p, rh}}, &e))) return q;
    *exc_out = e * w;
    return PW_OK;
  };
  double exc = 0;
  if ((rc = potentials(rho, &exc))) return rc;
  k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, (double*)S.vh.p, 1.0, (double*)S.vxc.p, (double*)S.vtot.p);
  // eigensolver state: start in the FP32 twin when mixed
  Dense& dn = cache_dense(cache);
  if ((rc = dn.init((cublasHandle_t)ctx->blas))) return rc;
  Solver& sv = cache_solver(cache);
  sv.eig.clear();
  sv.res.clear();
  sv.use_graph = p->graphs != 0 && !prof;   // the sub-phase timers synchronise, which a capture forbids
  auto bind = [&](pw_ctx* c) -> int {
    // captured graphs refer to the previous context's buffers
    sv.drop_graphs();
    sv.c = c;
    sv.nt = nt;
    sv.esz = c->esz;
    sv.nb = nb;
    int q;
    for (DevBuf* b : {&sv.X, &sv.HX, &sv.Y, &sv.HY, &sv.Z})
      if ((q = alloc_block(sv, *b, nb))) return q;
    return PW_OK;
  };
  pw_ctx* cur = p->mixed ? S.c32 : ctx;
  if ((rc = bind(cur))) return rc;
  {
    // random start, Gaussian (seeded Philox on the device), orthonormalised by
    // Cholesky-QR; or the bands of pw_scf_set_initial (isRestartWfn, scf.cpp:296-330)
    const long ntot_b = (long)nb * nt;
    if (ctx->init_nband == nb && (long)ctx->init_psi.size() == ntot_b) {
      if (cur->prec == PW_F64) {
        PWB_CUDA(cudaMemcpy(sv.X.p, ctx->init_psi.data(), ntot_b * 8, cudaMemcpyHostToDevice));
      } else {
        std::vector<float> f(ctx->init_psi.begin(), ctx->init_psi.end());
        PWB_CUDA(cudaMemcpy(sv.X.p, f.data(), ntot_b * 4, cudaMemcpyHostToDevice));
      }
    } else {
      PWB_CHECK(ctx->init_nband == 0, PW_EINVAL, "initial bands: count does not match nocc + nextra");
      if (cur->prec == PW_F64) k_gaussian<double><<<nblk(ntot_b / 4 + 1), 256>>>(ntot_b, p->seed, (double*)sv.X.p);
      else k_gaussian<float><<<nblk(ntot_b / 4 + 1), 256>>>(ntot_b, p->seed, (float*)sv.X.p);
    }
    ctx->init_rho.clear();
    ctx->init_psi.clear();
    ctx->init_nband = 0;
    PWB_CUDA(cudaGetLastError());
    if (cur->gs)   // sphere-cut bands: Im c_0 = 0
      PWB_CUDA(cudaMemset2D((char*)sv.X.p + cur->esz, nt * cur->esz, 0, cur->esz, nb));
    // filtered CheFSI: the start block lies in the span of P (the first
    // MultSpinor call filters psi in place, hamiltonian.cpp:3090-3116)
    if (use_filter && (rc = wfn_filter_pass(cur, sv.X.p, (int)nt, nb, nullptr))) return rc;
    if ((rc = cholqr(sv, dn, sv.X.p, nb, sv.Y.p))) return rc;
  }
  if (prof) {
    cudaDeviceSynchronize();
    tph[3] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup0).count();
  }
  const double tbeta = 315774.67 / p->temperature;
  double b_up = 0, lmin = 0;
  bool have_bounds = false, refined = !p->mixed;
  double best_dif = 1e300;
  int stall = 0;
  std::vector<double> occ, eig;
  double ef = 0, etot = 0, efree = 0, eharris = 0, ehart = 0;
  int it = 0, total_it = 0;
  bool conv = false;
  r->hpsi_bands = 0;
  // switch the eigensolver from the FP32 twin to FP64 (iterative refinement)
  // verbose == 3: the wall time of the steps of an iteration (synchronising;
  // graphs stay on)
  auto mark = [&](const char* what) {
    if (p->verbose != 3) return;
    cudaDeviceSynchronize();
    fprintf(stderr, "  %-10s t %.4f s\n", what,
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count());
  };
  auto refine_now = [&]() -> int {
    PhaseTimer pt_(prof, &tph[5]);
    DevBuf& x32 = sv.x32;      // kept in the solver: no allocation per run
    int q;
    mark("refine");
    if ((q = x32.alloc((size_t)nb * nt * 4))) return q;
    PWB_CUDA(cudaMemcpy(x32.p, sv.X.p, (size_t)nb * nt * 4, cudaMemcpyDeviceToDevice));
    std::vector<double> keep_eig = sv.eig;
    if ((q = bind(ctx))) return q;
    mark("bind");
    if ((q = copy_f2d_2d((int)nt, nb, (const float*)x32.p, nt, (double*)sv.X.p, nt, nullptr))) return q;
    // the FP32 bands carry rounding outside the span of P: filter them again in FP64
    if (use_filter && (q = wfn_filter_pass(ctx, sv.X.p, (int)nt, nb, nullptr))) return q;
    mark("filter");
    if ((q = cholqr(sv, dn, sv.X.p, nb, sv.Y.p))) return q;
    mark("cholqr");
    sv.eig = keep_eig;
    refined = true;
    r->refine_iter = total_it;
    return PW_OK;
  };
  bool hybrid_phase = false;   // inner loop of a phi iteration
  // one SCF loop (SCF::Iterate's iteration, scf.cpp:430-620); the mixing
  // history restarts with it, as the reference's loop index does
  auto scf_loop = [&]() -> int {
  conv = false;
  S.nhist = 0;
  S.hpos = 0;
  for (it = 1; it <= p->max_iter; ++it) {
    ++total_it;
    mark("iteration");
    if ((rc = set_vtot_dev(sv.c, (const double*)S.vtot.p))) return rc;
    mark("vtot");
    {
    PhaseTimer pt_(prof, &tph[0]);
    if (p->solver == PW_SOLVER_CHEBFSI) {
      if (!have_bounds) {
        double lo;
        if ((rc = lanczos_upper(sv, 16, &b_up, &lo))) return rc;
        r->hpsi_bands += 16;
        lmin = lo;
        have_bounds = true;
        // first cycle: cutoff from the free-electron counting estimate
        const double frac = std::pow((double)nb / (double)nt, 2.0 / 3.0);
        double a = lo + 2.0 * frac * (b_up - lo);
        const int ncyc = std::max(1, p->cheby_first_cycles);
        for (int cyc = 0; cyc < ncyc; ++cyc) {
          if ((rc = chebfsi_step(sv, dn, nb, p->cheby_degree, a, b_up, lmin))) return rc;
          r->hpsi_bands += (long)nb * (p->cheby_degree + 1);
          a = sv.eig[nb - 1];
          lmin = sv.eig[0];
        }
      } else {
        if ((rc = chebfsi_step_graph(sv, dn, nb, p->cheby_degree, b_up))) return rc;
        r->hpsi_bands += (long)nb * (p->cheby_degree + 1);
      }
    } else if (p->solver == PW_SOLVER_PPCG) {
      int li = 0;
      if ((rc = ppcg(sv, dn, nb, p->ppcg_sbsize > 0 ? p->ppcg_sbsize : 1, p->eig_max_iter, p->eig_tol, it == 1, &li)))
        return rc;
      r->hpsi_bands += (long)nb * (li + 1);
    } else if (p->solver == PW_SOLVER_DAVIDSON) {
      int li = 0;
      if ((rc = davidson(sv, dn, nb, p->davidson_maxdim >= 2 ? p->davidson_maxdim : 2, p->eig_max_iter, p->eig_tol,
                         it == 1, &li)))
        return rc;
      r->hpsi_bands += (long)nb * (li + 1);
    } else {
      int li = 0;
      const double tolnow = p->eig_tol;
      if ((rc = lobpcg(sv, dn, nb, p->eig_max_iter, tolnow, it == 1, &li))) return rc;
      r->hpsi_bands += (long)nb * (2 * li + 1);
    }
    }
    eig = sv.eig;
    occupations(eig, p->nocc, tbeta, p->smearing, occ, ef);
    double ekin = 0, ent = 0;
    for (int i = 0; i < nb; ++i) {
      ekin += 2.0 * eig[i] * occ[i];
      ent += 2.0 * smear_entropy(eig[i], ef, tbeta, p->smearing);
    }
    // new density, and with its norm (one reduction) the Harris energy of the
    // input density and potentials (scf.cpp:2025-2060)
    double* ro = (double*)S.rho_out.p;
    mark("eigensolve");
    {
      PhaseTimer pt_(prof, &tph[1]);
      std::vector<double> wv(nb + 2, 0.0);
      for (int i = 0; i < nb; ++i) wv[i] = 2.0 * occ[i];
      PWB_CUDA(cudaMemcpy(S.wocc.p, wv.data(), wv.size() * 8, cudaMemcpyHostToDevice));
      PWB_CUDA(cudaMemset(ro, 0, nf * 8));
      const int cap = sv.c->pair_cap;
      for (int b0 = 0; b0 < nb; b0 += 2 * cap) {
        const int npair = std::min(cap, (nb - b0 + 1) / 2);
        if ((rc = run_density(sv.c, sv.X.p, (int)nt, nb, b0, npair, (const double*)S.wocc.p, ro, nullptr))) return rc;
      }
      double hd[4];
      if ((rc = dots(S, nf, {{(const double*)S.vh.p, rho}, {(const double*)S.vh.p, rps},
                             {(const double*)S.vxc.p, rho}, {ro, nullptr}}, hd)))
        return rc;
      const double ehart_h = 0.5 * (hd[0] + hd[1]) * w, evxc = hd[2] * w;
      eharris = ekin + (exc - evxc) - ehart_h - eself + ent;
      k_lincomb<<<nblk(nf), 256>>>(nf, (2.0 * p->nocc * (double)nf) / (ctx->vol * hd[3]), ro, 0.0, nullptr, ro);
    }
    mark("density");
    {
      PhaseTimer pt_(prof, &tph[2]);
      if ((rc = potentials(ro, nullptr))) return rc;
    }
    k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, (double*)S.vh.p, 1.0, (double*)S.vxc.p, (double*)S.vtot_new.p);
    // SCF::CalculateError of the change of the output density (scf.cpp:1492-1496,
    // 2368-2396); of the potential change vtotNew - vtot in the phi
    // iterations' inner loop (scf.cpp:728-739)
    double snorm = 0.0;
    {
      double* drv = (double*)S.dr.p;
      if (hybrid_phase)
        k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, (const double*)S.vtot_new.p, -1.0, (const double*)S.vtot.p, drv);
      else
        k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, ro, -1.0, rho, drv);
      if ((rc = fft3_real(ctx->nf[0], false, (double2*)S.work.p, drv, nullptr, 1.0, (const double2*)S.tw.p,
                          nullptr)))
        return rc;
      PWB_CUDA(cudaMemset(S.bdots.p, 0, 8));
      k_wdot<<<nblk(nf), 256>>>(nf, (const double*)S.bw.p, (const double2*)S.work.p, (const double2*)S.work.p,
                                (double*)S.bdots.p);
    }
    // KS energy terms (scf.cpp:1834-1984) in one reduction; it also waits for the scfNorm sum
    double ed[4];
    if ((rc = dots(S, nf, {{(const double*)S.eps.p, ro}, {(const double*)S.vtot.p, ro}, {(const double*)S.vh.p, ro},
                           {(const double*)S.vh.p, rps}}, ed)))
      return rc;
    exc = ed[0] * w;
    ehart = 0.5 * (ed[2] - ed[3]) * w;
    etot = ekin + (-ed[1] * w) + exc + ehart - eself;
    efree = etot + ent;
    const double dif = std::fabs(efree - eharris) / natom;
    PWB_CUDA(cudaMemcpy(&snorm, S.bdots.p, 8, cudaMemcpyDeviceToHost));
    snorm /= (double)nf * (double)nf;
    r->scf_norm = snorm;
    if (p->verbose)
      fprintf(stderr, "SCF %3d %s Etot %.10f Efree %.10f Eharris %.10f dif %.3e scfnorm %.3e t %.4f s\n", it,
              sv.c->prec == PW_F32 ? "f32" : "f64", etot, efree, eharris, dif, snorm,
              std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count());
    PWB_CUDA(cudaMemcpy(rho, ro, nf * 8, cudaMemcpyDeviceToDevice));
    if (refined && (p->tol_rho > 0 ? snorm < p->tol_rho : dif < p->tol_efree)) { conv = true; break; }
    // switch the eigensolver to FP64 for the final iterations (iterative
    // refinement): below the threshold, or when the FP32 iteration has
    // stagnated (no 10% gain on its best |E_free - E_Harris| for 4 steps)
    // within a factor 100 of it -- the FP32 fixed point is biased at the
    // 1e-6 Ha/atom level and cannot reach the tolerance by itself
    if (!refined) {
      if (dif < 0.9 * best_dif) {
        best_dif = dif;
        stall = 0;
      } else {
        ++stall;
      }
    }
    if (!refined && (dif < p->refine_threshold || (stall >= 4 && dif < 100.0 * p->refine_threshold))) {
      if ((rc = refine_now())) return rc;
    }
    if (broyden) {
      // Broyden mixing of the potential (SCF::BroydenMix, scf.cpp:2144-2261):
      // density-sphere Fourier components, RhoDdot inner products
      PhaseTimer pt_(prof, &tph[4]);
      const int N = ctx->nf[0];
      const double2* tw = (const double2*)S.tw.p;
      const double* mask = (const double*)S.bmask.p;
      const double* bwp = (const double*)S.bw.p;
      double* vin = (double*)S.vtot.p;
      double2* A = (double2*)S.bA.p;    // GvOld
      double2* B = (double2*)S.bB.p;    // GvNew (the residual)
      double2* df = (double2*)S.bdf.p;
      double2* dv = (double2*)S.bdv.p;
      double2* cdf0 = (double2*)S.bcdf.p;
      double2* cdf1 = cdf0 + nf;
      const double sc = ctx->vol / (double)nf;
      if ((rc = fft3_real(N, false, A, vin, nullptr, 1.0, tw, nullptr))) return rc;
      k_clin<<<nblk(nf), 256>>>(nf, sc, A, 0.0, nullptr, mask, A);
      if ((rc = fft3_real(N, false, B, (const double*)S.vtot_new.p, nullptr, 1.0, tw, nullptr))) return rc;
      k_clin<<<nblk(nf), 256>>>(nf, sc, B, -1.0, A, mask, B);
      const int used = std::min(it - 1, mixdim);
      const int ipos = it - 1 - ((it - 2) / mixdim) * mixdim;
      if (it > 1) {
        k_clin<<<nblk(nf), 256>>>(nf, 1.0, cdf0, -1.0, B, nullptr, df + (size_t)(ipos - 1) * nf);
        k_clin<<<nblk(nf), 256>>>(nf, 1.0, cdf1, -1.0, A, nullptr, dv + (size_t)(ipos - 1) * nf);
      }
      PWB_CUDA(cudaMemcpy(cdf0, B, nf * 16, cudaMemcpyDeviceToDevice));
      PWB_CUDA(cudaMemcpy(cdf1, A, nf * 16, cudaMemcpyDeviceToDevice));
      if (used > 0) {
        // beta_ij = RhoDdot(df_j, df_i) and work_i = RhoDdot(df_i, GvNew): one batch of reductions
        double* dd = (double*)S.bdots.p;
        const size_t ndd = (size_t)used * used + used;
        PWB_CUDA(cudaMemset(dd, 0, ndd * 8));
        for (int i = 0; i < used; ++i)
          for (int j = i; j < used; ++j)
            k_wdot<<<nblk(nf), 256>>>(nf, bwp, df + (size_t)j * nf, df + (size_t)i * nf, dd + i * used + j);
        for (int i = 0; i < used; ++i)
          k_wdot<<<nblk(nf), 256>>>(nf, bwp, df + (size_t)i * nf, B, dd + used * used + i);
        std::vector<double> hd(ndd);
        PWB_CUDA(cudaMemcpy(hd.data(), dd, ndd * 8, cudaMemcpyDeviceToHost));
        // inverse of the symmetric (possibly indefinite) beta matrix (the
        // reference's sytrf / sytri): Gauss-Jordan with partial pivoting
        const int u = used;
        std::vector<double> a((size_t)u * 2 * u, 0.0);
        for (int i = 0; i < u; ++i) {
          for (int j = 0; j < u; ++j) a[(size_t)i * 2 * u + j] = hd[std::min(i, j) * u + std::max(i, j)];
          a[(size_t)i * 2 * u + u + i] = 1.0;
        }
        for (int c0 = 0; c0 < u; ++c0) {
          int piv = c0;
          for (int i = c0 + 1; i < u; ++i)
            if (std::fabs(a[(size_t)i * 2 * u + c0]) > std::fabs(a[(size_t)piv * 2 * u + c0])) piv = i;
          PWB_CHECK(a[(size_t)piv * 2 * u + c0] != 0.0, PW_ENUMERIC, "Broyden beta matrix is singular");
          if (piv != c0)
            for (int j = 0; j < 2 * u; ++j) std::swap(a[(size_t)piv * 2 * u + j], a[(size_t)c0 * 2 * u + j]);
          const double d = a[(size_t)c0 * 2 * u + c0];
          for (int j = 0; j < 2 * u; ++j) a[(size_t)c0 * 2 * u + j] /= d;
          for (int i = 0; i < u; ++i) {
            if (i == c0) continue;
            const double f = a[(size_t)i * 2 * u + c0];
            if (f != 0.0)
              for (int j = 0; j < 2 * u; ++j) a[(size_t)i * 2 * u + j] -= f * a[(size_t)c0 * 2 * u + j];
          }
        }
        for (int i = 0; i < u; ++i) {
          double g0 = 0.0;
          for (int j = 0; j < u; ++j) g0 += a[(size_t)j * 2 * u + u + i] * hd[(size_t)u * u + j];
          k_clin<<<nblk(nf), 256>>>(nf, 1.0, A, -g0, dv + (size_t)i * nf, nullptr, A);
          k_clin<<<nblk(nf), 256>>>(nf, 1.0, B, -g0, df + (size_t)i * nf, nullptr, B);
        }
      }
      k_clin<<<nblk(nf), 256>>>(nf, 1.0, A, p->mix_step, B, nullptr, A);
      // back to real space from the sphere components (backward x 1/vol)
      if ((rc = fft3_real(N, true, A, nullptr, vin, 1.0 / ctx->vol, tw, nullptr))) return rc;
      PWB_CUDA(cudaGetLastError());
    } else
    // Anderson mixing of the potential (scf.cpp:2299-2365)
    {
      PhaseTimer pt_(prof, &tph[4]);
      double* vin = (double*)S.vtot.p;
      double* vout = (double*)S.vtot_new.p;
      double* F = vout;   // F = vout - vin (in place)
      k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, vout, -1.0, vin, F);
      const int dim = std::min(S.nhist, mixdim);
      std::vector<double> theta(dim, 0.0);
      double* dv = (double*)S.dvh.p;
      double* df = (double*)S.dfh.p;
      double* difv = (double*)S.dif_v.p;
      double* diff = (double*)S.dif_f.p;
      if (dim > 0) {
        for (int i = 0; i < dim; ++i) {
          k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, dv + (size_t)i * nf, -1.0, vin, difv + (size_t)i * nf);
          k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, df + (size_t)i * nf, -1.0, F, diff + (size_t)i * nf);
        }
        cublasHandle_t h = (cublasHandle_t)ctx->blas;
        cublasSetStream(h, nullptr);
        DevBuf ov;
        if ((rc = ov.alloc((size_t)(dim + 1) * dim * 8))) return rc;
        const double one = 1.0, zero = 0.0;
        double* O = (double*)ov.p;
        cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, dim, dim, (int)nf, &one, diff, (int)nf, diff, (int)nf, &zero, O, dim);
        cublasDgemv(h, CUBLAS_OP_T, (int)nf, dim, &one, diff, (int)nf, F, 1, &zero, O + (size_t)dim * dim, 1);
        std::vector<double> hO((size_t)(dim + 1) * dim);
        PWB_CUDA(cudaMemcpy(hO.data(), O, hO.size() * 8, cudaMemcpyDeviceToHost));
        // Cholesky solve of the dim x dim system (lapack Potrf/Potrs, scf.cpp:2340-2341)
        std::vector<double> L((size_t)dim * dim, 0.0), b(hO.begin() + (size_t)dim * dim, hO.end());
        for (int j = 0; j < dim; ++j) {
          double s0 = hO[(size_t)j * dim + j];
          for (int k = 0; k < j; ++k) s0 -= L[(size_t)k * dim + j] * L[(size_t)k * dim + j];
          PWB_CHECK(s0 > 0, PW_ENUMERIC, "Anderson overlap not positive definite");
          L[(size_t)j * dim + j] = std::sqrt(s0);
          for (int i2 = j + 1; i2 < dim; ++i2) {
            double s1 = hO[(size_t)j * dim + i2];
            for (int k = 0; k < j; ++k) s1 -= L[(size_t)k * dim + i2] * L[(size_t)k * dim + j];
            L[(size_t)j * dim + i2] = s1 / L[(size_t)j * dim + j];
          }
        }
        for (int i2 = 0; i2 < dim; ++i2) {
          double s1 = b[i2];
          for (int k = 0; k < i2; ++k) s1 -= L[(size_t)k * dim + i2] * b[k];
          b[i2] = s1 / L[(size_t)i2 * dim + i2];
        }
        for (int i2 = dim - 1; i2 >= 0; --i2) {
          double s1 = b[i2];
          for (int k = i2 + 1; k < dim; ++k) s1 -= L[(size_t)i2 * dim + k] * b[k];
          b[i2] = s1 / L[(size_t)i2 * dim + i2];
        }
        theta = b;
      }
      // save history (Xin, F) before forming the mix
      const int slot = S.hpos % mixdim;
      PWB_CUDA(cudaMemcpy(dv + (size_t)slot * nf, vin, nf * 8, cudaMemcpyDeviceToDevice));
      PWB_CUDA(cudaMemcpy(df + (size_t)slot * nf, F, nf * 8, cudaMemcpyDeviceToDevice));
      for (int i = 0; i < dim; ++i) {
        k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, vin, -theta[i], difv + (size_t)i * nf, vin);
        k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, F, -theta[i], diff + (size_t)i * nf, F);
      }
      k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, vin, p->mix_step, F, vin);
      S.hpos++;
      S.nhist = std::min(S.nhist + 1, mixdim);
      PWB_CUDA(cudaGetLastError());
    }
  }
  return PW_OK;
  };
  if ((rc = scf_loop())) return rc;
  double efock = 0.0, dexx = 0.0;
  int phi_it = 0;
  if (hse) {
    // SCF::Iterate hybrid part, "nested" mixing (scf.cpp:628-925)
    if (!refined && (rc = refine_now())) return rc;
    // the graph-captured filter and step hold H*psi without the exchange term
    sv.drop_graphs();
    sv.use_graph = false;
    hse_frac = 0.25;
    if ((rc = potentials(rho, &exc))) return rc;
    k_lincomb<<<nblk(nf), 256>>>(nf, 1.0, (double*)S.vh.p, 1.0, (double*)S.vxc.p, (double*)S.vtot.p);
    if ((rc = pw_exx_setup(ctx, 0.25, 0.106, 1, p->ecut))) return rc;
    // phi <- psi, ACE (SetPhiEXX + CalculateVexxACE) and the Fock energy with it
    auto update_ace = [&]() -> int {
      int q;
      if ((q = pw_exx_set_phi(ctx, sv.X.p, (int)nt, nb, occ.data()))) return q;
      return pw_ace_build(ctx, sv.X.p, (int)nt, nb);
    };
    auto fock = [&](double* e) -> int { return pw_exx_energy(ctx, sv.X.p, (int)nt, nb, occ.data(), 2, 1, e); };
    double fock0 = 0.0, fock1 = 0.0, fock2 = 0.0;
    if ((rc = update_ace()) || (rc = fock(&fock0))) return rc;
    hybrid_phase = true;
    const int phimax = p->phi_max_iter > 0 ? p->phi_max_iter : 10;
    bool phi_conv = false;
    for (phi_it = 1; phi_it <= phimax; ++phi_it) {
      if ((rc = scf_loop())) return rc;
      if ((rc = fock(&fock1)) || (rc = update_ace()) || (rc = fock(&fock2))) return rc;
      dexx = 4.0 * std::fabs(fock1 - 0.5 * (fock0 + fock2));
      fock0 = fock2;
      efock = fock2;
      etot = etot - 2.0 * fock1 + efock;
      efree = efree - 2.0 * fock1 + efock;
      if (p->verbose)
        fprintf(stderr, "phi %3d inner %3d Efock %.10f Etot %.10f Efree %.10f dExx %.3e\n", phi_it, it, efock, etot,
                efree, dexx);
      if (dexx < p->phi_tol) {
        phi_conv = true;
        break;
      }
    }
    phi_it = std::min(phi_it, phimax);
    conv = phi_conv;
    exx_guard.mode = ctx->exx_mode;   // the context keeps the final ACE operator
  }
  r->efock = efock;
  r->dexx = dexx;
  r->phi_iterations = phi_it;
  PWB_CUDA(cudaDeviceSynchronize());
  const auto t_end = std::chrono::steady_clock::now();
  r->etot = etot;
  r->efree = efree;
  r->eharris = eharris;
  r->exc = exc;
  r->ehart = ehart;
  r->eself = eself;
  r->fermi = ef;
  r->iterations = total_it;
  r->converged = conv ? 1 : 0;
  r->time_s = std::chrono::duration<double>(t_end - t_start).count();
  for (int i = 0; i < 6; ++i) r->phase_s[i] = tph[i];
  for (int i = 0; i < 4; ++i) r->sub_s[i] = g_sub[i];
  g_sub_on = false;
  if (eig_out) std::copy(eig.begin(), eig.end(), eig_out);
  if (rho_out) PWB_CUDA(cudaMemcpy(rho_out, rho, nf * 8, cudaMemcpyDeviceToHost));
  // keep the final FP64 bands, occupations and output density for pw_scf_forces
  ctx->scf_nband = 0;
  if (sv.c == ctx) {
    if ((rc = ctx->scf_psi.alloc((size_t)nb * nt * 8)) || (rc = ctx->scf_rho.alloc(nf * 8))) return rc;
    PWB_CUDA(cudaMemcpy(ctx->scf_psi.p, sv.X.p, (size_t)nb * nt * 8, cudaMemcpyDeviceToDevice));
    PWB_CUDA(cudaMemcpy(ctx->scf_rho.p, rho, nf * 8, cudaMemcpyDeviceToDevice));
    ctx->scf_occ = occ;
    ctx->scf_nband = nb;
  }
  return PW_OK;
}

int pw_hartree(pw_ctx* ctx, const double* drho_dev, double ecut, double* vh_dev) {
  PWB_CHECK(ctx && drho_dev && vh_dev && ecut > 0, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const long nf = ctx->ntotf;
  DevBuf kern, work, tw;
  int rc;
  if ((rc = kern.alloc(nf * 8)) || (rc = work.alloc(nf * 16)) || (rc = tw.alloc(ctx->nf[0] * 16))) return rc;
  std::vector<double> k(nf);
  const int N0 = ctx->nf[0], N1 = ctx->nf[1], N2 = ctx->nf[2];
  for (int z = 0; z < N2; ++z)
    for (int y = 0; y < N1; ++y)
      for (int x = 0; x < N0; ++x) {
        const double m0 = x <= N0 / 2 ? x : x - N0, m1 = y <= N1 / 2 ? y : y - N1, m2 = z <= N2 / 2 ? z : z - N2;
        const double g0 = 2 * M_PI / ctx->L[0] * m0, g1 = 2 * M_PI / ctx->L[1] * m1, g2 = 2 * M_PI / ctx->L[2] * m2;
        const double gkk = (g0 * g0 + g1 * g1 + g2 * g2) / 2;
        k[x + (size_t)N0 * (y + (size_t)N1 * z)] = (gkk <= 1e-16 || gkk > 4.0 * ecut) ? 0.0 : 2.0 * M_PI / gkk / (double)nf;
      }
  PWB_CUDA(cudaMemcpy(kern.p, k.data(), nf * 8, cudaMemcpyHostToDevice));
  std::vector<double> t(2 * N0);
  for (int m = 0; m < N0; ++m) {
    t[2 * m] = std::cos(2 * M_PI * m / N0);
    t[2 * m + 1] = -std::sin(2 * M_PI * m / N0);
  }
  PWB_CUDA(cudaMemcpy(tw.p, t.data(), N0 * 16, cudaMemcpyHostToDevice));
  rc = hartree(ctx, (double2*)work.p, drho_dev, nullptr, (const double*)kern.p, vh_dev, (const double2*)tw.p, nullptr);
  if (rc) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

static int xc_gga_entry(pw_ctx* ctx, const double* rho_dev, double ecut, double* eps_dev, double* vxc_dev,
                        double hse_frac) {
  PWB_CHECK(ctx && rho_dev && eps_dev && vxc_dev && ecut > 0, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  const long nf = ctx->ntotf;
  const int N = ctx->nf[0];
  DevBuf a, b, g, tw;
  int rc;
  if ((rc = a.alloc(nf * 16)) || (rc = b.alloc(nf * 16)) || (rc = g.alloc(3 * nf * 8)) || (rc = tw.alloc(N * 16)))
    return rc;
  std::vector<double> t(2 * N);
  for (int m = 0; m < N; ++m) {
    t[2 * m] = std::cos(2 * M_PI * m / N);
    t[2 * m + 1] = -std::sin(2 * M_PI * m / N);
  }
  PWB_CUDA(cudaMemcpy(tw.p, t.data(), N * 16, cudaMemcpyHostToDevice));
  if ((rc = xc_pbe(ctx, rho_dev, ecut, eps_dev, vxc_dev, (double2*)a.p, (double2*)b.p, (double*)g.p,
                   (const double2*)tw.p, nullptr, hse_frac)))
    return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

int pw_xc_pbe(pw_ctx* ctx, const double* rho_dev, double ecut, double* eps_dev, double* vxc_dev) {
  return xc_gga_entry(ctx, rho_dev, ecut, eps_dev, vxc_dev, 0.0);
}

int pw_xc_hse06(pw_ctx* ctx, const double* rho_dev, double ecut, double* eps_dev, double* vxc_dev) {
  return xc_gga_entry(ctx, rho_dev, ecut, eps_dev, vxc_dev, 0.25);
}

int pw_xc_teter93(pw_ctx* ctx, const double* rho_dev, double* eps_dev, double* vxc_dev) {
  PWB_CHECK(ctx && rho_dev && eps_dev && vxc_dev, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  k_xc_teter93<<<nblk(ctx->ntotf), 256>>>(ctx->ntotf, rho_dev, eps_dev, vxc_dev);
  PWB_CUDA(cudaGetLastError());
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

int pw_ctx_build_twin(pw_ctx* ctx) {
  PWB_CHECK(ctx && ctx->prec == PW_F64, PW_EINVAL, "the twin is built for an FP64 context");
  PWB_CHECK(!ctx->atom_z.empty(), PW_ENOTREADY, "atoms not set (pw_set_atoms)");
  if (ctx->twin) return PW_OK;
  pw_ctx* c32 = nullptr;
  int rc = ctx->gs ? pw_ctx_create_gspace(ctx->L, ctx->nf, ctx->gs_ecut, PW_F32, ctx->device, &c32)
                   : pw_ctx_create(ctx->L, ctx->n, ctx->nf, PW_F32, ctx->device, &c32);
  if (rc) return rc;
  if ((rc = pw_set_band_batch(c32, std::max(2, 2 * ctx->pair_cap))) ||
      (rc = pw_set_atoms(c32, (int)ctx->atom_z.size(), ctx->atom_z.data(), ctx->atom_pos.data()))) {
    pw_ctx_destroy(c32);
    return rc;
  }
  ctx->twin = c32;
  return PW_OK;
}

int pw_cholqr(pw_ctx* ctx, void* X, int nb) {
  PWB_CHECK(ctx && X && nb > 0, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  Dense dn;
  int rc = dn.init((cublasHandle_t)ctx->blas);
  if (rc) return rc;
  Solver sv;
  sv.c = ctx;
  sv.nt = ctx->ntot;
  sv.esz = ctx->esz;
  if ((rc = alloc_block(sv, sv.Y, nb))) return rc;
  rc = cholqr(sv, dn, X, nb, sv.Y.p);
  PWB_CUDA(cudaDeviceSynchronize());
  dn.release();
  return rc;
}

int pw_eigsolve(pw_ctx* ctx, int solver, void* X, int nb, int maxit, double tol, int degree, double* eig,
                double* resnorm, int* iters) {
  PWB_CHECK(ctx && X && nb > 0, PW_EINVAL, "bad arguments");
  PWB_CHECK(ctx->have_vtot, PW_ENOTREADY, "local potential not set (pw_set_vtot)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  Dense dn;
  int rc = dn.init((cublasHandle_t)ctx->blas);
  if (rc) return rc;
  if ((rc = pw_set_band_batch(ctx, nb))) return rc;
  Solver sv;
  sv.c = ctx;
  sv.nt = ctx->ntot;
  sv.esz = ctx->esz;
  sv.nb = nb;
  for (DevBuf* b : {&sv.X, &sv.HX, &sv.Y, &sv.HY, &sv.Z})
    if ((rc = alloc_block(sv, *b, nb))) return rc;
  PWB_CUDA(cudaMemcpy(sv.X.p, X, (size_t)nb * sv.nt * sv.esz, cudaMemcpyDeviceToDevice));
  if (ctx->gs)   // sphere-cut bands: Im c_0 is not a degree of freedom
    PWB_CUDA(cudaMemset2D((char*)sv.X.p + ctx->esz, sv.nt * ctx->esz, 0, ctx->esz, nb));
  // the first MultSpinor call of a filtered Hamiltonian replaces psi by P psi
  // (hamiltonian.cpp:3090-3116)
  if (ctx->wfn_filter && (rc = wfn_filter_pass(ctx, sv.X.p, (int)sv.nt, nb, nullptr))) return rc;
  int it = 0;
  if (solver == PW_SOLVER_LOBPCG) {
    rc = lobpcg(sv, dn, nb, maxit, tol, true, &it);
  } else if (solver == PW_SOLVER_PPCG) {
    rc = ppcg(sv, dn, nb, degree > 0 ? degree : 1, maxit, tol, true, &it);
  } else if (solver == PW_SOLVER_DAVIDSON) {
    rc = davidson(sv, dn, nb, degree >= 2 ? degree : 2, maxit, tol, true, &it);
  } else {
    double up, lo;
    if ((rc = lanczos_upper(sv, 16, &up, &lo))) return rc;
    if ((rc = cholqr(sv, dn, sv.X.p, nb, sv.Y.p))) return rc;
    if ((rc = hpsi(ctx, sv.X.p, sv.HX.p, nb, nullptr))) return rc;
    if ((rc = rayleigh_ritz(sv, dn, sv.X.p, sv.HX.p, sv.Z.p, sv.HY.p, nb))) return rc;
    PWB_CUDA(cudaMemcpy(sv.X.p, sv.Z.p, (size_t)nb * sv.nt * sv.esz, cudaMemcpyDeviceToDevice));
    PWB_CUDA(cudaMemcpy(sv.HX.p, sv.HY.p, (size_t)nb * sv.nt * sv.esz, cudaMemcpyDeviceToDevice));
    const double frac = std::pow((double)nb / (double)sv.nt, 2.0 / 3.0);
    double a = lo + 2.0 * frac * (up - lo), a0 = lo;
    for (it = 1; it <= maxit; ++it) {
      if ((rc = chebfsi_step(sv, dn, nb, degree, a, up, a0))) break;
      a = sv.eig[nb - 1];
      a0 = sv.eig[0];
      if ((rc = residuals(sv, nb))) break;
      if (*std::max_element(sv.res.begin(), sv.res.end()) < tol) break;
    }
    it = std::min(it, maxit);
  }
  if (rc) return rc;
  if (sv.res.empty() && (rc = residuals(sv, nb))) return rc;
  PWB_CUDA(cudaMemcpy(X, sv.X.p, (size_t)nb * sv.nt * sv.esz, cudaMemcpyDeviceToDevice));
  if (eig) std::copy(sv.eig.begin(), sv.eig.end(), eig);
  if (resnorm) std::copy(sv.res.begin(), sv.res.end(), resnorm);
  if (iters) *iters = it;
  PWB_CUDA(cudaDeviceSynchronize());
  dn.release();
  return PW_OK;
}

int pw_density(pw_ctx* ctx, const void* psi, int ld, int nband, const double* occ_host, int nocc_total,
               double* rho_dev) {
  PWB_CHECK(ctx && psi && occ_host && rho_dev && nband > 0, PW_EINVAL, "bad arguments");
  PWB_CHECK(ld >= ctx->ntot, PW_EINVAL, "Domain size does not match.");
  PWB_CHECK(!ctx->gs || (ld % 2 == 0 && (uintptr_t)psi % (2 * ctx->esz) == 0), PW_EINVAL,
            "G-space bands are complex: even leading dimension and complex-aligned pointer");
  PWB_CUDA(cudaSetDevice(ctx->device));
  DevBuf wv;
  int rc = wv.alloc((nband + 2) * 8);
  if (rc) return rc;
  std::vector<double> h(nband + 2, 0.0);
  for (int i = 0; i < nband; ++i) h[i] = 2.0 * occ_host[i];
  PWB_CUDA(cudaMemcpy(wv.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice));
  PWB_CUDA(cudaMemset(rho_dev, 0, ctx->ntotf * 8));
  const int cap = ctx->pair_cap;
  for (int b0 = 0; b0 < nband; b0 += 2 * cap) {
    const int npair = std::min(cap, (nband - b0 + 1) / 2);
    if ((rc = run_density(ctx, psi, ld, nband, b0, npair, (const double*)wv.p, rho_dev, nullptr))) return rc;
  }
  // renormalise to 2 * nocc electrons (hamiltonian.cpp:2596-2600); nocc_total
  // <= 0: the raw sum (a rank's part of a band-distributed density)
  if (nocc_total <= 0) {
    PWB_CUDA(cudaDeviceSynchronize());
    return PW_OK;
  }
  DevBuf d;
  if ((rc = d.alloc(64))) return rc;
  PWB_CUDA(cudaMemset(d.p, 0, 64));
  DotSet ds{};
  ds.k = 1;
  ds.a[0] = rho_dev;
  ds.b[0] = nullptr;
  k_dots<<<nblk(ctx->ntotf), 256>>>(ctx->ntotf, ds, (double*)d.p);
  double tot;
  PWB_CUDA(cudaMemcpy(&tot, d.p, 8, cudaMemcpyDeviceToHost));
  k_lincomb<<<nblk(ctx->ntotf), 256>>>(ctx->ntotf, (2.0 * nocc_total * (double)ctx->ntotf) / (ctx->vol * tot), rho_dev,
                                       0.0, nullptr, rho_dev);
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

}  // extern "C"
