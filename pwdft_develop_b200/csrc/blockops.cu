// Device block operations for the eigensolvers and the SCF driver.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "blockops.hpp"
#include "gemm.hpp"

namespace pwb {

template <typename T>
__global__ void k_axpby(int n, int nb, double a, const T* __restrict__ X, long ldx, double b, T* __restrict__ Y,
                        long ldy) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = a * (double)X[(long)j * ldx + i] + (b == 0.0 ? 0.0 : b * (double)Y[(long)j * ldy + i]);
    Y[(long)j * ldy + i] = (T)v;
  }
}

template <typename T>
__global__ void k_axpbypcz(int n, int nb, double a, const T* __restrict__ X, double b, const T* __restrict__ Y,
                           double c, const T* __restrict__ W, T* __restrict__ Z, long ld) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long o = (long)j * ld + i;
    Z[o] = (T)(a * (double)X[o] + b * (double)Y[o] + c * (double)W[o]);
  }
}

template <typename T>
__global__ void k_colnorm2(int n, const T* __restrict__ X, long ld, double* __restrict__ out) {
  const int j = blockIdx.x;
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = (double)X[(long)j * ld + i];
    s += v * v;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[j] = s;
  }
}

template <typename T>
__global__ void k_colscale(int n, T* __restrict__ X, long ld, const double* __restrict__ s) {
  const int j = blockIdx.y;
  const double f = s[j];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    X[(long)j * ld + i] = (T)((double)X[(long)j * ld + i] * f);
}

template <typename A, typename B>
__global__ void k_convert2d(int n, const A* __restrict__ x, long ldx, B* __restrict__ y, long ldy) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[(long)j * ldy + i] = (B)x[(long)j * ldx + i];
}

static inline dim3 grid2(int n, int nb) { return dim3(std::max(1, std::min((n + 255) / 256, 256)), nb); }

template <typename T> int axpby(int n, int nb, double a, const T* X, long ldx, double b, T* Y, long ldy, cudaStream_t st) {
  if (n == 0 || nb == 0) return PW_OK;
  k_axpby<T><<<grid2(n, nb), 256, 0, st>>>(n, nb, a, X, ldx, b, Y, ldy);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
template <typename T>
int axpbypcz(int n, int nb, double a, const T* X, double b, const T* Y, double c, const T* W, T* Z, long ld,
             cudaStream_t st) {
  if (n == 0 || nb == 0) return PW_OK;
  k_axpbypcz<T><<<grid2(n, nb), 256, 0, st>>>(n, nb, a, X, b, Y, c, W, Z, ld);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
template <typename T> int colnorm2(int n, int nb, const T* X, long ld, double* out, cudaStream_t st) {
  if (nb == 0) return PW_OK;
  k_colnorm2<T><<<nb, 512, 0, st>>>(n, X, ld, out);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
template <typename T> int colscale(int n, int nb, T* X, long ld, const double* s, cudaStream_t st) {
  if (n == 0 || nb == 0) return PW_OK;
  k_colscale<T><<<grid2(n, nb), 256, 0, st>>>(n, X, ld, s);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
int copy_d2f_2d(int n, int nb, const double* x, long ldx, float* y, long ldy, cudaStream_t st) {
  if (n == 0 || nb == 0) return PW_OK;
  k_convert2d<double, float><<<grid2(n, nb), 256, 0, st>>>(n, x, ldx, y, ldy);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
int copy_f2d_2d(int n, int nb, const float* x, long ldx, double* y, long ldy, cudaStream_t st) {
  if (n == 0 || nb == 0) return PW_OK;
  k_convert2d<float, double><<<grid2(n, nb), 256, 0, st>>>(n, x, ldx, y, ldy);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
int copy_d2f(long n, const double* x, float* y, cudaStream_t st) { return copy_d2f_2d((int)n, 1, x, n, y, n, st); }
int copy_f2d(long n, const float* x, double* y, cudaStream_t st) { return copy_f2d_2d((int)n, 1, x, n, y, n, st); }

template int axpby<float>(int, int, double, const float*, long, double, float*, long, cudaStream_t);
template int axpby<double>(int, int, double, const double*, long, double, double*, long, cudaStream_t);
template int axpbypcz<float>(int, int, double, const float*, double, const float*, double, const float*, float*, long,
                             cudaStream_t);
template int axpbypcz<double>(int, int, double, const double*, double, const double*, double, const double*, double*,
                              long, cudaStream_t);
template int colnorm2<float>(int, int, const float*, long, double*, cudaStream_t);
template int colnorm2<double>(int, int, const double*, long, double*, cudaStream_t);
// B = alpha A for an m x n column-major block
__global__ void k_dense_scale(int m, int n, double alpha, const double* __restrict__ A, int lda, double* __restrict__ B,
                              int ldb) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)m * n) return;
  const int r = (int)(i % m), c = (int)(i / m);
  B[(long)c * ldb + r] = alpha * A[(long)c * lda + r];
}
int dense_scale(int m, int n, double alpha, const double* A, int lda, double* B, int ldb, cudaStream_t st) {
  if ((long)m * n == 0) return PW_OK;
  k_dense_scale<<<(unsigned)(((long)m * n + 255) / 256), 256, 0, st>>>(m, n, alpha, A, lda, B, ldb);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// v[i] <- 1 / sqrt(v[i])
__global__ void k_rsqrt(int n, double* v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = v[i] > 1e-300 ? 1.0 / sqrt(v[i]) : 0.0;
}
int vec_rsqrt(int n, double* v, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_rsqrt<<<(n + 255) / 256, 256, 0, st>>>(n, v);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// residual norms of the eigensolvers, ||r_k|| / max(1, |lambda_k|) with
// lambda_k = G(k, k) (lobpcg.cpp:705-709), and their maximum in out[n]; one CTA
__global__ void k_resnorm(int n, const double* __restrict__ nrm2, const double* __restrict__ G, int ldg,
                          double* __restrict__ out) {
  __shared__ double red[32];
  double mx = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double r = sqrt(nrm2[k]) / fmax(1.0, fabs(G[(long)k * ldg + k]));
    out[k] = r;
    mx = fmax(mx, r);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    out[n] = m;
  }
}
int resnorms(int n, const double* nrm2, const double* G, int ldg, double* out, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_resnorm<<<1, 256, 0, st>>>(n, nrm2, G, ldg, out);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

template int colscale<float>(int, int, float*, long, const double*, cudaStream_t);
template int colscale<double>(int, int, double*, long, const double*, cudaStream_t);

// Diagonal sb x sb blocks of U^T V over one grid-point split; partial sums
// written to part[(split * nsb + k) * SB * SB + i + j * SB].
template <typename T, int SB>
__global__ void __launch_bounds__(256)
k_bdiag_dots(int n, int width, int sb, const T* __restrict__ U, const T* __restrict__ V, long ld, int chunk,
             double* __restrict__ part) {
  const int k = blockIdx.x, split = blockIdx.y, nsb = gridDim.x;
  const int c0 = k * sb;
  const int sbk = min(sb, width - c0);
  const int g0 = split * chunk, g1 = min(n, g0 + chunk);
  double acc[SB * SB];
#pragma unroll
  for (int e = 0; e < SB * SB; ++e) acc[e] = 0.0;
  for (int g = g0 + threadIdx.x; g < g1; g += blockDim.x) {
    double u[SB], v[SB];
#pragma unroll
    for (int i = 0; i < SB; ++i) {
      u[i] = i < sbk ? (double)U[(long)(c0 + i) * ld + g] : 0.0;
      v[i] = i < sbk ? (double)V[(long)(c0 + i) * ld + g] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < SB; ++j)
#pragma unroll
      for (int i = 0; i < SB; ++i) acc[i + j * SB] += u[i] * v[j];
  }
  __shared__ double red[8][SB * SB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int e = 0; e < SB * SB; ++e) {
    double x = acc[e];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][e] = x;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < SB * SB; e += blockDim.x) {
    double x = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[w][e];
    part[((long)split * nsb + k) * SB * SB + e] = x;
  }
}

// Y[:, k*sb + j] = beta Y + sum_i X[:, k*sb + i] C[k*sb*sb + i + j*sb]
template <typename T, int SB>
__global__ void k_bdiag_rotate(int n, int width, int sb, const T* __restrict__ X, long ldx,
                               const double* __restrict__ C, T* __restrict__ Y, long ldy, double beta) {
  const int k = blockIdx.y;
  const int c0 = k * sb;
  const int sbk = min(sb, width - c0);
  const double* Ck = C + (long)k * sb * sb;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
    double x[SB];
#pragma unroll
    for (int i = 0; i < SB; ++i) x[i] = i < sbk ? (double)X[(long)(c0 + i) * ldx + g] : 0.0;
#pragma unroll
    for (int j = 0; j < SB; ++j) {
      if (j < sbk) {
        double y = 0;
#pragma unroll
        for (int i = 0; i < SB; ++i)
          if (i < sbk) y += x[i] * Ck[i + j * sb];
        T* yp = Y + (long)(c0 + j) * ldy + g;
        *yp = (T)(beta == 0.0 ? y : y + beta * (double)*yp);
      }
    }
  }
}

// Chebyshev recurrence steps with device-resident coefficients (so that a
// captured filter graph replays with new interval bounds):
// Y = c[0] HY + c[1] X;  Z = c[0] HY + c[1] Y + c[2] X
template <typename T>
__global__ void k_cheb_lin(int n, const double* __restrict__ c, const T* __restrict__ HY, const T* __restrict__ Y,
                           const T* __restrict__ X, T* __restrict__ Z, long ld, int three) {
  const int j = blockIdx.y;
  const double c0 = c[0], c1 = c[1], c2 = three ? c[2] : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long o = (long)j * ld + i;
    double v = c0 * (double)HY[o] + c1 * (double)Y[o];
    if (three) v += c2 * (double)X[o];
    Z[o] = (T)v;
  }
}

template <typename T>
int cheb_lin(int n, int nb, const double* coef_dev, const T* HY, const T* Y, const T* X, T* Z, long ld,
             cudaStream_t st) {
  k_cheb_lin<T><<<grid2(n, nb), 256, 0, st>>>(n, coef_dev, HY, Y, X, Z, ld, X ? 1 : 0);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
template int cheb_lin<float>(int, int, const double*, const float*, const float*, const float*, float*, long,
                             cudaStream_t);
template int cheb_lin<double>(int, int, const double*, const double*, const double*, const double*, double*, long,
                              cudaStream_t);

template <typename T>
int bdiag_dots(int n, int width, int sb, const T* U, const T* V, long ld, DevBuf& part, double* out_host,
               cudaStream_t st) {
  PWB_CHECK(sb >= 1 && sb <= 8, PW_EUNSUPPORTED, "sub-block size 1..8");
  const int nsb = (width + sb - 1) / sb;
  const int nsplit = std::max(1, std::min(64, (2 * 148 + nsb - 1) / nsb));
  const int chunk = (n + nsplit - 1) / nsplit;
  const int SBp = sb == 1 ? 1 : sb == 2 ? 2 : sb <= 4 ? 4 : 8;
  int rc = part.alloc((size_t)nsplit * nsb * SBp * SBp * 8);
  if (rc) return rc;
  double* pp = (double*)part.p;
  dim3 grid(nsb, nsplit);
  switch (SBp) {
    case 1: k_bdiag_dots<T, 1><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    case 2: k_bdiag_dots<T, 2><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    case 4: k_bdiag_dots<T, 4><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    default: k_bdiag_dots<T, 8><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
  }
  PWB_CUDA(cudaGetLastError());
  std::vector<double> h((size_t)nsplit * nsb * SBp * SBp);
  PWB_CUDA(cudaMemcpyAsync(h.data(), pp, h.size() * 8, cudaMemcpyDeviceToHost, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  // deterministic sum over splits; out_host[k][i + j*sb]
  for (int k = 0; k < nsb; ++k)
    for (int j = 0; j < sb; ++j)
      for (int i = 0; i < sb; ++i) {
        double x = 0;
        for (int sp = 0; sp < nsplit; ++sp) x += h[((size_t)sp * nsb + k) * SBp * SBp + i + j * SBp];
        out_host[(size_t)k * sb * sb + i + j * sb] = x;
      }
  return PW_OK;
}

// out[k * sb * sb + i + j * sb] = sum over the grid splits (fixed order)
__global__ void k_bdiag_sum(const double* __restrict__ part, int nsplit, int nsb, int SBp, int sb,
                            double* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nsb * sb * sb) return;
  const int k = idx / (sb * sb), r = idx % (sb * sb), i = r % sb, j = r / sb;
  double x = 0;
  for (int sp = 0; sp < nsplit; ++sp) x += part[((long)sp * nsb + k) * SBp * SBp + i + j * SBp];
  out[idx] = x;
}

template <typename T>
int bdiag_dots_dev(int n, int width, int sb, const T* U, const T* V, long ld, DevBuf& part, double* out_dev,
                   cudaStream_t st) {
  PWB_CHECK(sb >= 1 && sb <= 8, PW_EUNSUPPORTED, "sub-block size 1..8");
  const int nsb = (width + sb - 1) / sb;
  const int nsplit = std::max(1, std::min(64, (n + 4095) / 4096));
  const int chunk = (n + nsplit - 1) / nsplit;
  const int SBp = sb == 1 ? 1 : sb == 2 ? 2 : sb <= 4 ? 4 : 8;
  int rc = part.alloc((size_t)nsplit * nsb * SBp * SBp * 8);
  if (rc) return rc;
  double* pp = (double*)part.p;
  dim3 grid(nsb, nsplit);
  switch (SBp) {
    case 1: k_bdiag_dots<T, 1><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    case 2: k_bdiag_dots<T, 2><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    case 4: k_bdiag_dots<T, 4><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
    default: k_bdiag_dots<T, 8><<<grid, 256, 0, st>>>(n, width, sb, U, V, ld, chunk, pp); break;
  }
  const int tot = nsb * sb * sb;
  k_bdiag_sum<<<(tot + 255) / 256, 256, 0, st>>>(pp, nsplit, nsb, SBp, sb, out_dev);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
template int bdiag_dots_dev<float>(int, int, int, const float*, const float*, long, DevBuf&, double*, cudaStream_t);
template int bdiag_dots_dev<double>(int, int, int, const double*, const double*, long, DevBuf&, double*,
                                    cudaStream_t);

// ---------------------------------------------------------------------------
// PPCG sub-block generalized eigenproblems on the device: one warp per
// sub-block k solves A z = lambda B z (dim = numSet * m <= 24) with the cut of
// SolveGenEig: cyclic Jacobi of B, directions with sigma / sigma_max > 1e-8
// kept, Q = U_k sigma_k^-1/2, Jacobi of Q^T A Q, ascending order, Z = Q V; the
// coefficient blocks cx, cw, cp of x <- x cx + w cw + p cp (ppcg.cpp:
// 1001-1090).  Fewer kept directions than columns: x is kept (cx = I).
// ---------------------------------------------------------------------------
constexpr int SYGV_MAX = 24;

__device__ void warp_jacobi(int n, double* M, double* V) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < n * n; e += 32) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  __syncwarp();
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int e = lane; e < n * n; e += 32) {
      const double x = M[e];
      tot += x * x;
      if (e % n != e / n) off += x * x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if (off == 0.0 || off <= 1e-30 * tot) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = M[p + q * n];
        if (apq == 0.0) continue;
        const double app = M[p + p * n], aqq = M[q + q * n];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
          const double mkp = M[k + p * n], mkq = M[k + q * n];
          M[k + p * n] = c * mkp - sn * mkq;
          M[k + q * n] = sn * mkp + c * mkq;
        }
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
          const double mpk = M[p + k * n], mqk = M[q + k * n];
          M[p + k * n] = c * mpk - sn * mqk;
          M[q + k * n] = sn * mpk + c * mqk;
        }
        for (int k = lane; k < n; k += 32) {
          const double vkp = V[k + p * n], vkq = V[k + q * n];
          V[k + p * n] = c * vkp - sn * vkq;
          V[k + q * n] = sn * vkp + c * vkq;
        }
        __syncwarp();
      }
  }
}

struct SubGrams {
  const double *xax, *waw, *xaw, *xx, *ww, *xw, *pap, *xap, *wap, *pp, *xp, *wp;
};

__global__ void __launch_bounds__(32) k_ppcg_sygv(int width, int sb, int numSet, SubGrams g, double* Cx, double* Cw,
                                                  double* Cp) {
  __shared__ double a[SYGV_MAX * SYGV_MAX], b[SYGV_MAX * SYGV_MAX], U[SYGV_MAX * SYGV_MAX], Q[SYGV_MAX * SYGV_MAX],
      AQ[SYGV_MAX * SYGV_MAX], V[SYGV_MAX * SYGV_MAX];
  __shared__ int kept[SYGV_MAX], ord[SYGV_MAX];
  __shared__ int nkept;
  const int lane = threadIdx.x;
  const int k = blockIdx.x;
  const int m = min(sb, width - k * sb), n = numSet * m;
  const long o = (long)k * sb * sb;
  // A and B from the upper blocks (symmetric fill)
  for (int e = lane; e < n * n; e += 32) {
    const int i = e % n, j = e / n;
    const int ii = min(i, j), jj = max(i, j);
    const int bi = ii / m, bj = jj / m, ri = ii % m, rj = jj % m;
    const double *sa, *sbm;
    if (bi == 0 && bj == 0) { sa = g.xax; sbm = g.xx; }
    else if (bi == 1 && bj == 1) { sa = g.waw; sbm = g.ww; }
    else if (bi == 0 && bj == 1) { sa = g.xaw; sbm = g.xw; }
    else if (bi == 2 && bj == 2) { sa = g.pap; sbm = g.pp; }
    else if (bi == 0 && bj == 2) { sa = g.xap; sbm = g.xp; }
    else { sa = g.wap; sbm = g.wp; }
    a[e] = sa[o + ri + rj * sb];
    b[e] = sbm[o + ri + rj * sb];
  }
  __syncwarp();
  warp_jacobi(n, b, U);
  if (lane == 0) {
    double smax = 0.0;
    for (int i = 0; i < n; ++i) smax = fmax(smax, b[i + i * n]);
    int r = 0;
    for (int i = 0; i < n; ++i)
      if (smax > 0.0 && b[i + i * n] / smax > 1e-8) kept[r++] = i;
    nkept = r;
  }
  __syncwarp();
  const int r = nkept;
  double* cx = Cx + o;
  double* cw = Cw + o;
  double* cp = Cp + o;
  for (int e = lane; e < sb * sb; e += 32) {
    cx[e] = 0.0;
    cw[e] = 0.0;
    cp[e] = 0.0;
  }
  __syncwarp();
  if (r < m) {
    // fewer independent directions than columns: keep x
    for (int i = lane; i < m; i += 32) cx[i + i * sb] = 1.0;
    return;
  }
  for (int e = lane; e < n * r; e += 32) {
    const int i = e % n, j = e / n, c = kept[j];
    Q[i + j * n] = U[i + c * n] * (1.0 / sqrt(b[c + c * n]));
  }
  __syncwarp();
  for (int e = lane; e < n * r; e += 32) {
    const int i = e % n, j = e / n;
    double t = 0.0;
    for (int kk = 0; kk < n; ++kk) t += a[i + kk * n] * Q[kk + j * n];
    AQ[i + j * n] = t;
  }
  __syncwarp();
  double* M = b;   // B is no longer needed
  for (int e = lane; e < r * r; e += 32) {
    const int i = e % r, j = e / r;
    double t = 0.0;
    for (int kk = 0; kk < n; ++kk) t += Q[kk + i * n] * AQ[kk + j * n];
    U[i + j * r] = t;
  }
  __syncwarp();
  for (int e = lane; e < r * r; e += 32) {
    const int i = e % r, j = e / r;
    M[i + j * r] = (i == j) ? U[e] : 0.5 * (U[i + j * r] + U[j + i * r]);
  }
  __syncwarp();
  warp_jacobi(r, M, V);
  if (lane == 0) {
    for (int i = 0; i < r; ++i) ord[i] = i;
    for (int i = 1; i < r; ++i) {       // stable insertion sort by eigenvalue
      const int x = ord[i];
      int j = i - 1;
      while (j >= 0 && M[ord[j] + ord[j] * r] > M[x + x * r]) {
        ord[j + 1] = ord[j];
        --j;
      }
      ord[j + 1] = x;
    }
  }
  __syncwarp();
  for (int e = lane; e < n * m; e += 32) {
    const int i = e % n, jj = e / n, j = ord[jj];
    double t = 0.0;
    for (int kk = 0; kk < r; ++kk) t += Q[i + kk * n] * V[kk + j * r];
    const int blk = i / m, ri = i % m;
    double* dst = blk == 0 ? cx : blk == 1 ? cw : cp;
    dst[ri + jj * sb] = t;
  }
}

int ppcg_subblock_solve(int width, int sb, int numSet, const double* const* grams, double* Cx, double* Cw, double* Cp,
                        cudaStream_t st) {
  PWB_CHECK(sb >= 1 && sb <= 8 && numSet >= 2 && numSet <= 3, PW_EUNSUPPORTED, "PPCG sub-block 1..8");
  const int nsb = (width + sb - 1) / sb;
  SubGrams g{grams[0], grams[1], grams[2], grams[3], grams[4], grams[5],
             grams[6], grams[7], grams[8], grams[9], grams[10], grams[11]};
  k_ppcg_sygv<<<nsb, 32, 0, st>>>(width, sb, numSet, g, Cx, Cw, Cp);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

template <typename T>
int bdiag_rotate(int n, int width, int sb, const T* X, long ldx, const double* C_dev, T* Y, long ldy, double beta,
                 cudaStream_t st) {
  PWB_CHECK(sb >= 1 && sb <= 8, PW_EUNSUPPORTED, "sub-block size 1..8");
  const int nsb = (width + sb - 1) / sb;
  dim3 grid(std::max(1, std::min((n + 255) / 256, 128)), nsb);
  const int SBp = sb == 1 ? 1 : sb == 2 ? 2 : sb <= 4 ? 4 : 8;
  switch (SBp) {
    case 1: k_bdiag_rotate<T, 1><<<grid, 256, 0, st>>>(n, width, sb, X, ldx, C_dev, Y, ldy, beta); break;
    case 2: k_bdiag_rotate<T, 2><<<grid, 256, 0, st>>>(n, width, sb, X, ldx, C_dev, Y, ldy, beta); break;
    case 4: k_bdiag_rotate<T, 4><<<grid, 256, 0, st>>>(n, width, sb, X, ldx, C_dev, Y, ldy, beta); break;
    default: k_bdiag_rotate<T, 8><<<grid, 256, 0, st>>>(n, width, sb, X, ldx, C_dev, Y, ldy, beta); break;
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

template int bdiag_dots<float>(int, int, int, const float*, const float*, long, DevBuf&, double*, cudaStream_t);
template int bdiag_dots<double>(int, int, int, const double*, const double*, long, DevBuf&, double*, cudaStream_t);
template int bdiag_rotate<float>(int, int, int, const float*, long, const double*, float*, long, double, cudaStream_t);
template int bdiag_rotate<double>(int, int, int, const double*, long, const double*, double*, long, double,
                                  cudaStream_t);

// C (k x m, FP64 column-major) -> C^T as bf16 hi / lo rows (m rows of k, row stride ldo)
__global__ void k_split_c_t(const double* __restrict__ C, int ldc, int k, int m, __nv_bfloat16* __restrict__ hi,
                            __nv_bfloat16* __restrict__ lo, long ldo) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)k * m) return;
  const int b = (int)(i % k), j = (int)(i / k);
  const float v = (float)C[(long)j * ldc + b];
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  hi[(long)j * ldo + b] = h;
  lo[(long)j * ldo + b] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// FP64 tall-skinny rotation Out (n x m) (+)= X (n x k) C (k x m), column-major
// (X and Out grid-fastest): a CTA owns 128 grid rows x 64 columns, C and X
// staged through shared memory in k-chunks of 16, 8 x 4 outputs per thread
constexpr int RT_M = 128, RT_N = 64, RT_K = 16;
template <typename T>
__global__ void __launch_bounds__(256) k_rot_f64(int n, int m, int k, const T* __restrict__ X, long ldx,
                                                 const double* __restrict__ C, int ldc, T* __restrict__ Out,
                                                 long ldo, int accumulate) {
  __shared__ double Xs[RT_K][RT_M + 1];
  __shared__ double Cs[RT_K][RT_N + 1];
  const int g0 = blockIdx.x * RT_M, j0 = blockIdx.y * RT_N;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;    // 16 x 16 threads
  double acc[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int b0 = 0; b0 < k; b0 += RT_K) {
    for (int e = threadIdx.x; e < RT_K * RT_M; e += 256) {
      const int bb = e / RT_M, gg = e % RT_M;
      const int b = b0 + bb, g = g0 + gg;
      Xs[bb][gg] = (b < k && g < n) ? (double)X[(long)b * ldx + g] : 0.0;
    }
    for (int e = threadIdx.x; e < RT_K * RT_N; e += 256) {
      const int bb = e % RT_K, jj = e / RT_K;
      const int b = b0 + bb, j = j0 + jj;
      Cs[bb][jj] = (b < k && j < m) ? C[(long)j * ldc + b] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int bb = 0; bb < RT_K; ++bb) {
      double xv[8], cv[4];
#pragma unroll
      for (int a = 0; a < 8; ++a) xv[a] = Xs[bb][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) cv[b] = Cs[bb][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(xv[a], cv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int j = j0 + ty + 16 * b;
    if (j >= m) continue;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int g = g0 + tx + 16 * a;
      if (g < n) {
        T* o = Out + (long)j * ldo + g;
        *o = (T)(accumulate ? (double)*o + acc[a][b] : acc[a][b]);
      }
    }
  }
}

// FP32 rotation on the split-BF16 tensor-core GEMM: X^T split into bf16 hi / lo
// rows (grid-major, K = k bands), C^T likewise, Out^T written grid-fastest
static int rotate_tc(pw_ctx* c, int n, int m, const RotBlock& B, float* out, long ldo, int accumulate,
                     cudaStream_t st) {
  const int k = B.k;
  const long kp = (k + 7) / 8 * 8;
  int rc;
  if ((rc = c->s_rot_x.alloc((size_t)2 * n * kp * 2)) || (rc = c->s_rot.alloc((size_t)2 * m * kp * 2))) return rc;
  char* xh = (char*)c->s_rot_x.p;
  char* xl = xh + (size_t)n * kp * 2;
  char* ch = (char*)c->s_rot.p;
  char* cl = ch + (size_t)m * kp * 2;
  { Launch L_(c, st, KK_MISC);
  if ((rc = split_bf16_t((const float*)B.X, B.ldx, n, k, xh, xl, kp, st))) return rc; }
  { Launch L_(c, st, KK_MISC);
  const long tot = (long)k * m;
  k_split_c_t<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(B.C, B.ldc, k, m, (__nv_bfloat16*)ch,
                                                             (__nv_bfloat16*)cl, kp);
  PWB_CUDA(cudaGetLastError()); }
  SplitOperand A{xh, xl, n, kp};
  SplitOperand Bo{ch, cl, m, kp};
  Launch L_(c, st, KK_ROT);
  return gemm_tn_store(A, Bo, k, c->gemm_terms, out, ldo, accumulate, st, 1, 0);
}

int rotate(pw_ctx* c, int n, int m, const RotBlock* blocks, int nblk, void* out, long ldo, double beta, cudaStream_t st,
           bool exact) {
  PWB_CHECK(beta == 0.0 || beta == 1.0, PW_EINVAL, "rotation: beta must be 0 or 1");
  for (int b = 0; b < nblk; ++b) {
    const RotBlock& B = blocks[b];
    if (B.k == 0) continue;
    const int acc = (b == 0) ? (beta != 0.0) : 1;
    int rc;
    if (c->prec == PW_F64 || exact) {
      // FP64 accumulation (FP32 contexts: FP32 storage, the one-off products
      // that need more than the split-BF16 accuracy, e.g. the ACE vectors)
      dim3 grid((n + RT_M - 1) / RT_M, (m + RT_N - 1) / RT_N);
      Launch L_(c, st, KK_ROT);
      if (c->prec == PW_F64)
        k_rot_f64<double><<<grid, 256, 0, st>>>(n, m, B.k, (const double*)B.X, B.ldx, B.C, B.ldc, (double*)out, ldo,
                                                acc);
      else
        k_rot_f64<float><<<grid, 256, 0, st>>>(n, m, B.k, (const float*)B.X, B.ldx, B.C, B.ldc, (float*)out, ldo,
                                               acc);
      PWB_CUDA(cudaGetLastError());
    } else {
      if ((rc = rotate_tc(c, n, m, B, (float*)out, ldo, acc, st))) return rc;
    }
  }
  return PW_OK;
}

int Dense::init(cublasHandle_t b) {
  blas = b;
  return info.alloc(64);
}
void Dense::release() {}

// eigenvectors (in A) and ascending eigenvalues by the library's kernels
// (smalldense.cu): tridiagonal reduction, multisection and inverse iteration
// up to n = 2048 where the rows fit in shared memory, cyclic Jacobi beyond
int Dense::syevd(int n, double* A, int lda, double* w, cudaStream_t st) {
  return dense_syevh(n, A, lda, w, work, st);
}

int Dense::potrf_upper(int n, double* A, int lda, cudaStream_t st) {
  int rc = dense_potrf_upper(n, A, lda, (int*)info.p, st);
  if (rc) return rc;
  int hinfo = 0;
  PWB_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  PWB_CHECK(hinfo == 0, PW_ENUMERIC, "Cholesky factorisation of the Gram matrix failed");
  return PW_OK;
}

__global__ void k_sym_upper(int n, double* A, int lda) {
  const int j = blockIdx.x;
  for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(long)j * lda + i] = A[(long)i * lda + j];
}
// column j of an n x n column-major block: strict lower part zero (mode 0), or
// the identity (mode 1)
__global__ void k_tri_fill(int n, double* A, int lda, int mode) {
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (mode == 1) A[(long)j * lda + i] = (i == j) ? 1.0 : 0.0;
    else if (i > j) A[(long)j * lda + i] = 0.0;
  }
}
int dense_sym_upper(int n, double* A, int lda, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_sym_upper<<<n, 128, 0, st>>>(n, A, lda);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
int dense_zero_lower(int n, double* A, int lda, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_tri_fill<<<n, 128, 0, st>>>(n, A, lda, 0);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
int dense_identity(int n, double* A, int lda, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_tri_fill<<<n, 128, 0, st>>>(n, A, lda, 1);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}
// A(i,j) *= s[i] * s[j]  (s device)
__global__ void k_scale_sym(int n, double* A, int lda, const double* s, int both) {
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) A[(long)j * lda + i] *= s[i] * (both ? s[j] : 1.0);
}

int solve_gen_eig(Dense& d, int lda, int numCol, int width, double* A, double* B, double* eig_host, int* numKeepOut,
                  cudaStream_t st) {
  // symmetrise (lower <- upper), eig(B)
  k_sym_upper<<<numCol, 128, 0, st>>>(numCol, A, lda);
  k_sym_upper<<<numCol, 128, 0, st>>>(numCol, B, lda);
  int rc;
  if ((rc = d.wvec.alloc((size_t)lda * 8 * 3))) return rc;
  double* sig = (double*)d.wvec.p;
  double* inv = sig + lda;
  double* eigs = inv + lda;
  if ((rc = d.syevd(numCol, B, lda, sig, st))) return rc;
  std::vector<double> hs(numCol);
  PWB_CUDA(cudaMemcpyAsync(hs.data(), sig, numCol * 8, cudaMemcpyDeviceToHost, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  int numKeep = 0;
  for (int i = numCol - 1; i >= 0; --i) {
    if (hs[i] / hs[numCol - 1] > 1e-8) numKeep++;
    else break;
  }
  PWB_CHECK(numKeep >= width, PW_ENUMERIC, "there are not enough number of columns (SolveGenEig)");
  std::vector<double> hinv(numKeep);
  for (int i = 0; i < numKeep; ++i) hinv[i] = 1.0 / std::sqrt(hs[i + numCol - numKeep]);
  PWB_CUDA(cudaMemcpyAsync(inv, hinv.data(), numKeep * 8, cudaMemcpyHostToDevice, st));
  // Atilde = U_k^T A U_k
  if ((rc = d.tmp1.alloc((size_t)lda * lda * 8))) return rc;
  double* T1 = (double*)d.tmp1.p;
  const double* Uk = B + (long)(numCol - numKeep) * lda;
  if ((rc = dense_gemm(0, 0, numCol, numKeep, numCol, A, lda, Uk, lda, T1, lda, st)) ||
      (rc = dense_gemm(1, 0, numKeep, numKeep, numCol, Uk, lda, T1, lda, A, lda, st)))
    return rc;
  k_scale_sym<<<numKeep, 128, 0, st>>>(numKeep, A, lda, inv, 1);
  if ((rc = d.syevd(numKeep, A, lda, eigs, st))) return rc;
  PWB_CUDA(cudaMemcpyAsync(eig_host, eigs, width * 8, cudaMemcpyDeviceToHost, st));
  k_scale_sym<<<numKeep, 128, 0, st>>>(numKeep, A, lda, inv, 0);
  // C = U_k * Z'
  if ((rc = dense_gemm(0, 0, numCol, numKeep, numKeep, Uk, lda, A, lda, T1, lda, st))) return rc;
  PWB_CUDA(cudaMemcpy2DAsync(A, (size_t)lda * 8, T1, (size_t)lda * 8, (size_t)numCol * 8, numKeep,
                             cudaMemcpyDeviceToDevice, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  if (numKeepOut) *numKeepOut = numKeep;
  return PW_OK;
}

}  // namespace pwb
