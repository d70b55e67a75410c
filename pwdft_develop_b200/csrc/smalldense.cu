// Small dense FP64 algebra of the block eigensolvers on the device, written
// for this library (the reference calls LAPACK on its rank 0):
//   * upper Cholesky A = U^T U (EigenSolver::Orthogonalize's Potrf,
//     src/EigenSolver/eigensolver.cpp:301-384): in one CTA with the matrix in
//     shared memory up to n = 160; beyond, blocked right-looking: one CTA
//     factors the diagonal block and solves its panel row, a grid of CTAs
//     applies the rank-32 update to the trailing upper triangle;
//   * the inverse of an upper-triangular U (the Trsm of Orthogonalize applied
//     to the identity), one CTA per column, column-oriented back substitution;
//   * the symmetric eigen-decomposition (Syevd of SolveGenEig and of the final
//     Rayleigh-Ritz, eigensolver.cpp:133-299, lobpcg.cpp): up to n = 160
//     through the tridiagonal form (below), beyond that by cyclic two-sided
//     Jacobi in one CTA: round-robin pairings, all n/2 rotations of a round at
//     once (2 x 2 block updates J_i^T A_ij J_j), the working matrix in shared
//     memory when it fits, eigenvectors accumulated in global memory, then a
//     rank sort to ascending order; a batched variant solves many tiny
//     problems (the PPCG sub-block Rayleigh-Ritz) with one CTA each;
//   * C = op(A) op(B) for the small n x n products of SolveGenEig.
// All kernels run on the caller's stream; status flags stay on the device
// until the caller reads them.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <utility>

#include "blockops.hpp"
#include "common.hpp"

namespace pwb {

constexpr int CHOL_NB = 32;

// ---------------------------------------------------------------------------
// Cholesky
// ---------------------------------------------------------------------------
// factor the diagonal block [k0, k1) and solve the panel row U(k0:k1, k1:n) =
// U_kk^{-T} A(k0:k1, k1:n); info <- first failing column + 1
__global__ void __launch_bounds__(256) k_chol_panel(int n, double* A, int lda, int k0, int* info) {
  __shared__ double D[CHOL_NB][CHOL_NB + 1];
  const int k1 = min(n, k0 + CHOL_NB), b = k1 - k0;
  if (*info) return;
  for (int t = threadIdx.x; t < b * b; t += blockDim.x) {
    const int i = t % b, j = t / b;
    D[i][j] = (i <= j) ? A[(long)(k0 + j) * lda + k0 + i] : 0.0;
  }
  __syncthreads();
  __shared__ int bad;
  // the diagonal block by warp 0 alone (lane c owns column c): no block-wide
  // barrier inside the factorisation
  if (threadIdx.x < 32) {
    const int c = threadIdx.x;
    int fail = 0;
    for (int j = 0; j < b; ++j) {
      const double djj = D[j][j];
      if (!(djj > 0.0)) { fail = k0 + j + 1; break; }
      const double ujj = sqrt(djj);
      __syncwarp();
      if (c == j) D[j][j] = ujj;
      if (c > j && c < b) D[j][c] /= ujj;
      __syncwarp();
      if (c > j && c < b) {
        const double ujc = D[j][c];
        for (int i = j + 1; i <= c; ++i) D[i][c] -= D[j][i] * ujc;
      }
      __syncwarp();
    }
    if (c == 0) bad = fail;
  }
  __syncthreads();
  if (bad) {
    if (threadIdx.x == 0) *info = bad;
    return;
  }
  for (int t = threadIdx.x; t < b * b; t += blockDim.x) {
    const int i = t % b, j = t / b;
    if (i <= j) A[(long)(k0 + j) * lda + k0 + i] = D[i][j];
  }
  // panel row: for each column c >= k1, forward substitution with U_kk^T
  for (int c = k1 + threadIdx.x; c < n; c += blockDim.x) {
    double x[CHOL_NB];
    double* col = A + (long)c * lda + k0;
#pragma unroll
    for (int i = 0; i < CHOL_NB; ++i) {
      if (i < b) {
        double s = col[i];
        for (int l = 0; l < i; ++l) s -= D[l][i] * x[l];
        x[i] = s / D[i][i];
      }
    }
#pragma unroll
    for (int i = 0; i < CHOL_NB; ++i)
      if (i < b) col[i] = x[i];
  }
}

// trailing update A(i, c) -= sum_l U(l, i) U(l, c) over the panel rows l, for
// k1 <= i <= c < n; one 32 x 32 tile of the upper triangle per CTA
__global__ void __launch_bounds__(256) k_chol_update(int n, double* A, int lda, int k0, const int* info) {
  if (*info) return;
  const int k1 = min(n, k0 + CHOL_NB), b = k1 - k0;
  const int nt = (n - k1 + 31) / 32;
  // blockIdx.x enumerates the upper-triangle tiles (ti <= tj)
  int t = blockIdx.x, ti = 0;
  while (t >= nt - ti) { t -= nt - ti; ++ti; }
  const int tj = ti + t;
  const int r0 = k1 + 32 * ti, c0 = k1 + 32 * tj;
  __shared__ double Ui[CHOL_NB][33], Uc[CHOL_NB][33];
  for (int e = threadIdx.x; e < CHOL_NB * 32; e += blockDim.x) {
    const int l = e / 32, x = e % 32;
    Ui[l][x] = (l < b && r0 + x < n) ? A[(long)(r0 + x) * lda + k0 + l] : 0.0;
    Uc[l][x] = (l < b && c0 + x < n) ? A[(long)(c0 + x) * lda + k0 + l] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int x = e % 32, y = e / 32;      // row r0 + x, column c0 + y
    const int i = r0 + x, c = c0 + y;
    if (i < n && c < n && i <= c) {
      double s = 0;
#pragma unroll 8
      for (int l = 0; l < CHOL_NB; ++l) s += Ui[l][x] * Uc[l][y];
      A[(long)c * lda + i] -= s;
    }
  }
}

// the whole factorisation in one CTA for n <= CHOL1_NMAX, the upper triangle
// in shared memory: per column one barrier after the scaled row is formed and
// one after the trailing update (warp per row, upper part only)
constexpr int CHOL1_NMAX = 160;
__global__ void __launch_bounds__(1024) k_chol_small(int n, double* A, int lda, int* info) {
  extern __shared__ __align__(16) double cs[];
  const int P = n | 1;
  double* W = cs;                  // W[i P + j] = A(i, j), i <= j
  double* r = W + (size_t)n * P;   // row k of U
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    if (i <= j) W[i * P + j] = A[(long)j * lda + i];
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double dkk = W[k * P + k];
    if (!(dkk > 0.0)) {
      if (tid == 0) *info = k + 1;
      return;
    }
    const double ukk = sqrt(dkk), inv = 1.0 / ukk;
    for (int j = k + tid; j < n; j += blockDim.x) {
      const double x = (j == k) ? ukk : W[k * P + j] * inv;
      r[j] = x;
      W[k * P + j] = x;
    }
    __syncthreads();
    for (int i = k + 1 + wid; i < n; i += nw) {
      const double ri = r[i];
      double* wr = W + i * P;
      for (int j = i + lane; j < n; j += 32) wr[j] -= ri * r[j];
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    if (i <= j) A[(long)j * lda + i] = W[i * P + j];
  }
}

int dense_potrf_upper(int n, double* A, int lda, int* info_dev, cudaStream_t st) {
  PWB_CUDA(cudaMemsetAsync(info_dev, 0, sizeof(int), st));
  if (n <= CHOL1_NMAX) {
    static PerDeviceOnce attr;
    const size_t smax = ((size_t)CHOL1_NMAX * (CHOL1_NMAX | 1) + CHOL1_NMAX) * sizeof(double);
    if (!attr.done()) {
      PWB_CUDA(cudaFuncSetAttribute(k_chol_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
      attr.mark();
    }
    if (n > 0)
      k_chol_small<<<1, 1024, ((size_t)n * (n | 1) + n) * sizeof(double), st>>>(n, A, lda, info_dev);
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }
  for (int k0 = 0; k0 < n; k0 += CHOL_NB) {
    k_chol_panel<<<1, 256, 0, st>>>(n, A, lda, k0, info_dev);
    const int k1 = std::min(n, k0 + CHOL_NB);
    if (k1 < n) {
      const int nt = (n - k1 + 31) / 32;
      k_chol_update<<<nt * (nt + 1) / 2, 256, 0, st>>>(n, A, lda, k0, info_dev);
    }
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// ---------------------------------------------------------------------------
// Ui = U^{-1} for an upper-triangular U: column j solves U x = e_j
// ---------------------------------------------------------------------------
// one warp per column (8 columns per CTA), x in the warp's shared row; only
// warp-level synchronisation.  STAGE: U (n <= TRTRI_NSTAGE) is first copied
// into shared memory with its diagonal inverted, so the steps read no global
// memory and divide nowhere
constexpr int TRTRI_WARPS = 8;
constexpr int TRTRI_NSTAGE = 160;
template <bool STAGE>
__global__ void __launch_bounds__(32 * TRTRI_WARPS) k_trtri_upper(int n, const double* U, int ldu, double* Ui, int ldi) {
  extern __shared__ double xs[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int j = blockIdx.x * TRTRI_WARPS + wl;
  double* x = xs + (size_t)wl * n;
  double* us = xs + (size_t)TRTRI_WARPS * n;     // STAGE: U column-major, ld n, 1/U(l,l) on the diagonal
  if constexpr (STAGE) {
    const int jmax = min(n - 1, (int)(blockIdx.x * TRTRI_WARPS + TRTRI_WARPS - 1));
    for (int idx = threadIdx.x; idx < (jmax + 1) * n; idx += blockDim.x) {
      const int l = idx / n, i = idx - l * n;
      const double u = i <= l ? U[(long)l * ldu + i] : 0.0;
      us[idx] = (i == l) ? 1.0 / u : u;
    }
    __syncthreads();
  }
  if (j >= n) return;
  for (int i = lane; i < n; i += 32) x[i] = (i == j) ? 1.0 : 0.0;
  __syncwarp();
  for (int l = j; l >= 0; --l) {
    const double* ul = STAGE ? us + (size_t)l * n : U + (long)l * ldu;
    const double xl = STAGE ? x[l] * ul[l] : x[l] / ul[l];
    __syncwarp();
    if (lane == 0) x[l] = xl;
    for (int i = lane; i < l; i += 32) x[i] -= ul[i] * xl;
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) Ui[(long)j * ldi + i] = (i <= j) ? x[i] : 0.0;
}

int dense_trtri_upper(int n, const double* U, int ldu, double* Ui, int ldi, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  static PerDeviceOnce attr;
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_trtri_upper<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    PWB_CUDA(cudaFuncSetAttribute(k_trtri_upper<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    attr.mark();
  }
  const int nblk = (n + TRTRI_WARPS - 1) / TRTRI_WARPS;
  if (n <= TRTRI_NSTAGE) {
    const size_t sm = ((size_t)TRTRI_WARPS * n + (size_t)n * n) * 8;
    k_trtri_upper<true><<<nblk, 32 * TRTRI_WARPS, sm, st>>>(n, U, ldu, Ui, ldi);
  } else {
    const size_t sm = (size_t)TRTRI_WARPS * n * 8;
    PWB_CHECK(sm <= 227 * 1024, PW_EUNSUPPORTED, "triangular inverse: n too large");
    k_trtri_upper<false><<<nblk, 32 * TRTRI_WARPS, sm, st>>>(n, U, ldu, Ui, ldi);
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// ---------------------------------------------------------------------------
// small GEMM: C (m x n) = op(A) op(B), FP64, column-major; 32 x 32 tiles
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dgemm_small(int ta, int tb, int m, int n, int k, const double* A, int lda,
                                                     const double* B, int ldb, double* C, int ldc) {
  __shared__ double As[32][33], Bs[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;   // 8 rows of threads
  double acc[4] = {0, 0, 0, 0};
  for (int l0 = 0; l0 < k; l0 += 32) {
    for (int r = ty; r < 32; r += 8) {
      // As[ii][ll] = op(A)(i0 + ii, l0 + ll); Bs[ll][jj] = op(B)(l0 + ll, j0 + jj)
      {
        const int ii = ta ? r : tx, ll = ta ? tx : r;
        const int gi = i0 + ii, gl = l0 + ll;
        double v = 0;
        if (gi < m && gl < k) v = ta ? A[(long)gi * lda + gl] : A[(long)gl * lda + gi];
        As[ii][ll] = v;
      }
      {
        const int ll = tb ? r : tx, jj = tb ? tx : r;
        const int gl = l0 + ll, gj = j0 + jj;
        double v = 0;
        if (gl < k && gj < n) v = tb ? B[(long)gl * ldb + gj] : B[(long)gj * ldb + gl];
        Bs[ll][jj] = v;
      }
    }
    __syncthreads();
#pragma unroll 8
    for (int ll = 0; ll < 32; ++ll) {
      const double a = As[tx][ll];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += a * Bs[ll][ty + 8 * q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = i0 + tx, j = j0 + ty + 8 * q;
    if (i < m && j < n) C[(long)j * ldc + i] = acc[q];
  }
}

// the same product for m, n >= 64: 64 x 64 tiles, 16-deep k steps, each
// thread 4 x 4 outputs (rows ti + 16 a, columns tj + 16 b: the tile reads are
// one 128-byte row of A and a broadcast of B per warp)
__global__ void __launch_bounds__(256) k_dgemm_t64(int ta, int tb, int m, int n, int k, const double* A, int lda,
                                                   const double* B, int ldb, double* C, int ldc) {
  __shared__ double As[16][65], Bs[16][65];
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  const int t = threadIdx.x, ti = t % 16, tj = t / 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int l0 = 0; l0 < k; l0 += 16) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = t + 256 * q;
      {
        // As[l][i] = op(A)(i0 + i, l0 + l), the contiguous index on the fastest threads
        const int i = ta ? idx / 16 : idx % 64, l = ta ? idx % 16 : idx / 64;
        const int gi = i0 + i, gl = l0 + l;
        double v = 0.0;
        if (gi < m && gl < k) v = ta ? A[(long)gi * lda + gl] : A[(long)gl * lda + gi];
        As[l][i] = v;
      }
      {
        // Bs[l][j] = op(B)(l0 + l, j0 + j)
        const int j = tb ? idx % 64 : idx / 16, l = tb ? idx / 64 : idx % 16;
        const int gl = l0 + l, gj = j0 + j;
        double v = 0.0;
        if (gl < k && gj < n) v = tb ? B[(long)gl * ldb + gj] : B[(long)gj * ldb + gl];
        Bs[l][j] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < 16; ++l) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[l][ti + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[l][tj + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int j = j0 + tj + 16 * b;
    if (j >= n) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = i0 + ti + 16 * a;
      if (i < m) C[(long)j * ldc + i] = acc[a][b];
    }
  }
}

int dense_gemm(int ta, int tb, int m, int n, int k, const double* A, int lda, const double* B, int ldb, double* C,
               int ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0) return PW_OK;
  // the 64-wide tiles where their grid still covers the SMs (n = 480: 64 CTAs
  // of 64 x 64 leave most SMs idle and run no faster than 225 of 32 x 32)
  if (m >= 64 && n >= 64 && (long)((m + 63) / 64) * ((n + 63) / 64) >= 128) {
    dim3 grid((m + 63) / 64, (n + 63) / 64);
    k_dgemm_t64<<<grid, 256, 0, st>>>(ta, tb, m, n, k, A, lda, B, ldb, C, ldc);
  } else {
    dim3 grid((m + 31) / 32, (n + 31) / 32);
    k_dgemm_small<<<grid, 256, 0, st>>>(ta, tb, m, n, k, A, lda, B, ldb, C, ldc);
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

// ---------------------------------------------------------------------------
// Jacobi eigen-decomposition
// ---------------------------------------------------------------------------
// position -> index of the round-robin tournament of m (even) players, round r
__device__ __forceinline__ int rr_index(int pos, int r, int m) { return pos == 0 ? 0 : ((pos - 1 + r) % (m - 1)) + 1; }

// One CTA brings the m x m working matrix W (ldw = m; for odd n the last row
// and column are a zero dummy that never rotates) to diagonal form.  A pair
// (p, q) rotates when |W_pq| > tol * scale.  The rotations are not applied to
// the eigenvector matrix here: each round's (c, s) pairs go to `log`
// (round-major, np per round), and k_jacobi_vectors replays them on the rows
// of V afterwards, all rows in parallel.  Returns the sweeps run.
__device__ int jacobi_cta(int m, double* W, double2* log, int* sp, int* sq, double* sc, double* ss, int max_sweeps,
                          double tol, double scale) {
  const int np = m / 2;
  __shared__ int rotated;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < m - 1; ++r) {
      for (int k = threadIdx.x; k < np; k += blockDim.x) {
        int a = rr_index(k, r, m), b = rr_index(m - 1 - k, r, m);
        if (a > b) { const int t = a; a = b; b = t; }
        double c = 1.0, s = 0.0;
        const double apq = W[(long)b * m + a];
        if (fabs(apq) > tol * scale) {
          const double app = W[(long)a * m + a], aqq = W[(long)b * m + b];
          const double theta = (aqq - app) / (2.0 * apq);
          const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
          rotated = 1;
        }
        sp[k] = a;
        sq[k] = b;
        sc[k] = c;
        ss[k] = s;
        log[((long)sweep * (m - 1) + r) * np + k] = make_double2(c, s);
      }
      __syncthreads();
      // 2 x 2 blocks (bi <= bj) of W' = J^T W J
      for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
        const int bi = e % np, bj = e / np;
        if (bj < bi) continue;
        const double si = ss[bi], sj = ss[bj];
        if (si == 0.0 && sj == 0.0) continue;
        const int p = sp[bi], q = sq[bi], r2 = sp[bj], s2 = sq[bj];
        const double ci = sc[bi], cj = sc[bj];
        if (bi == bj) {
          const double apq = W[(long)q * m + p];
          const double t = si / ci;
          W[(long)p * m + p] -= t * apq;
          W[(long)q * m + q] += t * apq;
          W[(long)q * m + p] = 0.0;
          W[(long)p * m + q] = 0.0;
          continue;
        }
        const double apr = W[(long)r2 * m + p], aps = W[(long)s2 * m + p];
        const double aqr = W[(long)r2 * m + q], aqs = W[(long)s2 * m + q];
        // (M J_j), then J_i^T (M J_j); J = [[c, s], [-s, c]] on (p, q)
        const double t1 = cj * apr - sj * aps, t2 = sj * apr + cj * aps;
        const double t3 = cj * aqr - sj * aqs, t4 = sj * aqr + cj * aqs;
        const double npr = ci * t1 - si * t3, nps = ci * t2 - si * t4;
        const double nqr = si * t1 + ci * t3, nqs = si * t2 + ci * t4;
        W[(long)r2 * m + p] = npr;
        W[(long)s2 * m + p] = nps;
        W[(long)r2 * m + q] = nqr;
        W[(long)s2 * m + q] = nqs;
        W[(long)p * m + r2] = npr;
        W[(long)p * m + s2] = nps;
        W[(long)q * m + r2] = nqr;
        W[(long)q * m + s2] = nqs;
      }
      __syncthreads();
    }
    if (!rotated) break;
  }
  return min(sweep + 1, max_sweeps);
}

constexpr int JAC_THREADS = 1024;
constexpr int JAC_SMEM_MAX = 160;   // working matrix in shared memory up to m = 160 (FP64)
constexpr int JAC_MAX_SWEEPS = 40;

size_t syevj_smem(int n) {
  const int m = n + (n & 1), np = m / 2;
  size_t b = (size_t)2 * np * sizeof(int) + (size_t)2 * np * sizeof(double) + 16;
  b = (b + 15) / 16 * 16;
  if (m <= JAC_SMEM_MAX) b += (size_t)m * m * sizeof(double);
  return b;
}
// doubles of global workspace: the working matrix when it does not fit shared
// memory, the rotation log, the ranks
size_t syevj_ws(int n) {
  const int m = n + (n & 1), np = m / 2;
  return (size_t)m * m + (size_t)2 * JAC_MAX_SWEEPS * (m - 1) * np + (size_t)m;
}

// A (n x n, lda; the upper triangle is read, as syevd's UPLO = U): the
// eigenvalues ascending into w, their ranks and the rotation log into ws
__global__ void __launch_bounds__(JAC_THREADS) k_syevj(int n, const double* A, int lda, double* w, double* ws,
                                                       int* sweeps_out, double tol) {
  extern __shared__ __align__(16) unsigned char jsm_raw[];
  const int m = n + (n & 1), np = m / 2;
  double* sc = reinterpret_cast<double*>(jsm_raw);
  double* ss = sc + np;
  int* sp = reinterpret_cast<int*>(ss + np);
  int* sq = sp + np;
  double* wsm = reinterpret_cast<double*>(jsm_raw + (((size_t)2 * np * 8 + (size_t)2 * np * 4 + 16 + 15) / 16 * 16));
  double* W = (m <= JAC_SMEM_MAX) ? wsm : ws;
  double2* log = reinterpret_cast<double2*>(ws + (size_t)m * m);
  int* rank = reinterpret_cast<int*>(ws + (size_t)m * m + (size_t)2 * JAC_MAX_SWEEPS * (m - 1) * np);
  __shared__ double red[JAC_THREADS / 32];
  double f2 = 0;
  for (long e = threadIdx.x; e < (long)m * m; e += blockDim.x) {
    const int r = (int)(e % m), c = (int)(e / m);
    double v = 0.0;
    if (r < n && c < n) v = r <= c ? A[(long)c * lda + r] : A[(long)r * lda + c];
    W[e] = v;
    f2 += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) f2 += __shfl_xor_sync(0xffffffffu, f2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f2;
  __syncthreads();
  __shared__ double scale;
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    scale = sqrt(t);
  }
  __syncthreads();
  const int sw = jacobi_cta(m, W, log, sp, sq, sc, ss, JAC_MAX_SWEEPS, tol, scale);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double di = W[(long)i * m + i];
    int rk = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = W[(long)j * m + j];
      rk += (dj < di) || (dj == di && j < i);
    }
    w[rk] = di;
    rank[i] = rk;
  }
  if (threadIdx.x == 0) *sweeps_out = sw;
}

// V = J_1 J_2 ... from the rotation log, one warp per row of V (a row starts
// as e_row); columns written to A in ascending eigenvalue order
__global__ void __launch_bounds__(256) k_jacobi_vectors(int n, double* A, int lda, const double* ws,
                                                        const int* sweeps_in) {
  extern __shared__ double rows[];
  const int m = n + (n & 1), np = m / 2;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int row = blockIdx.x * (blockDim.x >> 5) + wid;
  double* v = rows + (size_t)wid * m;
  const double2* log = reinterpret_cast<const double2*>(ws + (size_t)m * m);
  const int* rank = reinterpret_cast<const int*>(ws + (size_t)m * m + (size_t)2 * JAC_MAX_SWEEPS * (m - 1) * np);
  if (row >= n) return;
  for (int i = lane; i < m; i += 32) v[i] = (i == row) ? 1.0 : 0.0;
  __syncwarp();
  const int nsteps = *sweeps_in * (m - 1);
  for (int st = 0; st < nsteps; ++st) {
    const int r = st % (m - 1);
    const double2* lg = log + (long)st * np;
    for (int k = lane; k < np; k += 32) {
      const double2 cs = lg[k];
      if (cs.y == 0.0) continue;
      int a = rr_index(k, r, m), b = rr_index(m - 1 - k, r, m);
      if (a > b) { const int t = a; a = b; b = t; }
      const double vp = v[a], vq = v[b];
      v[a] = cs.x * vp - cs.y * vq;
      v[b] = cs.y * vp + cs.x * vq;
    }
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) A[(long)rank[i] * lda + row] = v[i];
}

// ---------------------------------------------------------------------------
// Symmetric eigen-decomposition through the tridiagonal form (n <= TRD_NMAX):
//   1. Householder reduction A = Q T Q^T in one CTA, the matrix in shared
//      memory (lower form: reflector k zeroes column k below the subdiagonal,
//      H_k = I - tau_k v_k v_k^T with v_k(k+1) = 1), two barriers per column;
//   2. all eigenvalues of T by multisection on Sturm counts: one warp per
//      eigenvalue counts at 32 points of its bracket per step (a step shrinks
//      the bracket 33-fold; 11 steps reach the rounding level);
//   3. eigenvectors of T by inverse iteration with each computed eigenvalue
//      as the shift (LU of T - lambda I with partial pivoting), three solves
//      per vector, each followed by Gram-Schmidt against the earlier vectors
//      of its cluster (neighbours closer than 1e-8 ||T||), one warp per
//      cluster, then two Loewdin steps on all vectors (described with the
//      large form below);
//   4. X = Q Z: the reflectors applied to the columns of Z, 16 threads per
//      column, no block-wide synchronisation.
// About 8/3 n^3 flops against ~60 n^3 for ten Jacobi sweeps, and the
// sequential parts (a reflector step, a tridiagonal solve) cost O(n) each.
// ---------------------------------------------------------------------------
constexpr int TRD_THREADS = 1024;   // 32 warps: the reduction's row map assumes it
constexpr int TRD_NMAX = 160;
constexpr int TRD_RPW = (TRD_NMAX + 31) / 32;   // rows of a step per warp
constexpr int TRD_WARPS_STEIN = 4;

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// sum over the block, returned to every thread (two barriers; red holds 32)
__device__ double block_sum_d(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum_d(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0;
  for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

// workspace (doubles): V [n n] reflectors (column k), Z [n n] eigenvectors of
// T, d [n], e [n], tau [n], the eigenvalues in block order lam [n], then 3 n
// ints (in 2 n doubles): the first row of each row's block, one past its last
// row, and the ascending rank of each block-ordered eigenvalue
__host__ __device__ inline size_t trd_ws(int n) { return (size_t)2 * n * n + 6 * (size_t)n; }
struct TrdAux {
  double* lam;
  int* bs;
  int* be;
  int* rank;
};
__host__ __device__ inline TrdAux trd_aux(double* ws, int n) {
  double* lam = ws + 2 * (size_t)n * n + 3 * (size_t)n;
  int* ib = reinterpret_cast<int*>(lam + n);
  return TrdAux{lam, ib, ib + n, ib + 2 * n};
}

__global__ void __launch_bounds__(TRD_THREADS) k_trd_reduce(int n, const double* A, int lda, double* ws) {
  extern __shared__ __align__(16) double trd_sm[];
  const int P = n | 1;
  double* W = trd_sm;                  // W[i P + j] = A(i, j), full symmetric
  double* p = W + (size_t)n * P;       // tau A v of the current step
  double* zrow = p + n;                // a row of zeros: the rows of a warp past n point here
  double* V = ws;
  double* d = ws + 2 * (size_t)n * n;
  double* e = d + n;
  double* tau = e + n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int idx = tid; idx < n * n; idx += blockDim.x) {
    const int i = idx / n, j = idx - i * n;
    W[i * P + j] = i <= j ? A[(long)j * lda + i] : A[(long)i * lda + j];
    V[idx] = 0.0;
  }
  for (int j = tid; j < n; j += blockDim.x) zrow[j] = 0.0;
  __syncthreads();
  // Step k, two barriers.  Every warp forms the reflector of row k (= column
  // k, the matrix stays symmetric) itself: its lanes hold v at the columns
  // j_t = k+1+lane+32t, and v at its own rows i_m = k+1+wid+32m.  The warps
  // then form p = tau A22 v on their rows (barrier), and each warp the update
  // A22 -= v w^T + w v^T on its rows with w = p - (tau/2)(p.v) v formed from p
  // in registers (barrier).
  for (int k = 0; k + 2 < n; ++k) {
    const double* rk = W + k * P;
    double vj[TRD_RPW];
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < TRD_RPW; ++t) {
      const int j = k + 1 + lane + 32 * t;
      const double x = j < n ? rk[j] : 0.0;
      vj[t] = x;
      if (j >= k + 2) s += x * x;
    }
    s = warp_sum_d(s);
    const double alpha = rk[k + 1];
    double tk = 0.0, beta = alpha, scal = 0.0;
    if (s != 0.0) {
      const double mu = sqrt(alpha * alpha + s);
      beta = alpha <= 0.0 ? mu : -mu;
      tk = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
#pragma unroll
    for (int t = 0; t < TRD_RPW; ++t) {
      const int j = k + 1 + lane + 32 * t;
      vj[t] = j == k + 1 ? 1.0 : vj[t] * scal;
    }
    if (wid == 0) {
#pragma unroll
      for (int t = 0; t < TRD_RPW; ++t) {
        const int j = k + 1 + lane + 32 * t;
        if (j < n) V[(long)k * n + j] = vj[t];
      }
      if (lane == 0) {
        d[k] = rk[k];
        e[k] = beta;
        tau[k] = tk;
      }
    }
    if (tk == 0.0) continue;          // nothing to update; W is unchanged (every warp agrees)
    double* wr[TRD_RPW];
    double vi[TRD_RPW];
#pragma unroll
    for (int m = 0; m < TRD_RPW; ++m) {
      const int i = k + 1 + wid + 32 * m;
      wr[m] = i < n ? W + i * P : zrow;
      vi[m] = i < n ? (i == k + 1 ? 1.0 : rk[i] * scal) : 0.0;
    }
    // p = tau A22 v on the warp's rows, the row sums interleaved
    {
      double acc[TRD_RPW];
#pragma unroll
      for (int m = 0; m < TRD_RPW; ++m) acc[m] = 0.0;
#pragma unroll
      for (int t = 0; t < TRD_RPW; ++t) {
        const int j = k + 1 + lane + 32 * t;
        if (j < n) {
#pragma unroll
          for (int m = 0; m < TRD_RPW; ++m) acc[m] += wr[m][j] * vj[t];
        }
      }
#pragma unroll
      for (int m = 0; m < TRD_RPW; ++m) acc[m] = warp_sum_d(acc[m]);
      if (lane == 0) {
#pragma unroll
        for (int m = 0; m < TRD_RPW; ++m) {
          const int i = k + 1 + wid + 32 * m;
          if (i < n) p[i] = tk * acc[m];
        }
      }
    }
    __syncthreads();
    // w = p - (tau/2)(p.v) v, then A22 -= v w^T + w v^T on the warp's rows
    {
      double pj[TRD_RPW];
      double t2 = 0.0;
#pragma unroll
      for (int t = 0; t < TRD_RPW; ++t) {
        const int j = k + 1 + lane + 32 * t;
        pj[t] = j < n ? p[j] : 0.0;
        t2 += pj[t] * vj[t];
      }
      const double kc = 0.5 * tk * warp_sum_d(t2);
      double wi[TRD_RPW];
#pragma unroll
      for (int m = 0; m < TRD_RPW; ++m) {
        const int i = k + 1 + wid + 32 * m;
        wi[m] = i < n ? p[i] - kc * vi[m] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < TRD_RPW; ++t) {
        const int j = k + 1 + lane + 32 * t;
        if (j < n) {
          const double wj = pj[t] - kc * vj[t];
#pragma unroll
          for (int m = 0; m < TRD_RPW; ++m) wr[m][j] -= vi[m] * wj + wi[m] * vj[t];
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = W[(n - 2) * P + n - 2];
      e[n - 2] = W[(n - 1) * P + n - 2];
      tau[n - 2] = 0.0;
    }
    d[n - 1] = W[(n - 1) * P + n - 1];
    tau[n - 1] = 0.0;
  }
}

// 1/q by two Newton-Raphson steps, r <- r (2 - q r) (quadratic convergence),
// from the hardware's approximate reciprocal (q stays a finite normal number:
// the Sturm pivots are kept between pivmin >= the smallest normal double and
// 1e300 in magnitude)
__device__ __forceinline__ double recip_nr(double q) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
  r = r * fma(-q, r, 2.0);
  r = r * fma(-q, r, 2.0);
  return r;
}

// number of eigenvalues of T below x: negative pivots of the LDL^T
// factorisation of T - x I (Sturm sequence in ratio form), pivots kept off
// zero by pivmin
__device__ __forceinline__ int trd_sturm(int n, const double* d, const double* e2, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q <= 0.0;
  for (int j = 1; j < n; ++j) {
    q = (d[j] - x) - e2[j - 1] * recip_nr(q);
    if (fabs(q) < pivmin) q = -pivmin;
    c += q <= 0.0;
    q = fmin(fmax(q, -1e300), 1e300);   // keep q finite for the reciprocal (an overflow counts by its sign)
  }
  return c;
}

// T splits where an off-diagonal is negligible, |e_i| <= eps (|d_i| +
// |d_i+1|) (set to zero; the eigenvalues move by at most eps ||T||): the
// blocks' eigenvectors have disjoint supports, so degenerate eigenvalues of
// different blocks (an identity-like overlap matrix splits into 1 x 1 blocks)
// need no orthogonalisation against each other.  One CTA of TRD_SPLIT_T
// threads, n <= 2 TRD_SPLIT_T: bs[r] (the block's first row) is the running
// maximum of the block starts up to r, be[r] (one past its last row) the
// running minimum of the block ends from r on, both by scans in shared memory.
constexpr int TRD_SPLIT_T = 1024;
__global__ void __launch_bounds__(TRD_SPLIT_T) k_trd_split(int n, double* ws) {
  __shared__ int st[2 * TRD_SPLIT_T], en[2 * TRD_SPLIT_T];
  double* d = ws + 2 * (size_t)n * n;
  double* e = d + n;
  const TrdAux ax = trd_aux(ws, n);
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const bool cut = r + 1 == n || fabs(e[r]) <= 2.3e-16 * (fabs(d[r]) + fabs(d[r + 1]));
    // row r + 1 starts a block when r ends one
    en[r] = cut ? r + 1 : n;
    if (r + 1 < n) st[r + 1] = cut ? r + 1 : 0;
    if (r == 0) st[0] = 0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r + 1 < n; r += blockDim.x)
    if (en[r] == r + 1) e[r] = 0.0;
  // inclusive max-scan of st (forward) and min-scan of en (backward)
  for (int off = 1; off < n; off <<= 1) {
    int a[2], b[2];
    for (int q = 0; q < 2; ++q) {
      const int r = threadIdx.x + q * blockDim.x;
      a[q] = (r < n && r >= off) ? max(st[r], st[r - off]) : (r < n ? st[r] : 0);
      b[q] = (r < n && r + off < n) ? min(en[r], en[r + off]) : (r < n ? en[r] : n);
    }
    __syncthreads();
    for (int q = 0; q < 2; ++q) {
      const int r = threadIdx.x + q * blockDim.x;
      if (r < n) {
        st[r] = a[q];
        en[r] = b[q];
      }
    }
    __syncthreads();
  }
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    ax.bs[r] = st[r];
    ax.be[r] = en[r];
  }
}

// eigenvalues by blocks: warp g finds eigenvalue g - bs[g] of the block of row
// g (lam[g]; ascending within each block), its 32 lanes counting at 32
// interior points of the bracket per step (33-fold shrink: 11 steps reach the
// rounding level); T's diagonal and squared off-diagonal in shared memory,
// the Gershgorin interval of the whole T recomputed by every CTA
constexpr int TRD_BIS_WARPS = 4;
constexpr int TRD_BIS_STEPS = 11;
__global__ void __launch_bounds__(32 * TRD_BIS_WARPS) k_trd_bisect(int n, double* ws) {
  extern __shared__ __align__(16) double bis_sm[];   // 2 n doubles
  double* sd = bis_sm;
  double* se2 = bis_sm + n;
  __shared__ double s_gl, s_gu, s_pivmin;
  const double* d = ws + 2 * (size_t)n * n;
  const double* e = d + n;
  const TrdAux ax = trd_aux(ws, n);
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < n; i += blockDim.x) {
    sd[i] = d[i];
    se2[i] = i + 1 < n ? e[i] * e[i] : 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    double gl = 1e300, gu = -1e300, emax = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
      gl = fmin(gl, sd[i] - r);
      gu = fmax(gu, sd[i] + r);
      emax = fmax(emax, se2[i]);
    }
    const double tn = fmax(fabs(gl), fabs(gu));
    s_gl = gl - 2.3e-16 * tn * n - 1e-300;
    s_gu = gu + 2.3e-16 * tn * n + 1e-300;
    s_pivmin = 2.3e-308 * fmax(1.0, emax);
  }
  __syncthreads();
  const int g = blockIdx.x * TRD_BIS_WARPS + (tid >> 5);
  if (g >= n) return;
  const int b0 = ax.bs[g], m = ax.be[g] - b0, i = g - b0;
  double lo = s_gl, hi = s_gu;
  for (int step = 0; step < TRD_BIS_STEPS; ++step) {
    const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
    const int c = trd_sturm(m, sd + b0, se2 + b0, x, s_pivmin);
    // eigenvalue i of the block lies where its count passes i: count(lo) <= i < count(hi)
    double nl = c <= i ? x : lo, nh = c > i ? x : hi;
    for (int o = 16; o > 0; o >>= 1) {
      nl = fmax(nl, __shfl_xor_sync(0xffffffffu, nl, o));
      nh = fmin(nh, __shfl_xor_sync(0xffffffffu, nh, o));
    }
    lo = nl;
    hi = nh;
  }
  if (lane == 0) ax.lam[g] = 0.5 * (lo + hi);
}

// ascending rank of each block-ordered eigenvalue (ties by block order) and
// the sorted eigenvalues into w
__global__ void k_trd_rank(int n, double* ws, double* w) {
  const TrdAux ax = trd_aux(ws, n);
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const double x = ax.lam[g];
  int r = 0;
  for (int h = 0; h < n; ++h) {
    const double y = ax.lam[h];
    r += (y < x) || (y == x && h < g);
  }
  ax.rank[g] = r;
  w[r] = x;
}

__device__ __forceinline__ double trd_rand(int i, int r) {
  unsigned long long x = ((unsigned long long)(i + 1) << 32) ^ (unsigned long long)(r * 2654435761u + 12345u);
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// eigenvectors of T: one warp per cluster; lane 0 factors T - lambda I with
// partial pivoting and runs the solves, the warp orthogonalises and normalises.
// Shared memory: 6 n doubles per warp, then the cluster table (n + 2 ints).
// Clusters: neighbours closer than ortol_rel ||T||.
__global__ void __launch_bounds__(32 * TRD_WARPS_STEIN) k_trd_stein(int n, double* ws, double ortol_rel) {
  extern __shared__ __align__(16) double st_sm[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  const int g = blockIdx.x * wpc + wl;
  double* Z = ws + (size_t)n * n;
  const double* dT = ws + 2 * (size_t)n * n;
  const double* eT = dT + n;
  const TrdAux ax = trd_aux(ws, n);
  const double* w = ax.lam;
  // clusters of the block-ordered eigenvalues (every CTA scans them itself):
  // a new cluster at each block start and wherever the gap exceeds ortol
  int* clus = reinterpret_cast<int*>(st_sm + (size_t)wpc * 6 * n);
  if (threadIdx.x == 0) {
    double tn0 = 0.0;
    for (int i = 0; i < n; ++i) tn0 = fmax(tn0, fabs(dT[i]) + (i + 1 < n ? 2.0 * fabs(eT[i]) : 0.0));
    const double ortol = ortol_rel * tn0;
    int nc = 0;
    for (int i = 0; i < n; ++i)
      if (i == 0 || ax.bs[i] == i || w[i] - w[i - 1] > ortol) clus[1 + nc++] = i;
    clus[1 + nc] = n;
    clus[0] = nc;
  }
  __syncthreads();
  if (g >= clus[0]) return;
  // the cluster's block: rows [b0, b0 + nb) of T
  const int b0 = ax.bs[clus[1 + g]], nb = ax.be[clus[1 + g]] - b0;
  const double* d = dT + b0;
  const double* e = eT + b0;
  double* u = st_sm + (size_t)wl * 6 * n;
  double* s1 = u + n;
  double* s2 = s1 + n;
  double* l = s2 + n;
  double* y = l + n;
  double* sw = y + n;          // row interchange at step k (1) or not (0)
  double tn = 0.0;
  for (int i = lane; i < n; i += 32) tn = fmax(tn, fabs(dT[i]) + (i + 1 < n ? 2.0 * fabs(eT[i]) : 0.0));
  for (int o = 16; o > 0; o >>= 1) tn = fmax(tn, __shfl_xor_sync(0xffffffffu, tn, o));
  const double eps = 2.3e-16 * fmax(tn, 1e-300);
  const int c0 = clus[1 + g], c1 = clus[2 + g];
  for (int i = c0; i < c1; ++i) {
    const double lam = w[i];
    if (lane == 0) {
      // LU of the block's T - lam I with row interchanges (U: pivot u,
      // superdiagonals s1, s2; u then holds the pivots' reciprocals)
      double ak = d[0] - lam, bk = nb > 1 ? e[0] : 0.0;
      for (int k = 0; k + 1 < nb; ++k) {
        const double ck = e[k];
        double an = d[k + 1] - lam;
        const double bn = k + 2 < nb ? e[k + 1] : 0.0;
        if (fabs(ak) >= fabs(ck)) {
          if (ak == 0.0) ak = eps;
          const double m = ck / ak;
          u[k] = ak; s1[k] = bk; s2[k] = 0.0; l[k] = m; sw[k] = 0.0;
          an -= m * bk;
          ak = an;
          bk = bn;
        } else {
          const double m = ak / ck;
          u[k] = ck; s1[k] = an; s2[k] = bn; l[k] = m; sw[k] = 1.0;
          ak = bk - m * an;
          bk = -m * bn;
        }
      }
      u[nb - 1] = fabs(ak) < eps ? (ak < 0.0 ? -eps : eps) : ak;
      s1[nb - 1] = 0.0;       // read (times zero) by the register-carried back substitution
      s2[nb - 1] = 0.0;
      // the solves multiply by the pivots' reciprocals (tiny pivots raised to eps)
      for (int k = 0; k < nb; ++k) {
        const double uk = u[k];
        u[k] = 1.0 / (fabs(uk) < eps ? (uk < 0.0 ? -eps : eps) : uk);
      }
    }
    for (int r = lane; r < nb; r += 32) y[r] = trd_rand(i, b0 + r);
    __syncwarp();
    for (int it = 0; it < 3; ++it) {
      if (lane == 0) {
        // the running values stay in registers: one FMA (forward) or two
        // FMAs and a product (backward) per step on the dependency chain
        double yk = y[0];
#pragma unroll 4
        for (int k = 0; k + 1 < nb; ++k) {
          double yn = y[k + 1];
          if (sw[k] != 0.0) {
            const double t = yk;
            yk = yn;
            yn = t;
          }
          yn -= l[k] * yk;
          y[k] = yk;
          yk = yn;
        }
        y[nb - 1] = yk;
        double y1 = 0.0, y2 = 0.0;   // y[k+1], y[k+2] (zero past the end)
#pragma unroll 4
        for (int k = nb - 1; k >= 0; --k) {
          const double t = (y[k] - s1[k] * y1 - s2[k] * y2) * u[k];
          y[k] = t;
          y2 = y1;
          y1 = t;
        }
      }
      __syncwarp();
      // Gram-Schmidt against the cluster's earlier vectors (same block), then normalise
      for (int j = c0; j < i; ++j) {
        const double* zj = Z + (size_t)ax.rank[j] * n + b0;
        double dt = 0;
        for (int r = lane; r < nb; r += 32) dt += zj[r] * y[r];
        dt = warp_sum_d(dt);
        for (int r = lane; r < nb; r += 32) y[r] -= dt * zj[r];
        __syncwarp();
      }
      double nr = 0;
      for (int r = lane; r < nb; r += 32) nr += y[r] * y[r];
      nr = warp_sum_d(nr);
      const double inv = nr > 0.0 ? 1.0 / sqrt(nr) : 0.0;
      for (int r = lane; r < nb; r += 32) y[r] *= inv;
      __syncwarp();
    }
    // column rank(i) of Z: the block's rows, zero elsewhere
    double* zc = Z + (size_t)ax.rank[i] * n;
    for (int r = lane; r < n; r += 32) zc[r] = (r >= b0 && r < b0 + nb) ? y[r - b0] : 0.0;
    __syncwarp();
  }
}

// X = H_0 H_1 ... H_{n-3} Z into A's columns; 16 threads per column, the
// reflectors staged through shared memory TRD_KC at a time
constexpr int TRD_QMAX = (TRD_NMAX + 15) / 16;
constexpr int TRD_KC = 16;
__global__ void __launch_bounds__(256) k_trd_back(int n, double* A, int lda, const double* ws) {
  __shared__ double vs[TRD_KC][TRD_NMAX];
  __shared__ double ts[TRD_KC];
  const double* V = ws;
  const double* Z = ws + (size_t)n * n;
  const double* tau = ws + 2 * (size_t)n * n + 2 * (size_t)n;
  const int c = blockIdx.x * 16 + (threadIdx.x >> 4), t = threadIdx.x & 15;
  const bool act = c < n;
  double z[TRD_QMAX];
#pragma unroll
  for (int q = 0; q < TRD_QMAX; ++q) {
    const int r = t + 16 * q;
    z[q] = (act && r < n) ? Z[(size_t)c * n + r] : 0.0;
  }
  for (int kt = n - 3; kt >= 0; kt -= TRD_KC) {
    const int kb = max(0, kt - TRD_KC + 1), nk = kt - kb + 1;   // reflectors kb .. kt
    __syncthreads();
    for (int idx = threadIdx.x; idx < nk * n; idx += blockDim.x) {
      const int kk = idx / n, r = idx - kk * n;
      vs[kk][r] = V[(size_t)(kb + kk) * n + r];
    }
    if (threadIdx.x < nk) ts[threadIdx.x] = tau[kb + threadIdx.x];
    __syncthreads();
    for (int kk = nk - 1; kk >= 0; --kk) {
      const double tk = ts[kk];
      if (tk == 0.0) continue;
      const double* vk = vs[kk];
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < TRD_QMAX; ++q) {
        const int r = t + 16 * q;
        if (r < n) s += vk[r] * z[q];
      }
      for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      s *= tk;
#pragma unroll
      for (int q = 0; q < TRD_QMAX; ++q) {
        const int r = t + 16 * q;
        if (r < n) z[q] -= vk[r] * s;
      }
    }
  }
  if (!act) return;
#pragma unroll
  for (int q = 0; q < TRD_QMAX; ++q) {
    const int r = t + 16 * q;
    if (r < n) A[(long)c * lda + r] = z[q];
  }
}

// ---------------------------------------------------------------------------
// The same method for n > TRD_NMAX (LOBPCG's 3n subspace, Rayleigh-Ritz of
// several hundred bands):
//   1. the reduction runs on G co-resident CTAs (a cooperative launch), the
//      matrix held in their shared memory by rows (row i on CTA i mod G).
//      Step k: the owner of row k forms the reflector and publishes it
//      (column k of V, a release flag); every CTA forms p = tau A22 v on its
//      rows and publishes them (a counting barrier over the G CTAs, p double
//      buffered by the barrier's parity); every CTA then forms w = p - (tau/2)(p.v) v and updates its
//      rows.  One flag wait and one barrier per column, both bounded by
//      %globaltimer (TRD_WAIT_NS; on timeout the CTA records code 1 in the
//      sync record and returns).
//   2./3. multisection and inverse iteration as above, but Gram-Schmidt only
//      within clusters closer than 1e-8 ||T|| (the near-degenerate sets, where
//      independent solves may give nearly parallel vectors); every other pair
//      of computed vectors overlaps by at most ~ r / gap <= ~1e-6 (r ~ n eps
//      ||T|| the residual of a solve), and two symmetric (Loewdin) steps
//      Z <- Z (3 I - Z^T Z) / 2 make Z orthonormal to rounding.  Mixing two
//      vectors with coefficient ~ r / gap moves each residual by ~ r, so the
//      eigenpairs keep their accuracy; the 1e-3 ||T|| clusters of LAPACK's
//      inverse iteration chain into sets of hundreds of vectors at these
//      sizes (LOBPCG's overlap matrices), each solved one after another;
//   4. X = Q Z with one warp per column of Z, the column in registers, the
//      reflectors applied eight at a time in compact WY form.
// ---------------------------------------------------------------------------
constexpr int TRDL_THREADS = 512;
constexpr int TRD_NMAX_L = 2048;
constexpr unsigned long long TRD_WAIT_NS = 2000000000ull;

struct TrdSync {
  unsigned int count;   // barrier arrivals
  unsigned int vflag;   // reflectors published (k + 1 after step k)
  int err;              // 1: a wait ran out
  int pad;
};
// workspace of the large form: trd_ws(n) doubles, then p (2 n), the sync
// record (2), and two n x n blocks for the orthonormalisation of Z
size_t trd_ws_large(int n) { return trd_ws(n) + 2 * (size_t)n + 2 + 2 * (size_t)n * n; }

// M = (3 I - G) / 2 in place: one first-order step towards (Z^T Z)^{-1/2}
__global__ void k_lowdin_step(int n, double* G) {
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double g = G[(size_t)j * n + i];
    G[(size_t)j * n + i] = (i == j ? 1.5 : 0.0) - 0.5 * g;
  }
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long trd_gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// wait until *p >= target; false after TRD_WAIT_NS
__device__ bool trd_wait_geq(const unsigned int* p, unsigned int target) {
  if (ld_acquire_u32(p) >= target) return true;
  const unsigned long long t0 = trd_gtimer();
  for (;;) {
    __nanosleep(64);
    if (ld_acquire_u32(p) >= target) return true;
    if (trd_gtimer() - t0 > TRD_WAIT_NS) return false;
  }
}

__global__ void __launch_bounds__(TRDL_THREADS) k_trd_reduce_mc(int n, const double* A, int lda, double* ws) {
  extern __shared__ __align__(16) double rm_sm[];
  const int G = gridDim.x, c = blockIdx.x;
  const int nr = (n - c + G - 1) / G;      // rows c, c + G, c + 2G, ...
  double* R = rm_sm;                       // R[li n + j] = A(c + li G, j)
  double* vs = R + (size_t)nr * n;         // v of the step (entries past k)
  double* wsm = vs + n;                    // p, then w
  __shared__ double red[32];
  __shared__ int abort_s;
  double* V = ws;
  double* d = ws + 2 * (size_t)n * n;
  double* e = d + n;
  double* tau = e + n;
  double* pg = ws + trd_ws(n);             // 2 n: p, double buffered
  TrdSync* sy = reinterpret_cast<TrdSync*>(pg + 2 * (size_t)n);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < nr * n; idx += blockDim.x) {
    const int li = idx / n, j = idx - li * n;
    const int i = c + li * G;
    R[idx] = i <= j ? A[(long)j * lda + i] : A[(long)i * lda + j];
  }
  if (tid == 0) abort_s = 0;
  __syncthreads();
  unsigned int nbar = 0;
  for (int k = 0; k + 2 < n; ++k) {
    if (k % G == c && wid == 0) {
      // the owner forms the reflector of row k (= column k) and publishes it
      const double* rk = R + (size_t)(k / G) * n;
      double s = 0.0;
      for (int j = k + 2 + lane; j < n; j += 32) s += rk[j] * rk[j];
      s = warp_sum_d(s);
      const double alpha = rk[k + 1];
      double tk = 0.0, beta = alpha, scal = 0.0;
      if (s != 0.0) {
        const double mu = sqrt(alpha * alpha + s);
        beta = alpha <= 0.0 ? mu : -mu;
        tk = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      for (int j = lane; j < n; j += 32) V[(size_t)k * n + j] = j <= k ? 0.0 : (j == k + 1 ? 1.0 : rk[j] * scal);
      if (lane == 0) {
        d[k] = rk[k];
        e[k] = beta;
        tau[k] = tk;
      }
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        st_release_u32(&sy->vflag, (unsigned int)(k + 1));
      }
    }
    if (tid == 0 && !trd_wait_geq(&sy->vflag, (unsigned int)(k + 1))) {
      abort_s = 1;
      atomicExch(&sy->err, 1);
    }
    __syncthreads();
    if (abort_s) return;
    // v and tau in the same round trip (v is staged even when tau is zero)
    for (int j = k + 1 + tid; j < n; j += blockDim.x) vs[j] = __ldcg(&V[(size_t)k * n + j]);
    const double tk = __ldcg(&tau[k]);
    __syncthreads();
    if (tk == 0.0) continue;          // the same on every CTA: nothing to update
    // first local row past k
    const int li0 = k + 1 <= c ? 0 : (k + 1 - c + G - 1) / G;
    // p in half nbar & 1 (barriers completed so far): the last data in that half
    // belonged to barrier nbar - 2, read by every CTA before it arrived at nbar - 1
    double* ph = pg + (size_t)(nbar & 1) * n;
    for (int li = li0 + wid; li < nr; li += nw) {
      const double* r = R + (size_t)li * n;
      double acc = 0.0;
      for (int j = k + 1 + lane; j < n; j += 32) acc += r[j] * vs[j];
      acc = warp_sum_d(acc);
      if (lane == 0) ph[c + li * G] = tk * acc;
    }
    __syncthreads();
    ++nbar;
    if (tid == 0) {
      __threadfence();
      atomicAdd(&sy->count, 1u);
      if (!trd_wait_geq(&sy->count, nbar * (unsigned int)G)) {
        abort_s = 1;
        atomicExch(&sy->err, 1);
      }
    }
    __syncthreads();
    if (abort_s) return;
    double part = 0.0;
    for (int j = k + 1 + tid; j < n; j += blockDim.x) {
      const double pj = __ldcg(&ph[j]);
      wsm[j] = pj;
      part += pj * vs[j];
    }
    const double kc = 0.5 * tk * block_sum_d(part, red);
    for (int j = k + 1 + tid; j < n; j += blockDim.x) wsm[j] -= kc * vs[j];
    __syncthreads();
    for (int li = li0 + wid; li < nr; li += nw) {
      const int i = c + li * G;
      const double vi = vs[i], wi = wsm[i];
      double* r = R + (size_t)li * n;
      for (int j = k + 1 + lane; j < n; j += 32) r[j] -= vi * wsm[j] + wi * vs[j];
    }
    __syncthreads();
  }
  // the trailing 2 x 2 block (e from row n - 1, as in the one-CTA form)
  if (tid == 0) {
    if ((n - 2) % G == c) {
      d[n - 2] = R[(size_t)((n - 2) / G) * n + n - 2];
      tau[n - 2] = 0.0;
    }
    if ((n - 1) % G == c) {
      const double* r = R + (size_t)((n - 1) / G) * n;
      e[n - 2] = r[n - 2];
      d[n - 1] = r[n - 1];
      tau[n - 1] = 0.0;
    }
  }
}

// The reduction on one thread-block cluster (n up to ~640): the CL CTAs hold
// the rows in their shared memory (row i on CTA i mod CL) and exchange v and p
// through distributed shared memory; per column two hardware cluster barriers
// and no global round trip.  Step k: the owner of row k forms v in its own
// buffer (and writes it to V); barrier; every CTA copies v from the owner,
// forms p on its rows into its own buffer; barrier; every CTA gathers p from
// the owners of its entries, forms w and updates its rows.  A CTA rewrites
// its v / p buffers only after a later barrier that every reader of the old
// contents has passed.
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// load a double at the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ double ld_dsmem(const double* local, unsigned rank) {
  unsigned a = (unsigned)__cvta_generic_to_shared(local), ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
  return v;
}

__global__ void __launch_bounds__(TRDL_THREADS) k_trd_reduce_cl(int n, const double* A, int lda, double* ws) {
  extern __shared__ __align__(16) double rc_sm[];
  const int CL = (int)gridDim.x, c = (int)cluster_rank();
  const int nr = (n - c + CL - 1) / CL;
  // the buffers read by other CTAs sit at the same offset in every CTA (the
  // row counts differ by one between CTAs, so they come before the rows)
  double* vown = rc_sm;                    // v formed here when this CTA owns row k; vown[n] = tau
  double* vs = vown + n + 2;               // this CTA's copy of v
  double* pl = vs + n;                     // p at this CTA's rows (by global row index)
  double* wsm = pl + n;                    // p, then w, gathered
  double* R = wsm + n;                     // R[li n + j] = A(c + li CL, j)
  __shared__ double red[32];
  double* V = ws;
  double* d = ws + 2 * (size_t)n * n;
  double* e = d + n;
  double* tau = e + n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < nr * n; idx += blockDim.x) {
    const int li = idx / n, j = idx - li * n;
    const int i = c + li * CL;
    R[idx] = i <= j ? A[(long)j * lda + i] : A[(long)i * lda + j];
  }
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int own = k % CL;
    if (own == c && wid == 0) {
      const double* rk = R + (size_t)(k / CL) * n;
      double sq = 0.0;
      for (int j = k + 2 + lane; j < n; j += 32) sq += rk[j] * rk[j];
      sq = warp_sum_d(sq);
      const double alpha = rk[k + 1];
      double tk = 0.0, beta = alpha, scal = 0.0;
      if (sq != 0.0) {
        const double mu = sqrt(alpha * alpha + sq);
        beta = alpha <= 0.0 ? mu : -mu;
        tk = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      for (int j = lane; j < n; j += 32) vown[j] = j <= k ? 0.0 : (j == k + 1 ? 1.0 : rk[j] * scal);
      __syncwarp();
      if (lane == 0) {
        vown[n] = tk;
        vown[n + 1] = beta;
        // row k past the diagonal is dead after its reflector: beta and tau go there
        double* rw = R + (size_t)(k / CL) * n;
        rw[k + 1] = beta;
        rw[k + 2] = tk;
      }
    }
    cluster_sync_all();
    for (int j = k + 1 + tid; j < n; j += blockDim.x) vs[j] = ld_dsmem(vown + j, (unsigned)own);
    const double tk = ld_dsmem(vown + n, (unsigned)own);
    __syncthreads();
    // v(i) of the CTA's rows i >= k + 2 into their dead slot k (column k of V,
    // written out at the end: no global store inside the loop)
    {
      const int lk2 = k + 2 <= c ? 0 : (k + 2 - c + CL - 1) / CL;
      for (int li = lk2 + tid; li < nr; li += blockDim.x) R[(size_t)li * n + k] = vs[c + li * CL];
    }
    if (tk == 0.0) continue;          // the same on every CTA: nothing to update
    const int li0 = k + 1 <= c ? 0 : (k + 1 - c + CL - 1) / CL;
    // two rows per warp at a time (independent accumulations), four columns per lane step
    for (int li = li0 + 2 * wid; li < nr; li += 2 * nw) {
      const bool two = li + 1 < nr;
      const double* r0 = R + (size_t)li * n;
      const double* r1 = two ? r0 + n : r0;
      double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
      int j = k + 1 + lane;
      for (; j + 32 < n; j += 64) {
        const double v0 = vs[j], v1 = vs[j + 32];
        a0 += r0[j] * v0;
        b0 += r0[j + 32] * v1;
        a1 += r1[j] * v0;
        b1 += r1[j + 32] * v1;
      }
      if (j < n) {
        a0 += r0[j] * vs[j];
        a1 += r1[j] * vs[j];
      }
      a0 += b0;
      a1 += b1;
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      }
      if (lane == 0) {
        pl[c + li * CL] = tk * a0;
        if (two) pl[c + (li + 1) * CL] = tk * a1;
      }
    }
    cluster_sync_all();
    double part = 0.0;
    for (int j = k + 1 + tid; j < n; j += blockDim.x) {
      const double pj = ld_dsmem(pl + j, (unsigned)(j % CL));
      wsm[j] = pj;
      part += pj * vs[j];
    }
    const double kc = 0.5 * tk * block_sum_d(part, red);
    for (int j = k + 1 + tid; j < n; j += blockDim.x) wsm[j] -= kc * vs[j];
    __syncthreads();
    // the rank-2 update, two rows per warp at a time
    for (int li = li0 + 2 * wid; li < nr; li += 2 * nw) {
      const bool two = li + 1 < nr;
      const int i0 = c + li * CL, i1 = two ? i0 + CL : i0;
      const double v0 = vs[i0], w0 = wsm[i0], v1 = vs[i1], w1 = wsm[i1];
      double* r0 = R + (size_t)li * n;
      double* r1 = two ? r0 + n : r0;
      for (int j = k + 1 + lane; j < n; j += 32) {
        const double vj = vs[j], wj = wsm[j];
        r0[j] -= v0 * wj + w0 * vj;
        if (two) r1[j] -= v1 * wj + w1 * vj;
      }
    }
    __syncthreads();
  }
  // write out: d, e, tau of the CTA's rows and its entries of V (V(k, i) =
  // v_k(i): 0 for i <= k, 1 for i = k + 1, the stored slot beyond; e(n-2)
  // from row n - 1, as in the one-CTA form)
  for (int li = tid; li < nr; li += blockDim.x) {
    const int i = c + li * CL;
    const double* r = R + (size_t)li * n;
    d[i] = r[i];
    if (i + 2 < n) {
      e[i] = r[i + 1];
      tau[i] = r[i + 2];
    } else {
      tau[i] = 0.0;
      if (i == n - 1) e[n - 2] = r[n - 2];
    }
  }
  for (int idx = tid; idx < nr * (n - 2); idx += blockDim.x) {
    const int k = idx / nr, li = idx - k * nr;
    const int i = c + li * CL;
    V[(size_t)k * n + i] = i <= k ? 0.0 : (i == k + 1 ? 1.0 : R[(size_t)li * n + k]);
  }
  cluster_sync_all();     // no CTA leaves while another may still read its shared memory
}

// global -> shared copies that hold no register (cp.async, 8-byte elements)
__device__ __forceinline__ void cpa8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// The back-transformation in blocks of kc <= 8 reflectors (compact WY form):
// H_kb H_kb+1 ... H_kt = I - V T V^T with T upper triangular, T_ii = tau_i,
// T(0:i, i) = -tau_i T(0:i, 0:i) (V(:, 0:i)^T v_i).  Chunk c holds the
// reflectors kb .. kt with kt = n - 3 - c kc; its T goes to Tg[64 c] (8 x 8,
// T(j, i) at j * 8 + i), one CTA per chunk.
__global__ void __launch_bounds__(256) k_trd_wy_t(int n, int kc, const double* ws, double* Tg) {
  __shared__ double S[64], T[64];
  const int c = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int kt = n - 3 - c * kc, kb = max(0, kt - kc + 1), nk = kt - kb + 1;
  const double* V = ws + (size_t)kb * n;
  const double* tau = ws + 2 * (size_t)n * n + 2 * (size_t)n + kb;
  for (int e = wid; e < nk * nk; e += nw) {
    const int l = e / nk, i = e - l * nk;
    if (l > i) continue;
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc += V[(size_t)l * n + r] * V[(size_t)i * n + r];
    acc = warp_sum_d(acc);
    if (lane == 0) S[l * 8 + i] = acc;
  }
  if (threadIdx.x < 64) T[threadIdx.x] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < nk; ++i) {
      const double ti = tau[i];
      for (int j = 0; j < i; ++j) {
        double acc = 0.0;
        for (int l = j; l < i; ++l) acc += T[j * 8 + l] * S[l * 8 + i];
        T[j * 8 + i] = -ti * acc;
      }
      T[i * 8 + i] = ti;
    }
  }
  __syncthreads();
  if (threadIdx.x < 64) Tg[(size_t)c * 64 + threadIdx.x] = T[threadIdx.x];
}

// X = H_0 H_1 ... H_{n-3} Z into A's columns: one warp per column, rows
// lane + 32 q of the column in registers (QM >= n / 32).  Per chunk (from the
// last): y = V^T z (kc independent dots), u = T y, z -= V u.  The chunks are
// double-buffered in shared memory by cp.async (the next chunk's copies in
// flight while this one is applied).
// warps per CTA at most: one wave of CTAs over the SMs where the registers allow
template <int QM> constexpr int trd_back_maxw() { return QM == 48 ? 10 : 8; }
template <int QM>
__global__ void __launch_bounds__(32 * trd_back_maxw<QM>()) k_trd_back_w(int n, int kc, double* A, int lda,
                                                                         const double* ws, const double* Tg) {
  extern __shared__ __align__(16) double bw_sm[];   // two stages of kc x n reflectors + 64 (T)
  const size_t stage = (size_t)kc * n + 64;
  const double* V = ws;
  const double* Z = ws + (size_t)n * n;
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const bool act = col < n;
  const int nchunk = (n - 2 + kc - 1) / kc;    // reflectors 0 .. n - 3
  double z[QM];
#pragma unroll
  for (int q = 0; q < QM; ++q) {
    const int r = lane + 32 * q;
    z[q] = (act && r < n) ? Z[(size_t)col * n + r] : 0.0;
  }
  auto issue = [&](int c, int b) {
    const int kt = n - 3 - c * kc, kb = max(0, kt - kc + 1), nk = kt - kb + 1;
    double* dst = bw_sm + b * stage;
    const double* src = V + (size_t)kb * n;
    for (int idx = threadIdx.x; idx < nk * n; idx += blockDim.x) cpa8(dst + idx, src + idx);
    if (threadIdx.x < 64) cpa8(dst + (size_t)kc * n + threadIdx.x, Tg + (size_t)c * 64 + threadIdx.x);
  };
  issue(0, 0);
  cpa_commit();
  for (int c = 0; c < nchunk; ++c) {
    const int b = c & 1;
    if (c + 1 < nchunk) issue(c + 1, b ^ 1);
    cpa_commit();
    cpa_wait1();
    __syncthreads();
    const int kt = n - 3 - c * kc, kb = max(0, kt - kc + 1), nk = kt - kb + 1;
    const double* Vb = bw_sm + b * stage;          // Vb[l n + r] = v_{kb + l}(r)
    const double* Tb = Vb + (size_t)kc * n;
    double y[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) y[l] = 0.0;
#pragma unroll
    for (int q = 0; q < QM; ++q) {
      const int r = lane + 32 * q;
      if (r < n) {
        const double zq = z[q];
#pragma unroll
        for (int l = 0; l < 8; ++l)
          if (l < nk) y[l] += Vb[(size_t)l * n + r] * zq;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int l = 0; l < 8; ++l) y[l] += __shfl_xor_sync(0xffffffffu, y[l], o);
    }
    double u[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int l = j; l < 8; ++l)
        if (l < nk) acc += Tb[j * 8 + l] * y[l];
      u[j] = acc;
    }
#pragma unroll
    for (int q = 0; q < QM; ++q) {
      const int r = lane + 32 * q;
      if (r < n) {
        double acc = z[q];
#pragma unroll
        for (int l = 0; l < 8; ++l)
          if (l < nk) acc -= Vb[(size_t)l * n + r] * u[l];
        z[q] = acc;
      }
    }
    __syncthreads();    // the next issue refills this buffer
  }
  if (!act) return;
#pragma unroll
  for (int q = 0; q < QM; ++q) {
    const int r = lane + 32 * q;
    if (r < n) A[(long)col * lda + r] = z[q];
  }
}

// CTAs of the cooperative reduction for this n on this device (0: the rows do
// not fit in shared memory), and its dynamic shared memory
struct TrdLargePlan {
  int G = 0;
  size_t smem = 0;
};
static TrdLargePlan trd_large_plan_build(int n) {
  TrdLargePlan pl;
  if (n <= TRD_NMAX || n > TRD_NMAX_L) return pl;
  int dev = 0, nsm = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return pl;
  // one CTA per SM at most; about 16 rows per CTA where the SMs allow
  int G = std::min(nsm, std::max(1, (n + 15) / 16));
  for (;; ++G) {
    if (G > nsm) return pl;
    const int nr = (n + G - 1) / G;
    const size_t sm = ((size_t)nr * n + 2 * (size_t)n) * sizeof(double) + 1024;
    if (sm <= (size_t)optin) {
      pl.G = G;
      pl.smem = sm - 1024;
      return pl;
    }
  }
}

static TrdLargePlan trd_large_plan(int n);
bool trd_supported(int n) { return n <= TRD_NMAX || trd_large_plan(n).G > 0; }

// the cluster form: CTAs per cluster (0: not possible here) and shared memory
struct TrdClusterPlan {
  int CL = 0;
  size_t smem = 0;
};
static TrdClusterPlan trd_cluster_plan_build(int n) {
  TrdClusterPlan pl;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return pl;
  static PerDeviceOnce attr;
  if (!attr.done()) {
    if (cudaFuncSetAttribute(k_trd_reduce_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_trd_reduce_cl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return pl;
    }
    attr.mark();
  }
  for (int CL : {8, 16}) {
    const int nr = (n + CL - 1) / CL;
    const size_t sm = ((size_t)nr * n + 4 * (size_t)n + 2) * sizeof(double);
    if (sm + 1024 > (size_t)optin) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(TRDL_THREADS);
    cfg.dynamicSmemBytes = sm;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, k_trd_reduce_cl, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (ncl >= 1) {
      pl.CL = CL;
      pl.smem = sm;
      return pl;
    }
  }
  return pl;
}

// the plans per (device, n), built once (the occupancy queries cost host time)
static std::mutex g_trd_mu;
static TrdLargePlan trd_large_plan(int n) {
  static std::map<std::pair<int, int>, TrdLargePlan> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_trd_mu);
  auto it = cache.find({dev, n});
  if (it != cache.end()) return it->second;
  return cache[{dev, n}] = trd_large_plan_build(n);
}
static TrdClusterPlan trd_cluster_plan(int n) {
  static std::map<std::pair<int, int>, TrdClusterPlan> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lk(g_trd_mu);
    auto it = cache.find({dev, n});
    if (it != cache.end()) return it->second;
  }
  const TrdClusterPlan pl = trd_cluster_plan_build(n);
  std::lock_guard<std::mutex> lk(g_trd_mu);
  return cache[{dev, n}] = pl;
}

static int trd_reduce_cluster(int n, const double* A, int lda, double* wsp, const TrdClusterPlan& pl,
                              cudaStream_t st) {
  // the sync record is unused here; cleared so that trd_error reads no stale code
  PWB_CUDA(cudaMemsetAsync(wsp + trd_ws(n) + 2 * (size_t)n, 0, sizeof(TrdSync), st));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pl.CL);
  cfg.blockDim = dim3(TRDL_THREADS);
  cfg.dynamicSmemBytes = pl.smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = pl.CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  PWB_CUDA(cudaLaunchKernelEx(&cfg, k_trd_reduce_cl, n, A, lda, wsp));
  return PW_OK;
}

static int trd_reduce_large(int n, const double* A, int lda, double* wsp, cudaStream_t st) {
  {
    const TrdClusterPlan cp = trd_cluster_plan(n);
    if (cp.CL > 0) return trd_reduce_cluster(n, A, lda, wsp, cp, st);
  }
  const TrdLargePlan pl = trd_large_plan(n);
  PWB_CHECK(pl.G > 0, PW_EUNSUPPORTED, "tridiagonal reduction: n too large for shared memory");
  int optin = 0, dev = 0;
  PWB_CUDA(cudaGetDevice(&dev));
  PWB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  static PerDeviceOnce attr;
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_trd_reduce_mc, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024));
    attr.mark();
  }
  int per_sm = 0;
  PWB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trd_reduce_mc, TRDL_THREADS, pl.smem));
  PWB_CHECK(per_sm >= 1, PW_EUNSUPPORTED, "tridiagonal reduction: no resident CTA");
  TrdSync* sy = reinterpret_cast<TrdSync*>(wsp + trd_ws(n) + 2 * (size_t)n);
  PWB_CUDA(cudaMemsetAsync(sy, 0, sizeof(TrdSync), st));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pl.G);
  cfg.blockDim = dim3(TRDL_THREADS);
  cfg.dynamicSmemBytes = pl.smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  PWB_CUDA(cudaLaunchKernelEx(&cfg, k_trd_reduce_mc, n, A, lda, wsp));
  return PW_OK;
}

// Tg: at least 64 ceil((n - 2) / 8) doubles of scratch for the chunks' T
static int trd_back_large(int n, double* A, int lda, const double* wsp, double* Tg, cudaStream_t st) {
  int optin = 0, dev = 0;
  PWB_CUDA(cudaGetDevice(&dev));
  PWB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  // chunk size: two stages of kc x n reflectors (+ T) within shared memory
  const int kc = std::max(1, std::min(8, (int)(((size_t)optin / 16 - 64) / (size_t)n)));
  const int nchunk = (n - 2 + kc - 1) / kc;
  k_trd_wy_t<<<nchunk, 256, 0, st>>>(n, kc, wsp, Tg);
  // one warp per column, the columns spread over the SMs in one wave where the
  // CTA size allows (1 CTA per SM: the shared stages and the registers)
  int nsm = 148;
  PWB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int maxw = n <= 1024 ? 8 : (n <= 1536 ? 10 : 8);
  const int wpc = std::max(4, std::min(maxw, (n + nsm - 1) / nsm));
  const size_t sm = 2 * ((size_t)kc * n + 64) * sizeof(double);
  const dim3 grid((n + wpc - 1) / wpc), block(32 * wpc);
  static PerDeviceOnce attr;
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_trd_back_w<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    PWB_CUDA(cudaFuncSetAttribute(k_trd_back_w<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    PWB_CUDA(cudaFuncSetAttribute(k_trd_back_w<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    PWB_CUDA(cudaFuncSetAttribute(k_trd_back_w<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    attr.mark();
  }
  if (n <= 512) k_trd_back_w<16><<<grid, block, sm, st>>>(n, kc, A, lda, wsp, Tg);
  else if (n <= 1024) k_trd_back_w<32><<<grid, block, sm, st>>>(n, kc, A, lda, wsp, Tg);
  else if (n <= 1536) k_trd_back_w<48><<<grid, block, sm, st>>>(n, kc, A, lda, wsp, Tg);
  else k_trd_back_w<64><<<grid, block, sm, st>>>(n, kc, A, lda, wsp, Tg);
  return PW_OK;
}

// code recorded by the large reduction's waits (0: none); synchronous
int trd_error(int n, const DevBuf& ws) {
  if (n <= TRD_NMAX || !ws.p) return 0;
  TrdSync h{};
  if (cudaMemcpy(&h, (const double*)ws.p + trd_ws(n) + 2 * (size_t)n, sizeof(h), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return -1;
  return h.err;
}

int dense_syevh(int n, double* A, int lda, double* w, DevBuf& ws, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  if (!trd_supported(n)) return dense_syevj(n, A, lda, w, ws, nullptr, st);
  const bool large = n > TRD_NMAX;
  int rc;
  if ((rc = ws.alloc(trd_ws_large(n) * sizeof(double)))) return rc;
  static PerDeviceOnce attr;
  const size_t sm_red = ((size_t)TRD_NMAX * (TRD_NMAX | 1) + 2 * TRD_NMAX) * sizeof(double);
  int optin = 0, dev = 0;
  PWB_CUDA(cudaGetDevice(&dev));
  PWB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_trd_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_red));
    PWB_CUDA(cudaFuncSetAttribute(k_trd_stein, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    attr.mark();
  }
  double* wsp = (double*)ws.p;
  if (large) {
    if ((rc = trd_reduce_large(n, A, lda, wsp, st))) return rc;
  } else {
    k_trd_reduce<<<1, TRD_THREADS, ((size_t)n * (n | 1) + 2 * (size_t)n) * sizeof(double), st>>>(n, A, lda, wsp);
  }
  k_trd_split<<<1, TRD_SPLIT_T, 0, st>>>(n, wsp);
  k_trd_bisect<<<(n + TRD_BIS_WARPS - 1) / TRD_BIS_WARPS, 32 * TRD_BIS_WARPS, 2 * (size_t)n * sizeof(double), st>>>(
      n, wsp);
  k_trd_rank<<<(n + 127) / 128, 128, 0, st>>>(n, wsp, w);
  // warps per CTA of the inverse iteration: 6 n doubles each, plus the cluster table
  const size_t per_warp = 6 * (size_t)n * sizeof(double), tab = ((size_t)n + 2) * sizeof(int);
  const int wpc = (int)std::max<size_t>(1, std::min<size_t>(TRD_WARPS_STEIN, ((size_t)optin - tab) / per_warp));
  // Gram-Schmidt only inside near-degenerate sets, then two Loewdin steps (at
  // every size: the Rayleigh-Ritz matrices of symmetric cells chain their
  // 1e-3 ||T|| neighbours into long clusters even at n = 160)
  k_trd_stein<<<(n + wpc - 1) / wpc, 32 * wpc, wpc * per_warp + tab, st>>>(n, wsp, 1e-8);
  double* Gm = wsp + trd_ws(n) + 2 * (size_t)n + 2;
  {
    double* Z = wsp + (size_t)n * n;
    double* Z2 = Gm + (size_t)n * n;
    for (int pass = 0; pass < 2; ++pass) {
      double* zi = pass == 0 ? Z : Z2;
      double* zo = pass == 0 ? Z2 : Z;
      if ((rc = dense_gemm(1, 0, n, n, n, zi, n, zi, n, Gm, n, st))) return rc;
      k_lowdin_step<<<n, 128, 0, st>>>(n, Gm);
      if ((rc = dense_gemm(0, 0, n, n, n, zi, n, Gm, n, zo, n, st))) return rc;
    }
  }
  if (large) {
    if ((rc = trd_back_large(n, A, lda, wsp, Gm, st))) return rc;   // Gm is free again: the chunks' T
  } else {
    k_trd_back<<<(n + 15) / 16, 256, 0, st>>>(n, A, lda, wsp);
  }
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

int dense_syevj(int n, double* A, int lda, double* w, DevBuf& ws, int* sweeps_dev, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  const int m = n + (n & 1);
  int rc;
  if ((rc = ws.alloc((syevj_ws(n) + 2) * sizeof(double)))) return rc;
  int* sw = sweeps_dev ? sweeps_dev : reinterpret_cast<int*>((double*)ws.p + syevj_ws(n));
  static PerDeviceOnce attr;
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_syevj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)syevj_smem(JAC_SMEM_MAX)));
    attr.mark();
  }
  k_syevj<<<1, JAC_THREADS, syevj_smem(n), st>>>(n, A, lda, w, (double*)ws.p, sw, 1e-15);
  const int rows_per_cta = 8;
  k_jacobi_vectors<<<(n + rows_per_cta - 1) / rows_per_cta, 32 * rows_per_cta, (size_t)rows_per_cta * m * 8, st>>>(
      n, A, lda, (const double*)ws.p, sw);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

}  // namespace pwb

using namespace pwb;

extern "C" {

int pw_dense_potrf(pw_ctx* ctx, int n, double* A, int lda) {
  PWB_CHECK(ctx && n >= 0 && (n == 0 || A) && lda >= n, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  Dense d;
  int rc = d.init((cublasHandle_t)ctx->blas);
  if (rc) return rc;
  return n ? d.potrf_upper(n, A, lda, nullptr) : PW_OK;
}

int pw_dense_trtri(pw_ctx* ctx, int n, const double* U, int ldu, double* Ui, int ldi) {
  PWB_CHECK(ctx && n >= 0 && (n == 0 || (U && Ui)) && ldu >= n && ldi >= n, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  int rc = dense_trtri_upper(n, U, ldu, Ui, ldi, nullptr);
  if (rc) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  return PW_OK;
}

int pw_dense_syev(pw_ctx* ctx, int n, double* A, int lda, double* w, int* sweeps) {
  PWB_CHECK(ctx && n >= 0 && (n == 0 || (A && w)) && lda >= n, PW_EINVAL, "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  DevBuf ws, sw;
  int rc;
  if (trd_supported(n)) {
    if ((rc = dense_syevh(n, A, lda, w, ws, nullptr))) return rc;
    PWB_CUDA(cudaDeviceSynchronize());
    PWB_CHECK(trd_error(n, ws) == 0, PW_ETIMEOUT, "tridiagonal reduction: a wait ran out");
    if (sweeps) *sweeps = 0;
    return PW_OK;
  }
  if ((rc = sw.alloc(16))) return rc;
  if ((rc = dense_syevj(n, A, lda, w, ws, (int*)sw.p, nullptr))) return rc;
  PWB_CUDA(cudaDeviceSynchronize());
  if (sweeps) PWB_CUDA(cudaMemcpy(sweeps, sw.p, sizeof(int), cudaMemcpyDeviceToHost));
  return PW_OK;
}

int pw_solve_gen_eig(pw_ctx* ctx, int lda, int numCol, int width, double* A, double* B, double* eig, int* numKeep) {
  PWB_CHECK(ctx && A && B && eig && numCol > 0 && width > 0 && width <= numCol && lda >= numCol, PW_EINVAL,
            "bad arguments");
  PWB_CUDA(cudaSetDevice(ctx->device));
  Dense d;
  int rc = d.init((cublasHandle_t)ctx->blas);
  if (rc) return rc;
  return solve_gen_eig(d, lda, numCol, width, A, B, eig, numKeep, nullptr);
}

}  // extern "C"
