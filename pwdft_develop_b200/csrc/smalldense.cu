// Small dense FP64 algebra of the block eigensolvers on the device, written
// for this library (the reference calls LAPACK on its rank 0):
//   * upper Cholesky A = U^T U (EigenSolver::Orthogonalize's Potrf,
//     src/EigenSolver/eigensolver.cpp:301-384), blocked right-looking:
//     one CTA factors the diagonal block and solves its panel row, a grid of
//     CTAs applies the rank-32 update to the trailing upper triangle;
//   * the inverse of an upper-triangular U (the Trsm of Orthogonalize applied
//     to the identity), one CTA per column, column-oriented back substitution;
//   * the symmetric eigen-decomposition (Syevd of SolveGenEig and of the final
//     Rayleigh-Ritz, eigensolver.cpp:133-299, lobpcg.cpp) by cyclic two-sided
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
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < b; ++j) {
    if (threadIdx.x == 0) {
      const double d = D[j][j];
      if (!(d > 0.0)) bad = k0 + j + 1;
      else D[j][j] = sqrt(d);
    }
    __syncthreads();
    if (bad) break;
    const double ujj = D[j][j];
    for (int c = j + 1 + threadIdx.x; c < b; c += blockDim.x) D[j][c] /= ujj;
    __syncthreads();
    for (int t = threadIdx.x; t < b * b; t += blockDim.x) {
      const int i = t % b, c = t / b;
      if (i > j && i <= c) D[i][c] -= D[j][i] * D[j][c];
    }
    __syncthreads();
  }
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

int dense_potrf_upper(int n, double* A, int lda, int* info_dev, cudaStream_t st) {
  PWB_CUDA(cudaMemsetAsync(info_dev, 0, sizeof(int), st));
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
__global__ void __launch_bounds__(256) k_trtri_upper(int n, const double* U, int ldu, double* Ui, int ldi) {
  extern __shared__ double x[];
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (i == j) ? 1.0 : 0.0;
  __syncthreads();
  for (int l = j; l >= 0; --l) {
    const double xl = x[l] / U[(long)l * ldu + l];
    __syncthreads();
    if (threadIdx.x == 0) x[l] = xl;
    for (int i = threadIdx.x; i < l; i += blockDim.x) x[i] -= U[(long)l * ldu + i] * xl;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) Ui[(long)j * ldi + i] = (i <= j) ? x[i] : 0.0;
}

int dense_trtri_upper(int n, const double* U, int ldu, double* Ui, int ldi, cudaStream_t st) {
  if (n <= 0) return PW_OK;
  k_trtri_upper<<<n, 256, (size_t)n * 8, st>>>(n, U, ldu, Ui, ldi);
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

int dense_gemm(int ta, int tb, int m, int n, int k, const double* A, int lda, const double* B, int ldb, double* C,
               int ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0) return PW_OK;
  dim3 grid((m + 31) / 32, (n + 31) / 32);
  k_dgemm_small<<<grid, 256, 0, st>>>(ta, tb, m, n, k, A, lda, B, ldb, C, ldc);
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
