// Device block operations used by the eigensolvers and the SCF driver.
#pragma once
#include <cublas_v2.h>

#include "common.hpp"

namespace pwb {

// Y = a*X + b*Y for nb columns of length n (column stride ldx / ldy)
template <typename T> int axpby(int n, int nb, double a, const T* X, long ldx, double b, T* Y, long ldy, cudaStream_t st);
// Z = a*X + b*Y + c*W (three blocks, element-wise), used by the Chebyshev recurrence
template <typename T>
int axpbypcz(int n, int nb, double a, const T* X, double b, const T* Y, double c, const T* W, T* Z, long ld,
             cudaStream_t st);
// out[j] = sum_i X[j*ld + i]^2 (double)
template <typename T> int colnorm2(int n, int nb, const T* X, long ld, double* out, cudaStream_t st);
// X[:, j] *= s[j]
template <typename T> int colscale(int n, int nb, T* X, long ld, const double* s, cudaStream_t st);
// B = alpha A (m x n column-major FP64, B may be A); v <- 1 / sqrt(v) (0 where v <= 1e-300); residual norms
// out[k] = sqrt(nrm2[k]) / max(1, |G(k, k)|) with their maximum in out[n]
int dense_scale(int m, int n, double alpha, const double* A, int lda, double* B, int ldb, cudaStream_t st);
int vec_rsqrt(int n, double* v, cudaStream_t st);
int resnorms(int n, const double* nrm2, const double* G, int ldg, double* out, cudaStream_t st);
// copy with precision change
int copy_d2f(long n, const double* x, float* y, cudaStream_t st);
int copy_f2d(long n, const float* x, double* y, cudaStream_t st);
int copy_d2f_2d(int n, int nb, const double* x, long ldx, float* y, long ldy, cudaStream_t st);
int copy_f2d_2d(int n, int nb, const float* x, long ldx, double* y, long ldy, cudaStream_t st);

// Z = c[0] HY + c[1] Y (+ c[2] X when X is given); c device-resident (3 doubles)
template <typename T>
int cheb_lin(int n, int nb, const double* coef_dev, const T* HY, const T* Y, const T* X, T* Z, long ld,
             cudaStream_t st);

// Diagonal sb x sb blocks of U^T V (width columns, grid length n) for the PPCG
// sub-block sweep: out_host[k * sb * sb + i + j * sb], k < ceil(width / sb),
// FP64, summed over grid-point splits in a fixed order.  sb in 1..8.
template <typename T>
int bdiag_dots(int n, int width, int sb, const T* U, const T* V, long ld, DevBuf& part, double* out_host,
               cudaStream_t st);
// The same sums into a device array out_dev[k * sb * sb + i + j * sb]
template <typename T>
int bdiag_dots_dev(int n, int width, int sb, const T* U, const T* V, long ld, DevBuf& part, double* out_dev,
                   cudaStream_t st);
// PPCG sub-block eigenproblems on the device from the twelve sub-block Gram
// arrays (xax, waw, xaw, xx, ww, xw, pap, xap, wap, pp, xp, wp; the last six
// unused when numSet = 2) into the coefficient blocks Cx, Cw, Cp
int ppcg_subblock_solve(int width, int sb, int numSet, const double* const* grams, double* Cx, double* Cw, double* Cp,
                        cudaStream_t st);
// Y (+)= X * blockdiag(C_k): Y[:, k*sb + j] = beta Y + sum_i X[:, k*sb + i] C[k*sb*sb + i + j*sb]
template <typename T>
int bdiag_rotate(int n, int width, int sb, const T* X, long ldx, const double* C_dev, T* Y, long ldy, double beta,
                 cudaStream_t st);

// Out (n x m, ldo) = sum over blocks of X_b (n x k_b, ld) * C_b (k_b x m, FP64 column-major, ldc),
// beta = 0 or 1 for Out.  The context precision decides FP64 or FP32 storage of X / Out.
struct RotBlock {
  const void* X;
  long ldx;
  int k;
  const double* C;   // device, FP64
  int ldc;
};
// exact: FP64 accumulation also in FP32 contexts (otherwise FP32 contexts use
// the split-BF16 tensor-core GEMM)
int rotate(pw_ctx* c, int n, int m, const RotBlock* blocks, int nblk, void* out, long ldo, double beta, cudaStream_t st,
           bool exact = false);

// Small dense FP64 algebra on the device with this library's kernels
// (smalldense.cu), n up to a few thousand.
struct Dense {
  cublasHandle_t blas = nullptr;
  DevBuf work, info, tmp1, tmp2, tmp3, wvec;
  int init(cublasHandle_t b);
  void release();
  // eigen-decomposition in place: A (n x n, lda; upper triangle read) -> eigenvectors, w (device) ascending
  int syevd(int n, double* A, int lda, double* w, cudaStream_t st);
  // upper Cholesky A = U^T U in place; returns PW_ENUMERIC if not positive definite
  int potrf_upper(int n, double* A, int lda, cudaStream_t st);
};

// smalldense.cu: blocked upper Cholesky (info_dev: 0, or the failing column + 1),
// inverse of an upper-triangular matrix (strict lower part of Ui zeroed),
// C = op(A) op(B) (ta / tb: 1 = transposed), Jacobi eigen-decomposition (ws:
// workspace, sweeps_dev may be NULL)
int dense_potrf_upper(int n, double* A, int lda, int* info_dev, cudaStream_t st);
int dense_trtri_upper(int n, const double* U, int ldu, double* Ui, int ldi, cudaStream_t st);
int dense_gemm(int ta, int tb, int m, int n, int k, const double* A, int lda, const double* B, int ldb, double* C,
               int ldc, cudaStream_t st);
int dense_syevj(int n, double* A, int lda, double* w, DevBuf& ws, int* sweeps_dev, cudaStream_t st);
// the same result through the tridiagonal form (Householder reduction,
// multisection on Sturm counts, inverse iteration) for n <= 160; larger n
// fall back to dense_syevj
int dense_syevh(int n, double* A, int lda, double* w, DevBuf& ws, cudaStream_t st);

// n x n column-major blocks on the device, queued on st: lower part from the
// upper triangle, strict lower part zeroed, identity
int dense_sym_upper(int n, double* A, int lda, cudaStream_t st);
int dense_zero_lower(int n, double* A, int lda, cudaStream_t st);
int dense_identity(int n, double* A, int lda, cudaStream_t st);

// Symmetric generalized eigenproblem of EigenSolver::SolveGenEig (serial path,
// src/EigenSolver/eigensolver.cpp:224-297): symmetrise from the upper triangle,
// eig(B), keep sigma/sigma_max > 1e-8, eig of the reduced A, C = U sigma^-1/2 Z.
// On exit A holds C (numCol x numKeep), eig (host) the first `width` values.
int solve_gen_eig(Dense& d, int lda, int numCol, int width, double* A, double* B, double* eig_host, int* numKeep,
                  cudaStream_t st);

}  // namespace pwb
