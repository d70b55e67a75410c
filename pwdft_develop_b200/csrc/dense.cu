// Grid-reduction Gram products and subspace operations for the block
// eigensolvers (EigenSolver::Orthogonalize, SolveGenEig, LOBPCG / PPCG
// Gram blocks: src/EigenSolver/eigensolver.cpp:133-384, lobpcg.cpp:683-874).
// FP32 contexts use the split-BF16 tcgen05 GEMMs, FP64 contexts FP64 GEMMs.
#include <cublas_v2.h>

#include <algorithm>

#include "common.hpp"
#include "blockops.hpp"
#include "gemm.hpp"

using namespace pwb;

namespace pwb {

// G (nx x ny, column-major, ldg, double, device) = X^T Y over the first nrow
// grid rows (nrow < 0: the whole coarse grid)
int gram(pw_ctx* c, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G, int ldg,
         cudaStream_t st, int nrow = -1) {
  const int nt = nrow >= 0 ? nrow : (int)c->ntot;
  if (nx == 0 || ny == 0) return PW_OK;
  if (c->prec == PW_F64) {
    cublasHandle_t h = (cublasHandle_t)c->blas;
    cublasSetStream(h, st);
    const double one = 1.0, zero = 0.0;
    c->lib_launches++;
    if (cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nx, ny, nt, &one, (const double*)X, ldx, (const double*)Y, ldy, &zero,
                    G, ldg) != CUBLAS_STATUS_SUCCESS) {
      set_error("FP64 Gram GEMM failed");
      return PW_ECUDA;
    }
    return PW_OK;
  }
  int rc;
  const bool same = (X == Y && ldx == ldy && nx == ny);
  // split rows padded to a multiple of 8 elements (16-byte TMA strides; the
  // tensor maps cover K = nt, so the pad is never read)
  const long ntp = (nt + 7) / 8 * 8;
  const size_t bx = (size_t)nx * ntp * 2, by = (size_t)ny * ntp * 2;
  if ((rc = c->s_gx_bf.alloc(2 * bx)) || (!same && (rc = c->s_gy_bf.alloc(2 * by)))) return rc;
  char* xb = (char*)c->s_gx_bf.p;
  char* yb = same ? xb : (char*)c->s_gy_bf.p;
  {
    Launch L_(c, st, KK_MISC);
    if ((rc = split_bf16((const float*)X, ldx, nt, nx, xb, xb + bx, ntp, 1.0f, st))) return rc;
  }
  if (!same) {
    Launch L_(c, st, KK_MISC);
    if ((rc = split_bf16((const float*)Y, ldy, nt, ny, yb, yb + by, ntp, 1.0f, st))) return rc;
  }
  SplitOperand A{xb, xb + bx, nx, ntp};
  SplitOperand B{yb, yb + (same ? bx : by), ny, ntp};
  ReduceOut ro;
  ro.out = G;
  ro.ldo = ldg;
  ro.f64 = 1;
  ro.transpose = 1;    // G[j*ldg + i] = sum_g X[i][g] Y[j][g]
  c->launches += 1;   // the reduction kernel; the GEMM is counted by L_
  Launch L_(c, st, KK_GRAM);
  return gemm_tn_reduce(A, B, nt, c->gemm_terms, c->s_ws, ro, st, 0, same ? 1 : 0);
}

}  // namespace pwb

extern "C" {

int pw_gram(pw_ctx* ctx, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G, int ldg,
            void* stream) {
  PWB_CHECK(ctx && (nx == 0 || X) && (ny == 0 || Y) && (nx * ny == 0 || G), PW_EINVAL, "null argument");
  PWB_CHECK(ldx >= ctx->ntot && ldy >= ctx->ntot && ldg >= nx, PW_EINVAL, "bad leading dimension");
  PWB_CUDA(cudaSetDevice(ctx->device));
  int rc = gram(ctx, X, ldx, nx, Y, ldy, ny, G, ldg, (cudaStream_t)stream);
  if (rc) return rc;
  if (ctx->check_errors) return gemm_error_check();
  return PW_OK;
}

int pw_gram_rows(pw_ctx* ctx, int nrow, const void* X, int ldx, int nx, const void* Y, int ldy, int ny, double* G,
                 int ldg, void* stream) {
  PWB_CHECK(ctx && nrow >= 0 && (nx == 0 || X) && (ny == 0 || Y) && (nx * ny == 0 || G), PW_EINVAL, "null argument");
  PWB_CHECK(ldx >= nrow && ldy >= nrow && ldg >= nx, PW_EINVAL, "bad leading dimension");
  PWB_CHECK(ctx->prec == PW_F64 || (nrow % 8 == 0 && ldx % 8 == 0 && ldy % 8 == 0), PW_EINVAL,
            "FP32 row blocks: row count and leading dimensions must be multiples of 8 (16-byte tensor rows)");
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (nrow == 0) {
    for (int j = 0; j < ny; ++j) PWB_CUDA(cudaMemsetAsync(G + (size_t)j * ldg, 0, (size_t)nx * 8, (cudaStream_t)stream));
    return PW_OK;
  }
  int rc = gram(ctx, X, ldx, nx, Y, ldy, ny, G, ldg, (cudaStream_t)stream, nrow);
  if (rc) return rc;
  if (ctx->check_errors) return gemm_error_check();
  return PW_OK;
}

int pw_rotate_rows(pw_ctx* ctx, int nrow, const void* X, int ldx, int k, const double* C, int ldc, int m, void* Out,
                   int ldo, int accumulate, void* stream) {
  PWB_CHECK(ctx && nrow >= 0 && k >= 0 && m >= 0 && (k * m == 0 || (X && C && Out)), PW_EINVAL, "null argument");
  PWB_CHECK(ldx >= nrow && ldo >= nrow && ldc >= k, PW_EINVAL, "bad leading dimension");
  PWB_CUDA(cudaSetDevice(ctx->device));
  if (m == 0 || nrow == 0) return PW_OK;
  if (k == 0) {
    if (!accumulate)
      PWB_CUDA(cudaMemset2DAsync(Out, (size_t)ldo * ctx->esz, 0, (size_t)nrow * ctx->esz, m, (cudaStream_t)stream));
    return PW_OK;
  }
  RotBlock rb{X, ldx, k, C, ldc};
  int rc = rotate(ctx, nrow, m, &rb, 1, Out, ldo, accumulate ? 1.0 : 0.0, (cudaStream_t)stream);
  if (rc) return rc;
  if (ctx->check_errors) return gemm_error_check();
  return PW_OK;
}

int pw_rotate(pw_ctx* ctx, const void* X, int ldx, int k, const double* C, int ldc, int m, void* Out, int ldo,
              int accumulate, void* stream) {
  PWB_CHECK(ctx, PW_EINVAL, "null argument");
  PWB_CHECK(ldx >= ctx->ntot && ldo >= ctx->ntot, PW_EINVAL, "bad leading dimension");
  return pw_rotate_rows(ctx, (int)ctx->ntot, X, ldx, k, C, ldc, m, Out, ldo, accumulate, stream);
}

}  // extern "C"
