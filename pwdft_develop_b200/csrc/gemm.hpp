// Split-BF16 tensor-core GEMM interface (see gemm.cu).
#pragma once
#include "common.hpp"

namespace pwb {

// A K-major operand already split into bf16 hi / lo arrays: `rows` rows of
// K elements with row stride `ld` (elements, multiple of 8).
struct SplitOperand {
  const void* hi;
  const void* lo;
  int rows;
  long ld;
};

// Destination of a split-K reduction: out[m][n] (or [n][m] if transpose),
// scaled by row_scale[m] * col_scale[n] when given; optionally also written as
// a bf16 hi/lo pair (for chaining into another GEMM).
struct ReduceOut {
  void* out = nullptr;
  long ldo = 0;
  int f64 = 0;
  int transpose = 0;
  const float* row_scale = nullptr;
  const float* col_scale = nullptr;
  void* bf_hi = nullptr;
  void* bf_lo = nullptr;
  long ldb = 0;
};

int split_bf16(const float* x, long ld_in, int ncol, int nrow, void* hi, void* lo, long ld_out, float scale,
               cudaStream_t st);
int split_bf16_t(const float* x, long ld_in, int ncol, int nrow, void* hi, void* lo, long ld_out, cudaStream_t st);
// C[m][n] = sum_k A[m][k] B[n][k] with split-K and a deterministic reduction
// bn: tile width override (0 = heuristic; otherwise one of 32, 64, 96, 128, 160, 192, 256)
// sym: A and B are the same operand (a symmetric product): only the tiles not
// strictly below the diagonal are computed, the reduction mirrors the rest
int gemm_tn_reduce(const SplitOperand& A, const SplitOperand& B, int K, int nterms, DevBuf& ws, const ReduceOut& out,
                   cudaStream_t st, int bn = 0, int sym = 0);
// C[m*ldc + n] (+)= sum_k A[m][k] B[n][k]  (K small); with transposed = 1
// the tile is written as C[n*ldc + m] (coalesced when M is the long dimension)
int gemm_tn_store(const SplitOperand& A, const SplitOperand& B, int K, int nterms, float* C, long ldc, int accumulate,
                  cudaStream_t st, int transposed = 0, int bn = 0);
// PW_ETIMEOUT (and clears the flag) if a GEMM pipeline wait gave up
int gemm_error_check();
// limit of the GEMM pipeline waits on the current device (drain waits keep >= 2 s)
int set_wait_limit_ns(unsigned long long ns);
// a bounded wait that nothing releases: PW_ETIMEOUT after limit_ns, the context stays usable
int wait_probe(unsigned long long limit_ns, cudaStream_t st);

}  // namespace pwb
