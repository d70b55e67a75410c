// Device block operations for the eigensolvers and the SCF driver.
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
template int colscale<float>(int, int, float*, long, const double*, cudaStream_t);
template int colscale<double>(int, int, double*, long, const double*, cudaStream_t);

int rotate(pw_ctx* c, int n, int m, const RotBlock* blocks, int nblk, void* out, long ldo, double beta, cudaStream_t st) {
  cublasHandle_t h = (cublasHandle_t)c->blas;
  cublasSetStream(h, st);
  for (int b = 0; b < nblk; ++b) {
    const RotBlock& B = blocks[b];
    if (B.k == 0) continue;
    const double be = (b == 0) ? beta : 1.0;
    c->lib_launches++;
    if (c->prec == PW_F64) {
      const double one = 1.0;
      if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, m, B.k, &one, (const double*)B.X, (int)B.ldx, B.C, B.ldc, &be,
                      (double*)out, (int)ldo) != CUBLAS_STATUS_SUCCESS) {
        set_error("rotation GEMM failed");
        return PW_ECUDA;
      }
    } else {
      // FP32 storage: the small FP64 coefficient block is rounded to FP32
      int rc = c->s_rot.alloc((size_t)B.k * m * 4);
      if (rc) return rc;
      float* Cf = (float*)c->s_rot.p;
      if ((rc = copy_d2f_2d(B.k, m, B.C, B.ldc, Cf, B.k, st))) return rc;
      const float one = 1.0f, bf = (float)be;
      if (cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, m, B.k, &one, (const float*)B.X, (int)B.ldx, Cf, B.k, &bf,
                      (float*)out, (int)ldo) != CUBLAS_STATUS_SUCCESS) {
        set_error("rotation GEMM failed");
        return PW_ECUDA;
      }
    }
  }
  return PW_OK;
}

int Dense::init(cublasHandle_t b) {
  blas = b;
  if (!sol && cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnCreate failed");
    return PW_ECUDA;
  }
  return info.alloc(64);
}
void Dense::release() {
  if (sol) cusolverDnDestroy(sol);
  sol = nullptr;
}

int Dense::syevd(int n, double* A, int lda, double* w, cudaStream_t st) {
  cusolverDnSetStream(sol, st);
  int lw = 0;
  if (cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, A, lda, w, &lw) !=
      CUSOLVER_STATUS_SUCCESS) {
    set_error("syevd buffer query failed");
    return PW_ECUDA;
  }
  int rc = work.alloc((size_t)std::max(lw, 1) * 8);
  if (rc) return rc;
  if (cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, A, lda, w, (double*)work.p, lw,
                       (int*)info.p) != CUSOLVER_STATUS_SUCCESS) {
    set_error("syevd failed");
    return PW_ECUDA;
  }
  int hinfo = 0;
  PWB_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  PWB_CHECK(hinfo == 0, PW_ENUMERIC, "syevd did not converge");
  return PW_OK;
}

int Dense::potrf_upper(int n, double* A, int lda, cudaStream_t st) {
  cusolverDnSetStream(sol, st);
  int lw = 0;
  if (cusolverDnDpotrf_bufferSize(sol, CUBLAS_FILL_MODE_UPPER, n, A, lda, &lw) != CUSOLVER_STATUS_SUCCESS) {
    set_error("potrf buffer query failed");
    return PW_ECUDA;
  }
  int rc = work.alloc((size_t)std::max(lw, 1) * 8);
  if (rc) return rc;
  if (cusolverDnDpotrf(sol, CUBLAS_FILL_MODE_UPPER, n, A, lda, (double*)work.p, lw, (int*)info.p) !=
      CUSOLVER_STATUS_SUCCESS) {
    set_error("potrf failed");
    return PW_ECUDA;
  }
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
  const double one = 1.0, zero = 0.0;
  cublasSetStream(d.blas, st);
  const double* Uk = B + (long)(numCol - numKeep) * lda;
  if (cublasDgemm(d.blas, CUBLAS_OP_N, CUBLAS_OP_N, numCol, numKeep, numCol, &one, A, lda, Uk, lda, &zero, T1, lda) !=
          CUBLAS_STATUS_SUCCESS ||
      cublasDgemm(d.blas, CUBLAS_OP_T, CUBLAS_OP_N, numKeep, numKeep, numCol, &one, Uk, lda, T1, lda, &zero, A, lda) !=
          CUBLAS_STATUS_SUCCESS) {
    set_error("SolveGenEig GEMM failed");
    return PW_ECUDA;
  }
  k_scale_sym<<<numKeep, 128, 0, st>>>(numKeep, A, lda, inv, 1);
  if ((rc = d.syevd(numKeep, A, lda, eigs, st))) return rc;
  PWB_CUDA(cudaMemcpyAsync(eig_host, eigs, width * 8, cudaMemcpyDeviceToHost, st));
  k_scale_sym<<<numKeep, 128, 0, st>>>(numKeep, A, lda, inv, 0);
  // C = U_k * Z'
  if (cublasDgemm(d.blas, CUBLAS_OP_N, CUBLAS_OP_N, numCol, numKeep, numKeep, &one, Uk, lda, A, lda, &zero, T1, lda) !=
      CUBLAS_STATUS_SUCCESS) {
    set_error("SolveGenEig GEMM failed");
    return PW_ECUDA;
  }
  PWB_CUDA(cudaMemcpy2DAsync(A, (size_t)lda * 8, T1, (size_t)lda * 8, (size_t)numCol * 8, numKeep,
                             cudaMemcpyDeviceToDevice, st));
  PWB_CUDA(cudaStreamSynchronize(st));
  if (numKeepOut) *numKeepOut = numKeep;
  return PW_OK;
}

}  // namespace pwb
