// 3-D FFT of the fine grid, one axis per launch (FP64 for the Hartree
// potential and its gradient; FP64 or FP32 for the sphere-cut exchange).
#pragma once
#include "fft.cuh"

namespace pwb {

// 16 pencils per CTA
constexpr int AX_TILE = 16;
constexpr int AX_THREADS = 256;

// axis 0 (x, contiguous): CTA = 16 consecutive rows; axis 1 (y): CTA = (z, x tile);
// axis 2 (z): CTA = (y, x tile, field blockIdx.z).  A batch of F fields stored
// back to back runs as one launch: nz * F planes for axes 0 and 1 (nz = N * F
// for axis 0, gridDim.y = nz * F for axis 1), gridDim.z = F for axis 2, whose
// multiplier kern (MODE 2 / 4) is the same nx * ny * nz array for every field.  MODE 0: plain, 1: real input (load re(x) -
// y_sub), 2: multiply by kern after the forward transform and inverse in place,
// 3: store the real part scaled into out, 4: as 2 with the multiplier i * kern
// (a spectral derivative).
// T (the real type) is never deduced from the arguments: FP64 unless given
template <typename T> struct AxNoDeduce { using t = T; };
template <int N, int DIR, int AXIS, int MODE, typename T = double>
__global__ void __launch_bounds__(AX_THREADS)
k_fft_axis(typename C2<T>::t* __restrict__ data, int nx, int ny, int nz,
           const typename AxNoDeduce<T>::t* __restrict__ rin, const typename AxNoDeduce<T>::t* __restrict__ rsub,
           const typename AxNoDeduce<T>::t* __restrict__ kern, typename AxNoDeduce<T>::t* __restrict__ rout,
           typename AxNoDeduce<T>::t scale, const typename C2<T>::t* tw_g) {
  using V = typename C2<T>::t;
  constexpr int P = AX_TILE + 1;
  __shared__ V buf[N * P];
  __shared__ V tw[N];
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
  long base;
  long estride;
  int cnt;
  if (AXIS == 0) {
    const long row0 = (long)blockIdx.x * AX_TILE;
    const long nrow = (long)ny * nz;
    cnt = (int)min((long)AX_TILE, nrow - row0);
    base = row0 * nx;
    estride = 1;
    // rows: element e of row r at base + r*nx + e -> buf[e*P + r]
    for (int i = threadIdx.x; i < N * AX_TILE; i += blockDim.x) {
      const int r = i / N, e = i - r * N;
      V v = mkc<V>(0, 0);
      if (r < cnt) {
        const long g = base + (long)r * nx + e;
        if (MODE == 1) v = mkc<V>(rin[g] - (rsub ? rsub[g] : (T)0), (T)0);
        else v = data[g];
      }
      buf[e * P + r] = v;
    }
  } else {
    const int x0 = blockIdx.x * AX_TILE;
    cnt = min(AX_TILE, nx - x0);
    if (AXIS == 1) { base = (long)blockIdx.y * nx * ny + x0; estride = nx; }
    else { base = (long)blockIdx.y * nx + x0; estride = (long)nx * ny; }
    const long fofs = AXIS == 2 ? (long)blockIdx.z * nx * ny * nz : 0;
    for (int i = threadIdx.x; i < N * AX_TILE; i += blockDim.x) {
      const int e = i / AX_TILE, c = i - e * AX_TILE;
      buf[e * P + c] = (c < cnt) ? data[fofs + base + e * estride + c] : mkc<V>(0, 0);
    }
  }
  __syncthreads();
  smem_fft_cb<N, DIR, P, 1>(buf, cnt, tw);
  __syncthreads();
  if (MODE == 2 || MODE == 4) {
    for (int i = threadIdx.x; i < N * AX_TILE; i += blockDim.x) {
      const int e = i / AX_TILE, c = i - e * AX_TILE;
      if (c < cnt) {
        const T k = kern[base + e * estride + c];
        const V v = buf[e * P + c];
        buf[e * P + c] = MODE == 2 ? cscale(v, k) : mkc<V>(-k * v.y, k * v.x);
      }
    }
    __syncthreads();
    smem_fft_cb<N, -DIR, P, 1>(buf, cnt, tw);
    __syncthreads();
  }
  if (AXIS == 0) {
    for (int i = threadIdx.x; i < N * AX_TILE; i += blockDim.x) {
      const int r = i / N, e = i - r * N;
      if (r < cnt) {
        const long g = base + (long)r * nx + e;
        if (MODE == 3) rout[g] = buf[e * P + r].x * scale;
        else data[g] = buf[e * P + r];
      }
    }
  } else {
    const long fofs = AXIS == 2 ? (long)blockIdx.z * nx * ny * nz : 0;
    for (int i = threadIdx.x; i < N * AX_TILE; i += blockDim.x) {
      const int e = i / AX_TILE, c = i - e * AX_TILE;
      if (c < cnt) data[fofs + base + e * estride + c] = buf[e * P + c];
    }
  }
}

}  // namespace pwb
