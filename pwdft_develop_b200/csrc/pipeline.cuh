#pragma once
// Band-pair H*psi pipeline on sm_100a (kernels and the per-grid Plan;
// included by grid_instance.cu, one translation unit per grid).
//
// Two real bands a, b of the Gamma-point wavefunction are packed into one
// complex field Z = psi_a + i psi_b.  The reference's real-to-complex path
// (Spinor::AddMultSpinorFineR2C, src/SCF/spinor.cpp:377-525) is a real-linear
// map, so running its complex-linear extension on Z gives H psi_a + i H psi_b.
// The coarse->fine spectrum placement of IP_c2f / IP_f2c
// (src/utility.cpp:3150-3275: a coefficient whose index is Nyquist in the set
// S of axes goes, halved, to the all-plus and the all-minus fine positions)
// is separable once every Nyquist coefficient is given a "+" and a "-" slot;
// the z-pencil kernels do that unfolding so the fine-plane kernels only see
// plain zero padding.
//
// Kernels (one launch each per band batch, all pairs in the grid):
//   k_cxy_fwd    coarse plane: FFT x, FFT y                     psi -> A
//   k_zpad       coarse z FFT, kinetic, unfold + pad, fine z IFFT  A -> K, B
//   k_fplane<G>  fine plane: IFFT y, IFFT x, projector partial dots  B -> Wp
//   k_nl_reduce  sum partial dots, scale by gamma*vol/N_fine     Wp -> W
//   k_fplane<A>  fine plane: IFFT y, IFFT x, *V + projector scatter,
//                FFT x, FFT y, truncate                           B -> C (in place)
//   k_zfold      fine z FFT, fold (IP_f2c rule) + kinetic, coarse z IFFT  C,K -> D
//   k_cxy_inv    coarse plane: IFFT y, IFFT x, (accumulate) into hpsi   D -> hpsi
#include <cublas_v2.h>

#include <mutex>
#include <string>
#include <type_traits>

#include "common.hpp"
#include "fft.cuh"
#include "gemm.hpp"
#include "grid_registry.hpp"

namespace pwb {

// bytes of one k-point's split-BF16 projector operands (kpoint.cu)
size_t kq_bf_bytes(const pw_ctx* c);

// kx columns per z-pencil CTA: 24 for FP32 grids divisible by 24 (two
// balanced tiles at n0 = 48), otherwise 16
template <typename T, int N0> struct PencilTile {
  static constexpr int v = (sizeof(T) == 4 && N0 % 24 == 0) ? 24 : 16;
};
constexpr int PLANE_THREADS = 256;
constexpr int PENCIL_THREADS = 256;

template <typename T> using VT = typename C2<T>::t;

// Shared-memory layout of the coarse plane kernels (k_cxy_*, k_exx_*): row y
// at y P0, FR / FC the first-pass lane maps (smem_fft_c's FB) of the x (row)
// and y (column) transforms.  The specialised planes use the pitch and maps
// with the fewest shared-memory wavefronts in a bank model of their 8- /
// 16-byte accesses (twiddle loads included): 48 x 48 27 % (FP32) / 6 % (FP64)
// fewer than P0 = 49 (measured FP32: forward 69 -> 63 us, inverse 54 -> 50 us
// on the 160-band Si64 batch), 24 x 24 17 % / 20 %, 72 x 72 23 % / 4 %.  The
// same search on the z pencils found 12-15 % fewer wavefronts in the
// transforms but slower kernels (the copy phases lose more), so they keep
// rows padded by one.
template <typename T, int N0, int N1> struct PlaneLayout {
  static constexpr int P0 = N0 + 1;
  static constexpr bool FR = false, FC = false;
};
#define PWB_PLANE_LAYOUT(T_, N_, P0_, FR_, FC_) \
  template <> struct PlaneLayout<T_, N_, N_> {  \
    static constexpr int P0 = P0_;              \
    static constexpr bool FR = FR_, FC = FC_;   \
  };
PWB_PLANE_LAYOUT(float, 24, 28, true, true)
PWB_PLANE_LAYOUT(double, 24, 25, true, true)
PWB_PLANE_LAYOUT(float, 48, 53, false, true)
PWB_PLANE_LAYOUT(double, 48, 53, true, true)
PWB_PLANE_LAYOUT(float, 72, 76, true, true)
PWB_PLANE_LAYOUT(double, 72, 73, true, true)
#undef PWB_PLANE_LAYOUT

__device__ __forceinline__ int sgn_idx(int k, int n) { return k <= n / 2 ? k : k - n; }
// slot s in [0, n]: s < n is the FFT index (Nyquist = "+" slot), s == n is the "-" Nyquist slot
__device__ __forceinline__ int slot_fine(int s, int n, int nf) {
  int m = (s < n) ? sgn_idx(s, n) : -(n / 2);
  return (m + nf) % nf;
}

// fine index e of a length-N axis -> slot (coarse size n = N/2), -1 if none;
// slot n is the "-" Nyquist partner at fine index N - n/2
template <int N> __host__ __device__ constexpr int fine_slot(int e) {
  constexpr int n = N / 2, h = n / 2;
  return e <= h ? e : (e > N - h ? e - N + n : (e == N - h ? n : -1));
}
// whether any fine index in [lo, lo + cnt) of a length-N axis has a slot: the
// transform stages of k_floc2 skip, at compile time, inputs known to be zero
// and outputs known to be discarded
template <int N> constexpr bool any_slot(int lo, int cnt) {
  for (int e = lo; e < lo + cnt; ++e)
    if (fine_slot<N>(e) >= 0) return true;
  return false;
}
// inputs j1 of the first stage (fine index N2 j1 + j2, j2 < N2) that are
// zero for every j2, as a bit mask
template <int N, int N1, int N2> constexpr unsigned zero_inputs() {
  unsigned m = 0;
  for (int j1 = 0; j1 < N1; ++j1)
    if (!any_slot<N>(N2 * j1, N2)) m |= 1u << j1;
  return m;
}
// outputs k2 of the second stage (fine index k1 + N1 k2, k1 < N1) that are no
// slot for any k1, as a bit mask
template <int N, int N1, int N2> constexpr unsigned dead_outputs() {
  unsigned m = 0;
  for (int k2 = 0; k2 < N2; ++k2)
    if (!any_slot<N>(N1 * k2, N1)) m |= 1u << k2;
  return m;
}

template <typename V>
__device__ __forceinline__ void load_tw(V* dst, const V* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// global -> shared copies that do not hold a register (cp.async): a thread
// can issue all of its loads before waiting once
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
template <typename E> __device__ __forceinline__ void cp_async(E* dst, const E* src) {
  static_assert(sizeof(E) == 4 || sizeof(E) == 8 || sizeof(E) == 16, "cp.async element size");
  if constexpr (sizeof(E) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"((int)sizeof(E))
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------------------
// coarse plane forward: psi (two real bands) -> A[pair][z][ky][kx]
// ---------------------------------------------------------------------------
template <typename T, int N0, int N1, bool CPLX = false>
__global__ void __launch_bounds__(PLANE_THREADS)
k_cxy_fwd(const T* __restrict__ psi, int ld, int nband, int band0, VT<T>* __restrict__ A,
          const VT<T>* twx_g, const VT<T>* twy_g) {
  using V = VT<T>;
  using PL = PlaneLayout<T, N0, N1>;
  constexpr int P0 = PL::P0;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* pl = reinterpret_cast<V*>(smraw);
  V* twx = pl + N1 * P0;
  V* twy = twx + N0;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  const int z = blockIdx.x, p = blockIdx.y;
  const long ntot_plane = (long)N0 * N1;
  if (CPLX) {
    // one complex band per field (ld in complex elements)
    const V* pc = reinterpret_cast<const V*>(psi) + (long)(band0 + p) * ld + z * ntot_plane;
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
      const int y = i / N0, x = i - y * N0;
      cp_async(&pl[y * P0 + x], &pc[i]);
    }
  } else {
    const int ba = band0 + 2 * p, bb = ba + 1;
    const T* pa = psi + (long)ba * ld + z * ntot_plane;
    const T* pb = (bb < nband) ? psi + (long)bb * ld + z * ntot_plane : nullptr;
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
      const int y = i / N0, x = i - y * N0;
      T* d = reinterpret_cast<T*>(&pl[y * P0 + x]);
      cp_async(d, &pa[i]);
      if (pb) cp_async(d + 1, &pb[i]);
      else d[1] = (T)0;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  smem_fft_cb<N0, -1, 1, P0, PL::FR>(pl, N1, twx);
  __syncthreads();
  smem_fft_cb<N1, -1, P0, 1, PL::FC>(pl, N0, twy);
  __syncthreads();
  const int N2 = gridDim.x;
  V* Ap = A + ((long)p * N2 + z) * ntot_plane;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
    const int y = i / N0, x = i - y * N0;
    Ap[i] = pl[y * P0 + x];
  }
}

// ---------------------------------------------------------------------------
// column bookkeeping shared by k_zpad and k_zfold.
// Tile: fixed ky, kx in [kx0, kx0+TX).  Output/input columns:
//   ky not Nyquist: col i <-> (ky, kx0+i); if kx0+i == n0/2 its "-" partner is col TX
//   ky Nyquist:     col i <-> (ky+, kx0+i (+ slot)); col TX+i <-> (ky-, kx0+i or n0 if kx Nyquist)
// ---------------------------------------------------------------------------
struct ColMap {
  int ncols;
  bool nyy;
  int nyx_i;  // tile-local index of the kx Nyquist column, -1 if none
};
template <int TX> __device__ __forceinline__ ColMap colmap(int ky, int kx0, int tw, int n0, int n1) {
  ColMap m;
  m.nyy = (ky == n1 / 2);
  m.nyx_i = (n0 / 2 >= kx0 && n0 / 2 < kx0 + tw) ? (n0 / 2 - kx0) : -1;
  m.ncols = m.nyy ? 2 * TX : (m.nyx_i >= 0 ? TX + 1 : TX);
  return m;
}
// slot coordinates of column c
template <int TX>
__device__ __forceinline__ void col_slot(const ColMap& m, int c, int ky, int kx0, int n0, int n1,
                                         int& ky_s, int& kx_s) {
  if (m.nyy) {
    if (c < TX) { ky_s = ky; kx_s = kx0 + c; }
    else { ky_s = n1; kx_s = (kx0 + c - TX == n0 / 2) ? n0 : kx0 + c - TX; }
  } else {
    if (c < TX) { ky_s = ky; kx_s = kx0 + c; }
    else { ky_s = ky; kx_s = n0; }
  }
}

// The tile's used columns in compact order: j < tw -> column j, then the
// Nyquist partners (column TX for a kx Nyquist, TX + j' for a ky Nyquist row).
__device__ __forceinline__ int ncompact(const ColMap& m, int tw) {
  return tw + (m.nyy ? tw : (m.nyx_i >= 0 ? 1 : 0));
}
template <int TX> __device__ __forceinline__ int compact_col(int j, int tw) { return j < tw ? j : TX + (j - tw); }

// for (i = threadIdx.x; i < rows * n; i += blockDim.x) f(i / n, i % n) without
// a division per step
template <typename F> __device__ __forceinline__ void for_rows_cols(int rows, int n, F&& f) {
  const int step = blockDim.x;
  const int q = step / n, r = step - q * n;
  int a = threadIdx.x / n, b = threadIdx.x - a * n;
  while (a < rows) {
    f(a, b);
    a += q;
    b += r;
    if (b >= n) { b -= n; ++a; }
  }
}

// ---------------------------------------------------------------------------
// z pencils: coarse FFT z, kinetic, Nyquist unfold, fine pad, fine IFFT z
// ---------------------------------------------------------------------------
template <typename T, int NZ, int NZF, int TX>
__global__ void __launch_bounds__(PENCIL_THREADS, sizeof(T) == 4 ? 4 : 2)
k_zpad(const VT<T>* __restrict__ A, VT<T>* __restrict__ K, VT<T>* __restrict__ B,
       const T* __restrict__ ekin, int n0, int n1, T inv_nc,
       const VT<T>* twz_g, const VT<T>* twzf_g, int cplx = 0, int kf0 = 0, int fpk = 1 << 30, long kstride = 0) {
  using V = VT<T>;
  constexpr int PI = TX + 1;
  constexpr int PO = 2 * TX + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* in = reinterpret_cast<V*>(smraw);     // [NZ][PI]
  V* out = in + NZ * PI;                   // [NZF][PO]
  V* twz = out + NZF * PO;
  V* twzf = twz + NZ;
  __shared__ int colofs[2 * TX];           // slot offset of output column c in a fine plane, -1 if unused
  load_tw(twz, twz_g, NZ);
  load_tw(twzf, twzf_g, NZF);
  const int ky = blockIdx.x, kx0 = blockIdx.y * TX, p = blockIdx.z;
  const int tw = min(TX, n0 - kx0);
  const long nplane = (long)n0 * n1;
  const int nsx = n0 + 1, nsy = n1 + 1;
  const V* Ap = A + (long)p * NZ * nplane + (long)ky * n0 + kx0;
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int z = i / TX, c = i - z * TX;
    if (c < tw) cp_async(&in[z * PI + c], &Ap[z * nplane + c]);
    else in[z * PI + c] = mkc<V>(0, 0);
  }
  const ColMap m = colmap<TX>(ky, kx0, tw, n0, n1);
  if (threadIdx.x < 2 * TX) {
    const int c = threadIdx.x;
    const bool valid = c < m.ncols && !(c < TX && c >= tw) && !(m.nyy && c >= TX && c - TX >= tw);
    int ky_s = 0, kx_s = 0;
    col_slot<TX>(m, c, ky, kx0, n0, n1, ky_s, kx_s);
    colofs[c] = valid ? ky_s * nsx + kx_s : -1;
  }
  for (int i = threadIdx.x; i < NZF * PO; i += blockDim.x) out[i] = mkc<V>(0, 0);
  cp_async_wait_all();
  __syncthreads();
  smem_fft_cb<NZ, -1, PI, 1>(in, tw, twz);
  __syncthreads();
  V* Kp = K ? K + (long)p * NZ * nplane + (long)ky * n0 + kx0 : nullptr;
  // k-point batches: field kf0 + p belongs to k-point (kf0 + p) / fpk
  const T* ek = ekin + (long)((kf0 + p) / fpk) * kstride + (long)ky * n0 + kx0;
  const bool splitrow = m.nyy;
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int kz = i / TX, c = i - kz * TX;
    if (c >= tw) continue;
    const long g = kz * nplane + c;
    const V v = cscale(in[kz * PI + c], inv_nc);
    if (Kp) Kp[g] = cscale(v, ek[g]);
    const bool nyz = (kz == NZ / 2);
    const int fz = kz <= NZ / 2 ? kz : kz + (NZF - NZ);
    const bool split = splitrow || (c == m.nyx_i);
    if (cplx) {
      // complex bands (idxFineGrid, fourier.cpp:291-311): a coarse Nyquist
      // coefficient goes to the "+" fine position only; "-" slots stay zero
      out[fz * PO + c] = v;
    } else if (!split) {
      if (nyz) {
        out[(NZ / 2) * PO + c] = cscale(v, (T)0.5);
        out[(NZF - NZ / 2) * PO + c] = cscale(v, (T)0.5);
      } else {
        out[fz * PO + c] = v;
      }
    } else {
      const int cp = c, cm = splitrow ? TX + c : TX;
      const V h = cscale(v, (T)0.5);
      if (nyz) {
        out[(NZ / 2) * PO + cp] = h;
        out[(NZF - NZ / 2) * PO + cm] = h;
      } else {
        out[fz * PO + cp] = h;
        out[fz * PO + cm] = h;
      }
    }
  }
  __syncthreads();
  // the padded rows between the coarse halves are zero: the first pass of the
  // fine transform skips them
  smem_fft_cb<NZF, +1, PO, 1, false, zero_inputs<NZF, Split<NZF>::n1, NZF / Split<NZF>::n1>()>(out, m.ncols, twzf);
  __syncthreads();
  V* Bp = B + (long)p * NZF * nsy * nsx;
  const long fplane = (long)nsy * nsx;
  for_rows_cols(NZF, ncompact(m, tw), [&](int zf, int j) {
    const int c = compact_col<TX>(j, tw);
    Bp[zf * fplane + colofs[c]] = out[zf * PO + c];
  });
  // the two Nyquist corner slots that no coarse coefficient reaches
  if (m.nyy && m.nyx_i >= 0) {
    for (int zf = threadIdx.x; zf < NZF; zf += blockDim.x) {
      Bp[((long)zf * nsy + n1 / 2) * nsx + n0] = mkc<V>(0, 0);
      Bp[((long)zf * nsy + n1) * nsx + n0 / 2] = mkc<V>(0, 0);
    }
  }
}

// ---------------------------------------------------------------------------
// fine plane kernel (gather or apply mode)
// ---------------------------------------------------------------------------
struct NLArgs {
  const int* ent_xy;
  const void* ent_beta;
  const int* tile_slot;
  const int* slot_atom;
  const int* slot_ent;
  int nent, npmax, nchunk, cr;
  bool present;
};

template <typename T, int NXF, int NYF, bool APPLY>
__global__ void __launch_bounds__(PLANE_THREADS)
k_fplane(VT<T>* __restrict__ BC, const T* __restrict__ vtot, NLArgs nl, VT<T>* __restrict__ Wp,
         const VT<T>* __restrict__ W, int natom, int nslot, T inv_nf,
         const VT<T>* twx_g, const VT<T>* twy_g) {
  using V = VT<T>;
  constexpr int n0 = NXF / 2, n1 = NYF / 2;
  constexpr int nsx = n0 + 1, nsy = n1 + 1;
  constexpr int PS = nsx;          // odd pitch
  constexpr int PR = NXF + 1;      // odd pitch
  const int CR = nl.cr;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* S = reinterpret_cast<V*>(smraw);     // [NYF][PS]
  V* R = S + NYF * PS;                     // [CR][PR]
  V* twx = R + CR * PR;
  V* twy = twx + NXF;
  load_tw(twx, twx_g, NXF);
  load_tw(twy, twy_g, NYF);
  const int zf = blockIdx.x, p = blockIdx.y;
  const int NZF = gridDim.x;
  V* Bp = BC + ((long)p * NZF + zf) * nsy * nsx;
  for (int i = threadIdx.x; i < NYF * PS; i += blockDim.x) S[i] = mkc<V>(0, 0);
  __syncthreads();
  for (int i = threadIdx.x; i < nsy * nsx; i += blockDim.x) {
    const int ys = i / nsx, xs = i - ys * nsx;
    S[slot_fine(ys, n1, NYF) * PS + xs] = Bp[i];
  }
  __syncthreads();
  smem_fft<NYF, +1>(S, nsx, PS, 1, twy);
  __syncthreads();
  const T* beta = reinterpret_cast<const T*>(nl.ent_beta);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = 0; c < nl.nchunk; ++c) {
    const int y0 = c * CR;
    for (int i = threadIdx.x; i < CR * PR; i += blockDim.x) R[i] = mkc<V>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < CR * nsx; i += blockDim.x) {
      const int yl = i / nsx, xs = i - yl * nsx;
      R[yl * PR + slot_fine(xs, n0, NXF)] = S[(y0 + yl) * PS + xs];
    }
    __syncthreads();
    smem_fft<NXF, +1>(R, CR, 1, PR, twx);
    __syncthreads();
    const int tile = zf * nl.nchunk + c;
    if (!APPLY) {
      if (nl.present) {
        const int s0 = nl.tile_slot[tile], s1 = nl.tile_slot[tile + 1];
        for (int s = s0 + warp; s < s1; s += nw) {
          V acc[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) acc[q] = mkc<V>(0, 0);
          const int e0 = nl.slot_ent[s], e1 = nl.slot_ent[s + 1];
          for (int e = e0 + lane; e < e1; e += 32) {
            const int xy = nl.ent_xy[e];
            const int yl = xy / NXF - y0, x = xy - (xy / NXF) * NXF;
            const V v = R[yl * PR + x];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              if (q < nl.npmax) {
                const T b = beta[(long)q * nl.nent + e];
                acc[q].x += b * v.x;
                acc[q].y += b * v.y;
              }
            }
          }
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (q < nl.npmax) {
              T ax = acc[q].x, ay = acc[q].y;
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) {
                ax += __shfl_xor_sync(0xffffffffu, ax, o);
                ay += __shfl_xor_sync(0xffffffffu, ay, o);
              }
              if (lane == 0) Wp[((long)p * nslot + s) * nl.npmax + q] = mkc<V>(ax, ay);
            }
          }
        }
      }
      __syncthreads();
    } else {
      const T* vp = vtot + ((long)zf * NYF + y0) * NXF;
      for (int i = threadIdx.x; i < CR * NXF; i += blockDim.x) {
        const int yl = i / NXF, x = i - yl * NXF;
        R[yl * PR + x] = cscale(R[yl * PR + x], vp[i]);
      }
      __syncthreads();
      if (nl.present) {
        const int s0 = nl.tile_slot[tile], s1 = nl.tile_slot[tile + 1];
        for (int s = s0 + warp; s < s1; s += nw) {
          const int a = nl.slot_atom[s];
          V w[8];
#pragma unroll
          for (int q = 0; q < 8; ++q)
            w[q] = (q < nl.npmax) ? W[((long)p * natom + a) * nl.npmax + q] : mkc<V>(0, 0);
          const int e0 = nl.slot_ent[s], e1 = nl.slot_ent[s + 1];
          for (int e = e0 + lane; e < e1; e += 32) {
            const int xy = nl.ent_xy[e];
            const int yl = xy / NXF - y0, x = xy - (xy / NXF) * NXF;
            T ax = 0, ay = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              if (q < nl.npmax) {
                const T b = beta[(long)q * nl.nent + e];
                ax += b * w[q].x;
                ay += b * w[q].y;
              }
            }
            atomicAdd(&R[yl * PR + x].x, ax);
            atomicAdd(&R[yl * PR + x].y, ay);
          }
        }
      }
      __syncthreads();
      smem_fft<NXF, -1>(R, CR, 1, PR, twx);
      __syncthreads();
      for (int i = threadIdx.x; i < CR * nsx; i += blockDim.x) {
        const int yl = i / nsx, xs = i - yl * nsx;
        S[(y0 + yl) * PS + xs] = R[yl * PR + slot_fine(xs, n0, NXF)];
      }
      __syncthreads();
    }
  }
  if (APPLY) {
    smem_fft<NYF, -1>(S, nsx, PS, 1, twy);
    __syncthreads();
    for (int i = threadIdx.x; i < nsy * nsx; i += blockDim.x) {
      const int ys = i / nsx, xs = i - ys * nsx;
      Bp[i] = cscale(S[slot_fine(ys, n1, NYF) * PS + xs], inv_nf);
    }
  }
}


// ---------------------------------------------------------------------------
// exact exchange pair fields (AddMultSpinorEXX, src/SCF/spinor.cpp:682-781).
// Field f = (band k0 + f / njp, orbital pair jp = f % njp): the plane of
// psi_k (phi_ja + i phi_jb), ja = j0 + 2 jp, jb = ja + 1 (zero past nphi),
// forward 2-D FFT in shared memory, stored like k_cxy_fwd's output.
// ---------------------------------------------------------------------------
template <typename T, int N0, int N1>
__global__ void __launch_bounds__(PLANE_THREADS)
k_exx_fwd(const T* __restrict__ psi, int ld, int k0, const T* __restrict__ phi, int ldp, int j0, int nphi, int njp,
          VT<T>* __restrict__ A, const VT<T>* twx_g, const VT<T>* twy_g) {
  using V = VT<T>;
  using PL = PlaneLayout<T, N0, N1>;
  constexpr int P0 = PL::P0;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* pl = reinterpret_cast<V*>(smraw);
  V* twx = pl + N1 * P0;
  V* twy = twx + N0;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  const int z = blockIdx.x, f = blockIdx.y;
  const int kk = f / njp, jp = f - kk * njp;
  const long ntot_plane = (long)N0 * N1;
  const int ja = j0 + 2 * jp, jb = ja + 1;
  const T* pk = psi + (long)(k0 + kk) * ld + z * ntot_plane;
  const T* pa = phi + (long)ja * ldp + z * ntot_plane;
  const T* pb = (jb < nphi) ? phi + (long)jb * ldp + z * ntot_plane : nullptr;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
    const int y = i / N0, x = i - y * N0;
    const T v = pk[i];
    pl[y * P0 + x] = mkc<V>(v * pa[i], pb ? v * pb[i] : (T)0);
  }
  __syncthreads();
  smem_fft_cb<N0, -1, 1, P0, PL::FR>(pl, N1, twx);
  __syncthreads();
  smem_fft_cb<N1, -1, P0, 1, PL::FC>(pl, N0, twy);
  __syncthreads();
  const int N2 = gridDim.x;
  V* Ap = A + ((long)f * N2 + z) * ntot_plane;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
    const int y = i / N0, x = i - y * N0;
    Ap[i] = pl[y * P0 + x];
  }
}

// inverse 2-D FFT of the njp fields of band k0 + blockIdx.y on plane z and
// out_k (+)= sum_jp w_ja phi_ja Re + w_jb phi_jb Im, accumulated in shared memory
template <typename T, int N0, int N1>
__global__ void __launch_bounds__(PLANE_THREADS)
k_exx_inv(const VT<T>* __restrict__ A, int njp, const T* __restrict__ phi, int ldp, int j0, int nphi,
          const T* __restrict__ wj, T* __restrict__ out, int ldo, int k0, int accumulate, const VT<T>* twx_g,
          const VT<T>* twy_g) {
  using V = VT<T>;
  using PL = PlaneLayout<T, N0, N1>;
  constexpr int P0 = PL::P0;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* pl = reinterpret_cast<V*>(smraw);
  V* twx = pl + N1 * P0;
  V* twy = twx + N0;
  T* acc = reinterpret_cast<T*>(twy + N1);
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  const int z = blockIdx.x, kk = blockIdx.y;
  const int N2 = gridDim.x;
  const long ntot_plane = (long)N0 * N1;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) acc[i] = (T)0;
  for (int jp = 0; jp < njp; ++jp) {
    const V* Dp = A + ((long)(kk * njp + jp) * N2 + z) * ntot_plane;
    __syncthreads();
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
      const int y = i / N0, x = i - y * N0;
      pl[y * P0 + x] = Dp[i];
    }
    __syncthreads();
    smem_fft_cb<N1, +1, P0, 1, PL::FC>(pl, N0, twy);
    __syncthreads();
    smem_fft_cb<N0, +1, 1, P0, PL::FR>(pl, N1, twx);
    __syncthreads();
    const int ja = j0 + 2 * jp, jb = ja + 1;
    const T wa = wj[ja], wb = (jb < nphi) ? wj[jb] : (T)0;
    const T* pa = phi + (long)ja * ldp + z * ntot_plane;
    const T* pb = (jb < nphi) ? phi + (long)jb * ldp + z * ntot_plane : pa;
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
      const int y = i / N0, x = i - y * N0;
      const V v = pl[y * P0 + x];
      acc[i] += wa * pa[i] * v.x + wb * pb[i] * v.y;
    }
  }
  __syncthreads();
  T* o = out + (long)(k0 + kk) * ldo + z * ntot_plane;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) o[i] = accumulate ? o[i] + acc[i] : acc[i];
}

// ---------------------------------------------------------------------------
// fine plane, local potential only (the projectors are applied on the coarse
// grid as dense GEMMs): IFFT y on the slot columns, then per warp a group of
// rows: IFFT x, * V_loc, FFT x, truncate; FFT y; truncate.  MODE 1 starts
// from two real fine-grid fields instead (used to build the coarse projector
// matrix) and skips the inverse transforms and the potential.
// ---------------------------------------------------------------------------
constexpr int FLOC_THREADS = 256;

template <typename T, int NXF, int NYF, int MODE>
__global__ void __launch_bounds__(FLOC_THREADS, sizeof(T) == 4 ? 3 : 1)
k_floc(VT<T>* __restrict__ BC, const T* __restrict__ vtot, const T* __restrict__ fin, long fin_pair_stride,
       T inv_nf, const VT<T>* twx_g, const VT<T>* twy_g, int deriv = 0, T gfac = 0) {
  using V = VT<T>;
  constexpr int n0 = NXF / 2, n1 = NYF / 2;
  constexpr int nsx = n0 + 1, nsy = n1 + 1;
  constexpr int PS = nsx;
  constexpr int PR = NXF + 1;
  constexpr int F = FftGroup<NXF>::f;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* S = reinterpret_cast<V*>(smraw);          // [NYF][PS]
  V* twx = S + NYF * PS;
  V* twy = twx + NXF;
  V* Rall = twy + NYF;                          // [nwarps][F][PR]
  load_tw(twx, twx_g, NXF);
  load_tw(twy, twy_g, NYF);
  const int zf = blockIdx.x, p = blockIdx.y;
  const int NZF = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  V* Rw = Rall + warp * F * PR;
  V* Bp = BC + ((long)p * NZF + zf) * nsy * nsx;
  if (MODE == 0) {
    for (int i = threadIdx.x; i < NYF * PS; i += blockDim.x) S[i] = mkc<V>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < nsy * nsx; i += blockDim.x) {
      const int ys = i / nsx, xs = i - ys * nsx;
      S[slot_fine(ys, n1, NYF) * PS + xs] = Bp[i];
    }
    __syncthreads();
    smem_fft_cb<NYF, +1, PS, 1>(S, nsx, twy);
  }
  __syncthreads();
  for (int r0 = warp * F; r0 < NYF; r0 += nw * F) {
    const int nr = min(F, NYF - r0);
    if (MODE == 0) {
      for (int i = lane; i < F * PR; i += 32) Rw[i] = mkc<V>(0, 0);
      __syncwarp();
      for (int i = lane; i < nr * nsx; i += 32) {
        const int f = i / nsx, xs = i - f * nsx;
        Rw[f * PR + slot_fine(xs, n0, NXF)] = S[(r0 + f) * PS + xs];
      }
      __syncwarp();
      smem_fft_c<NXF, +1, 1, PR>(Rw, nr, twx, 0, 1);
      const T* vp = vtot + ((long)zf * NYF + r0) * NXF;
      for (int i = lane; i < nr * NXF; i += 32) {
        const int f = i / NXF, x = i - f * NXF;
        Rw[f * PR + x] = cscale(Rw[f * PR + x], vp[i]);
      }
    } else {
      const T* fa = fin + (long)(2 * p) * fin_pair_stride + ((long)zf * NYF + r0) * NXF;
      const T* fb = fin + (long)(2 * p + 1) * fin_pair_stride + ((long)zf * NYF + r0) * NXF;
      for (int i = lane; i < nr * NXF; i += 32) {
        const int f = i / NXF, x = i - f * NXF;
        Rw[f * PR + x] = mkc<V>(fa[i], fb[i]);
      }
    }
    __syncwarp();
    smem_fft_c<NXF, -1, 1, PR>(Rw, nr, twx, 0, 1);
    if (MODE == 1 && deriv == 1) {
      // spectral d/dx: multiply by i G_x of the fine frequency
      for (int i = lane; i < nr * NXF; i += 32) {
        const int f = i / NXF, x = i - f * NXF;
        const T g = gfac * (T)sgn_idx(x, NXF);
        const V v = Rw[f * PR + x];
        Rw[f * PR + x] = mkc<V>(-g * v.y, g * v.x);
      }
      __syncwarp();
    }
    for (int i = lane; i < nr * nsx; i += 32) {
      const int f = i / nsx, xs = i - f * nsx;
      S[(r0 + f) * PS + xs] = Rw[f * PR + slot_fine(xs, n0, NXF)];
    }
    __syncwarp();
  }
  __syncthreads();
  smem_fft_cb<NYF, -1, PS, 1>(S, nsx, twy);
  __syncthreads();
  if (MODE == 1 && deriv == 2) {
    for (int i = threadIdx.x; i < NYF * nsx; i += blockDim.x) {
      const int y = i / nsx, xs = i - y * nsx;
      const T g = gfac * (T)sgn_idx(y, NYF);
      const V v = S[y * PS + xs];
      S[y * PS + xs] = mkc<V>(-g * v.y, g * v.x);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < nsy * nsx; i += blockDim.x) {
    const int ys = i / nsx, xs = i - ys * nsx;
    Bp[i] = cscale(S[slot_fine(ys, n1, NYF) * PS + xs], inv_nf);
  }
}


// ---------------------------------------------------------------------------
// fine plane, local potential only, fused form (the hot apply of H*psi).
// Same result as k_floc MODE 0 with fewer shared-memory passes:
//  * the y inverse transform reads the slot rows of B straight from global
//    memory (non-slot rows are zero), no zero fill or scatter;
//  * per row the x inverse transform reads the slot columns of S, its second
//    pass multiplies by V and runs the first stage of the forward transform
//    in the same registers (the k1 + N1 k2 distribution of the inverse's output
//    is the stride the forward's decimation needs), and the forward's second
//    stage writes only the slot columns back;
//  * the y forward transform's second pass writes the slot rows of C
//    directly (x 1/N_fine).
// ---------------------------------------------------------------------------
// Shared-memory layout of k_floc2: S tile (slot columns of the fine plane)
// with row y at y PS + SKS (y / NY2), per-warp row buffers with element e of
// row f at f PR + e + SKR (e / NX2), and whether the first pass of the column
// (FA) and row (FB) transforms puts the transform index on the fastest lanes.
// The specialised planes use the layout with the fewest shared-memory
// wavefronts found by a search over pitches, skews and lane maps with a bank
// model of their 8- / 16-byte accesses (twiddle loads included; 96: 31 % /
// 20 % fewer than plain padded rows for FP32 / FP64, 48: 19 % / 15 %, 144:
// 9 % / 19 %); other planes keep plain padded rows.
template <typename T, int NXF, int NYF> struct FlocLayout {
  static constexpr int PS = NXF / 2 + 1, SKS = 0, PR = NXF + 1, SKR = 0;
  static constexpr bool FA = false, FB = false;
};
#define PWB_FLOC_LAYOUT(T_, N_, PS_, SKS_, PR_, SKR_, FA_, FB_)               \
  template <> struct FlocLayout<T_, N_, N_> {                                 \
    static constexpr int PS = PS_, SKS = SKS_, PR = PR_, SKR = SKR_;          \
    static constexpr bool FA = FA_, FB = FB_;                                 \
  };
PWB_FLOC_LAYOUT(float, 96, 60, 2, 108, 1, true, true)
PWB_FLOC_LAYOUT(double, 96, 52, 1, 106, 1, true, true)
PWB_FLOC_LAYOUT(float, 48, 37, 3, 54, 1, true, true)
PWB_FLOC_LAYOUT(double, 48, 29, 3, 54, 1, true, false)
PWB_FLOC_LAYOUT(float, 144, 73, 1, 156, 1, false, false)
PWB_FLOC_LAYOUT(double, 144, 74, 1, 156, 1, false, false)
#undef PWB_FLOC_LAYOUT
// elements of the S tile of k_floc2 for a plane of NYF rows split NY2 per skew step
template <typename LY, int NYF, int NY2> constexpr int floc_s_size() { return NYF * LY::PS + LY::SKS * (NYF / NY2); }
// the plain padded layout (the alternative radix decomposition uses it)
template <int NXF> struct FlocLayoutPlain {
  static constexpr int PS = NXF / 2 + 1, SKS = 0, PR = NXF + 1, SKR = 0;
  static constexpr bool FA = false, FB = false;
};
template <typename T, int NXF, int NYF, int VAR>
using FlocLayoutVar = typename std::conditional<VAR == 1, FlocLayoutPlain<NXF>, FlocLayout<T, NXF, NYF>>::type;

// Lane order of the local potential for the row pass of k_floc2 (fft_variant
// 2): lane f NX1 + k1 of a warp holds row r0 + f (rows in groups of FX) and
// needs V(x = k1 + NX1 k2) for k2 = 0 .. NX2-1.  The permuted copy stores, per
// fine plane and row group, NQ blocks of 32 lanes x VW consecutive k2 values,
// so each vector load of a warp reads 32 VW contiguous reals.  Unused lanes
// (rows past the plane, lanes past FX NX1) hold zeros.
template <typename T, int NXF, int NYF> struct VpermLayout {
  static constexpr int NX1 = Split<NXF>::n1, NX2 = NXF / NX1, FX = 32 / NX1;
  static constexpr int VW = 16 / (int)sizeof(T);                // reals per 16-byte load
  static constexpr bool OK = NX2 % VW == 0;
  static constexpr int NQ = NX2 / VW, NG = (NYF + FX - 1) / FX;
  static constexpr long PLANE = (long)NG * NQ * 32 * VW;        // reals per fine plane
};
template <typename T, int NXF, int NYF>
__global__ void k_vperm(const T* __restrict__ v, T* __restrict__ vp, int nzf) {
  using LY = VpermLayout<T, NXF, NYF>;
  const long total = LY::PLANE * nzf;
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < total; o += (long)gridDim.x * blockDim.x) {
    const long zf = o / LY::PLANE;
    long r = o - zf * LY::PLANE;
    const int i = (int)(r % LY::VW);
    r /= LY::VW;
    const int lane = (int)(r % 32);
    r /= 32;
    const int q = (int)(r % LY::NQ);
    const int g = (int)(r / LY::NQ);
    const int f = lane / LY::NX1, k1 = lane - f * LY::NX1;
    const int y = g * LY::FX + f, x = k1 + LY::NX1 * (q * LY::VW + i);
    vp[o] = (f < LY::FX && y < NYF) ? v[(zf * NYF + y) * NXF + x] : (T)0;
  }
}

// VAR selects the radix decomposition of the x and y transforms (0: Split,
// 1: SplitAlt) and where the inter-stage twiddles come from (0, 1: the shared
// tables; 2: Split with W^{j k} formed in registers from one table entry per
// transform), the autotuner's FFT candidates
template <typename T, int NXF, int NYF, int VAR = 0>
__global__ void __launch_bounds__(FLOC_THREADS, sizeof(T) == 4 ? 3 : 1)
k_floc2(VT<T>* __restrict__ BC, const T* __restrict__ vtot, T inv_nf, const VT<T>* twx_g, const VT<T>* twy_g,
        const T* __restrict__ vperm) {
  using V = VT<T>;
  constexpr int n0 = NXF / 2;
  constexpr int nsx = n0 + 1, nsy = NYF / 2 + 1;
  using LY = FlocLayoutVar<T, NXF, NYF, VAR>;
  constexpr int PS = LY::PS, SKS = LY::SKS, PR = LY::PR, SKR = LY::SKR;
  constexpr bool FA = LY::FA, FB = LY::FB;
  constexpr bool RTW = VAR == 2;
  constexpr int NX1 = SplitVar<NXF, VAR>::n1, NX2 = NXF / NX1, FX = 32 / NX1;
  constexpr int NY1 = SplitVar<NYF, VAR>::n1, NY2 = NYF / NY1, FY = 32 / NY1;
  constexpr int RX = (FX * NX2 + 31) / 32;
  static_assert(PS >= nsx && PR >= NXF + SKR * (NX1 - 1), "k_floc2 layout rows overlap");
  extern __shared__ __align__(16) unsigned char smraw[];
  V* S = reinterpret_cast<V*>(smraw);          // row y at y PS + SKS (y / NY2)
  V* twx = S + floc_s_size<LY, NYF, NY2>();
  V* twy = twx + NXF;
  V* Rall = twy + NYF;                          // [nwarps][FX][PR]
  load_tw(twx, twx_g, NXF);
  load_tw(twy, twy_g, NYF);
  const int zf = blockIdx.x, p = blockIdx.y;
  const int NZF = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  V* Bp = BC + ((long)p * NZF + zf) * nsy * nsx;
  __syncthreads();

  // A: inverse y transform of the nsx slot columns, GA columns per warp step
  // (variant 2: twice the FY of the second pass when that fills whole warp
  // rounds in the first pass, 96: 8 columns x 12 = 3 rounds instead of 4 x 12
  // in two half-empty rounds)
  constexpr int GA = (RTW && (2 * FY * NY2) % 32 == 0) ? 2 * FY : FY;
  constexpr int RA = (GA * NY2 + 31) / 32;
  for (int g = warp * GA; g < nsx; g += nw * GA) {
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int it = lane + 32 * r;
      const int f = FA ? it % GA : it / NY2, j2 = FA ? it / GA : it - f * NY2;
      const int c = g + f;
      if (it < GA * NY2 && c < nsx) {
        V t[NY1];
        sfor<0, NY1>([&](auto jI) {
          constexpr int j1 = decltype(jI)::value;
          if constexpr (!RTW || any_slot<NYF>(NY2 * j1, NY2)) {
            const int s = fine_slot<NYF>(NY2 * j1 + j2);
            t[j1] = s >= 0 ? Bp[s * nsx + c] : mkc<V>(0, 0);
          } else {
            t[j1] = mkc<V>(0, 0);
          }
        });
        if constexpr (RTW) DFTZ<NY1, +1, V, zero_inputs<NYF, NY1, NY2>()>::run(t);
        else DFT<NY1, +1, V>::run(t);
        if constexpr (RTW) {
          V p_[NY1];
          V w = twy[j2];
          w.y = -w.y;
          twiddle_powers<NY1>(w, p_);
#pragma unroll
          for (int k1 = 1; k1 < NY1; ++k1) t[k1] = cmul(t[k1], p_[k1]);
        } else {
#pragma unroll
          for (int k1 = 1; k1 < NY1; ++k1) {
            V w = twy[j2 * k1];
            w.y = -w.y;
            t[k1] = cmul(t[k1], w);
          }
        }
#pragma unroll
        for (int k1 = 0; k1 < NY1; ++k1) S[(NY2 * k1 + j2) * PS + SKS * k1 + c] = t[k1];
      }
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < GA / FY; ++h) {
      const int f = lane / NY1, k1 = lane - f * NY1;
      const int c = g + h * FY + f;
      const bool act = lane < FY * NY1 && c < nsx;
      V u[NY2];
      if (act) {
#pragma unroll
        for (int j2 = 0; j2 < NY2; ++j2) u[j2] = S[(NY2 * k1 + j2) * PS + SKS * k1 + c];
        DFT<NY2, +1, V>::run(u);
      }
      __syncwarp();
      if (act) {
#pragma unroll
        for (int k2 = 0; k2 < NY2; ++k2) {
          const int y = k1 + NY1 * k2;
          S[y * PS + SKS * (y / NY2) + c] = u[k2];
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();

  // B: rows (x): inverse, x V, forward, keep the slot columns
  V* Rw = Rall + warp * FX * PR;
  for (int r0 = warp * FX; r0 < NYF; r0 += nw * FX) {
    const int nr = min(FX, NYF - r0);
#pragma unroll
    for (int r = 0; r < RX; ++r) {
      const int it = lane + 32 * r;
      const int f = FB ? it % FX : it / NX2, j2 = FB ? it / FX : it - f * NX2;
      if (it < FX * NX2 && f < nr) {
        V t[NX1];
        const V* srow = S + (r0 + f) * PS + SKS * ((r0 + f) / NY2);
        sfor<0, NX1>([&](auto jI) {
          constexpr int j1 = decltype(jI)::value;
          if constexpr (!RTW || any_slot<NXF>(NX2 * j1, NX2)) {
            const int s = fine_slot<NXF>(NX2 * j1 + j2);
            t[j1] = s >= 0 ? srow[s] : mkc<V>(0, 0);
          } else {
            t[j1] = mkc<V>(0, 0);
          }
        });
        if constexpr (RTW) DFTZ<NX1, +1, V, zero_inputs<NXF, NX1, NX2>()>::run(t);
        else DFT<NX1, +1, V>::run(t);
        if constexpr (RTW) {
          V p_[NX1];
          V w = twx[j2];
          w.y = -w.y;
          twiddle_powers<NX1>(w, p_);
#pragma unroll
          for (int k1 = 1; k1 < NX1; ++k1) t[k1] = cmul(t[k1], p_[k1]);
        } else {
#pragma unroll
          for (int k1 = 1; k1 < NX1; ++k1) {
            V w = twx[j2 * k1];
            w.y = -w.y;
            t[k1] = cmul(t[k1], w);
          }
        }
#pragma unroll
        for (int k1 = 0; k1 < NX1; ++k1) Rw[f * PR + (NX2 + SKR) * k1 + j2] = t[k1];
      }
    }
    __syncwarp();
    {
      const int f = lane / NX1, k1 = lane - f * NX1;
      const bool act = lane < FX * NX1 && f < nr;
      if (act) {
        V u[NX2];
        V* rr = Rw + f * PR + (NX2 + SKR) * k1;
#pragma unroll
        for (int j2 = 0; j2 < NX2; ++j2) u[j2] = rr[j2];
        DFT<NX2, +1, V>::run(u);                    // u[k2] = x[k1 + NX1 k2]
        if constexpr (RTW && VpermLayout<T, NXF, NYF>::OK) {
          using PL = VpermLayout<T, NXF, NYF>;
          using VV = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
          const VV* vq = reinterpret_cast<const VV*>(vperm + ((long)zf * PL::NG + r0 / FX) * PL::NQ * 32 * PL::VW) + lane;
#pragma unroll
          for (int q = 0; q < PL::NQ; ++q) {
            const VV vv = vq[32 * q];
            if constexpr (sizeof(T) == 4) {
              u[4 * q + 0] = cscale(u[4 * q + 0], (T)vv.x);
              u[4 * q + 1] = cscale(u[4 * q + 1], (T)vv.y);
              u[4 * q + 2] = cscale(u[4 * q + 2], (T)vv.z);
              u[4 * q + 3] = cscale(u[4 * q + 3], (T)vv.w);
            } else {
              u[2 * q + 0] = cscale(u[2 * q + 0], (T)vv.x);
              u[2 * q + 1] = cscale(u[2 * q + 1], (T)vv.y);
            }
          }
        } else {
          const T* vrow = vtot + ((long)zf * NYF + r0 + f) * NXF + k1;
#pragma unroll
          for (int k2 = 0; k2 < NX2; ++k2) u[k2] = cscale(u[k2], vrow[NX1 * k2]);
        }
        DFT<NX2, -1, V>::run(u);                    // forward, first stage over k2
        if constexpr (RTW) {
          V p_[NX2];
          twiddle_powers<NX2>(twx[k1], p_);
#pragma unroll
          for (int m2 = 1; m2 < NX2; ++m2) u[m2] = cmul(u[m2], p_[m2]);
        } else {
#pragma unroll
          for (int m2 = 1; m2 < NX2; ++m2) u[m2] = cmul(u[m2], twx[k1 * m2]);
        }
#pragma unroll
        for (int m2 = 0; m2 < NX2; ++m2) rr[m2] = u[m2];
      }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < RX; ++r) {
      const int it = lane + 32 * r;
      const int f = FB ? it % FX : it / NX2, m2 = FB ? it / FX : it - f * NX2;
      if (it < FX * NX2 && f < nr) {
        V t[NX1];
#pragma unroll
        for (int k1 = 0; k1 < NX1; ++k1) t[k1] = Rw[f * PR + (NX2 + SKR) * k1 + m2];
        DFT<NX1, -1, V>::run(t);                    // forward, second stage over k1
        V* srow = S + (r0 + f) * PS + SKS * ((r0 + f) / NY2);
        sfor<0, NX1>([&](auto mI) {
          constexpr int m1 = decltype(mI)::value;
          if constexpr (!RTW || any_slot<NXF>(NX2 * m1, NX2)) {
            const int s = fine_slot<NXF>(m2 + NX2 * m1);
            if (s >= 0) srow[s] = t[m1];
          }
        });
      }
    }
    __syncwarp();
  }
  __syncthreads();

  // C: forward y transform of the slot columns, slot rows straight to C
  for (int g = warp * GA; g < nsx; g += nw * GA) {
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int it = lane + 32 * r;
      const int f = FA ? it % GA : it / NY2, j2 = FA ? it / GA : it - f * NY2;
      const int c = g + f;
      if (it < GA * NY2 && c < nsx) {
        V t[NY1];
#pragma unroll
        for (int j1 = 0; j1 < NY1; ++j1) t[j1] = S[(NY2 * j1 + j2) * PS + SKS * j1 + c];
        DFT<NY1, -1, V>::run(t);
        if constexpr (RTW) {
          V p_[NY1];
          twiddle_powers<NY1>(twy[j2], p_);
#pragma unroll
          for (int k1 = 1; k1 < NY1; ++k1) t[k1] = cmul(t[k1], p_[k1]);
        } else {
#pragma unroll
          for (int k1 = 1; k1 < NY1; ++k1) t[k1] = cmul(t[k1], twy[j2 * k1]);
        }
#pragma unroll
        for (int k1 = 0; k1 < NY1; ++k1) S[(NY2 * k1 + j2) * PS + SKS * k1 + c] = t[k1];
      }
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < GA / FY; ++h) {
      const int f = lane / NY1, k1 = lane - f * NY1;
      const int c = g + h * FY + f;
      if (lane < FY * NY1 && c < nsx) {
        V u[NY2];
#pragma unroll
        for (int j2 = 0; j2 < NY2; ++j2) u[j2] = S[(NY2 * k1 + j2) * PS + SKS * k1 + c];
        DFT<NY2, -1, V>::run(u);
        sfor<0, NY2>([&](auto kI) {
          constexpr int k2 = decltype(kI)::value;
          if constexpr (!RTW || any_slot<NYF>(NY1 * k2, NY1)) {
            const int s = fine_slot<NYF>(k1 + NY1 * k2);
            if (s >= 0) Bp[s * nsx + c] = cscale(u[k2], inv_nf);
          }
        });
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// density: rho(r) += w_a |Re psi_f|^2 + w_b |Im psi_f|^2 over the pairs of a
// chunk (CalculateDensity, src/SCF/hamiltonian.cpp:2511-2547).  One CTA owns
// one fine plane for `ppc` pairs and keeps its partial sums in registers.
// ---------------------------------------------------------------------------
template <typename T, int NXF, int NYF>
__global__ void __launch_bounds__(FLOC_THREADS)
k_fdens(const VT<T>* __restrict__ BC, int npair, int ppc, const double* __restrict__ w, double* __restrict__ rho,
        const VT<T>* twx_g, const VT<T>* twy_g) {
  using V = VT<T>;
  constexpr int n0 = NXF / 2, n1 = NYF / 2;
  constexpr int nsx = n0 + 1, nsy = n1 + 1;
  constexpr int PS = nsx;
  constexpr int PR = NXF + 1;
  constexpr int F = FftGroup<NXF>::f;
  constexpr int NW = FLOC_THREADS / 32;
  constexpr int RG = (NYF + NW * F - 1) / (NW * F);
  constexpr int EPL = (F * NXF + 31) / 32;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* S = reinterpret_cast<V*>(smraw);
  V* twx = S + NYF * PS;
  V* twy = twx + NXF;
  V* Rall = twy + NYF;
  load_tw(twx, twx_g, NXF);
  load_tw(twy, twy_g, NYF);
  const int zf = blockIdx.x;
  const int NZF = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  V* Rw = Rall + warp * F * PR;
  double acc[RG][EPL];
#pragma unroll
  for (int a = 0; a < RG; ++a)
#pragma unroll
    for (int k = 0; k < EPL; ++k) acc[a][k] = 0.0;
  const int p0 = blockIdx.y * ppc, p1 = min(npair, p0 + ppc);
  for (int p = p0; p < p1; ++p) {
    const V* Bp = BC + ((long)p * NZF + zf) * nsy * nsx;
    const double wa = w[2 * p], wb = w[2 * p + 1];
    __syncthreads();
    for (int i = threadIdx.x; i < NYF * PS; i += blockDim.x) S[i] = mkc<V>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < nsy * nsx; i += blockDim.x) {
      const int ys = i / nsx, xs = i - ys * nsx;
      S[slot_fine(ys, n1, NYF) * PS + xs] = Bp[i];
    }
    __syncthreads();
    smem_fft_cb<NYF, +1, PS, 1>(S, nsx, twy);
    __syncthreads();
#pragma unroll
    for (int rg = 0; rg < RG; ++rg) {
      const int r0 = (warp + rg * NW) * F;
      if (r0 < NYF) {
        const int nr = min(F, NYF - r0);
        for (int i = lane; i < F * PR; i += 32) Rw[i] = mkc<V>(0, 0);
        __syncwarp();
        for (int i = lane; i < nr * nsx; i += 32) {
          const int f = i / nsx, xs = i - f * nsx;
          Rw[f * PR + slot_fine(xs, n0, NXF)] = S[(r0 + f) * PS + xs];
        }
        __syncwarp();
        smem_fft_c<NXF, +1, 1, PR>(Rw, nr, twx, 0, 1);
#pragma unroll
        for (int k = 0; k < EPL; ++k) {
          const int i = lane + 32 * k;
          if (i < nr * NXF) {
            const int f = i / NXF, x = i - f * NXF;
            const V v = Rw[f * PR + x];
            acc[rg][k] += wa * (double)v.x * (double)v.x + wb * (double)v.y * (double)v.y;
          }
        }
        __syncwarp();
      }
    }
  }
#pragma unroll
  for (int rg = 0; rg < RG; ++rg) {
    const int r0 = (warp + rg * NW) * F;
    if (r0 < NYF) {
      const int nr = min(F, NYF - r0);
#pragma unroll
      for (int k = 0; k < EPL; ++k) {
        const int i = lane + 32 * k;
        if (i < nr * NXF) atomicAdd(&rho[((long)zf * NYF + r0) * NXF + i], acc[rg][k]);
      }
    }
  }
}

// projector fields: field[l][idx] = beta for the projectors of one batch
template <typename T>
__global__ void k_scatter_beta(T* __restrict__ fields, long nf, const int* __restrict__ idx,
                               const double* __restrict__ beta, const long* __restrict__ pidx_off,
                               const long* __restrict__ pbeta_off, const int* __restrict__ pnpts, int l0, int nl) {
  const int l = blockIdx.y;
  if (l0 + l >= nl) return;
  const long io = pidx_off[l0 + l], bo = pbeta_off[l0 + l];
  const int np = pnpts[l0 + l];
  T* f = fields + (long)l * nf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) f[idx[io + i]] = (T)beta[bo + i];
}

// complex projector field conj(e^{i k.d}) beta for projector l0 + l into the
// real / imaginary field pair (2l, 2l + 1); d = grid point - atom (Cartesian)
template <typename T>
__global__ void k_scatter_beta_k(T* __restrict__ fields, long nf, const int* __restrict__ idx,
                                 const double* __restrict__ beta, const double* __restrict__ disp,
                                 const long* __restrict__ pidx_off, const long* __restrict__ pbeta_off,
                                 const int* __restrict__ pnpts, int l0, int nl, double kx, double ky, double kz) {
  const int l = blockIdx.y;
  if (l0 + l >= nl) return;
  const long io = pidx_off[l0 + l], bo = pbeta_off[l0 + l];
  const int np = pnpts[l0 + l];
  T* fr = fields + (long)(2 * l) * nf;
  T* fi = fr + nf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const double* d = disp + 3 * (io + i);
    double sn, cs;
    sincos(kx * d[0] + ky * d[1] + kz * d[2], &sn, &cs);
    const double b = beta[bo + i];
    fr[idx[io + i]] = (T)(b * cs);
    fi[idx[io + i]] = (T)(-b * sn);
  }
}

// complex W[l][b] *= d[l] (d real)
template <typename T>
__global__ void k_scale_rows_c(VT<T>* __restrict__ W, const T* __restrict__ d, int nproj, int nb) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < (long)nproj * nb) W[i] = cscale(W[i], d[i % nproj]);
}

// W[l][b] *= d[l]  (W column-major nproj x nb)
template <typename T>
__global__ void k_scale_rows(T* __restrict__ W, const T* __restrict__ d, int nproj, int nb) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < (long)nproj * nb) W[i] *= d[i % nproj];
}

// W[p][a][q] = wgt[a][q] * sum over the atom's slots of Wp[p][slot][q]
template <typename T>
__global__ void k_nl_reduce(const VT<T>* __restrict__ Wp, VT<T>* __restrict__ W, const int* atom_slot,
                            const int* atom_slot_list, const T* wgt, int natom, int nslot, int npmax) {
  using V = VT<T>;
  const int p = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natom * npmax) return;
  const int a = i / npmax, q = i - a * npmax;
  T sx = 0, sy = 0;
  for (int j = atom_slot[a]; j < atom_slot[a + 1]; ++j) {
    const V v = Wp[((long)p * nslot + atom_slot_list[j]) * npmax + q];
    sx += v.x;
    sy += v.y;
  }
  const T g = wgt[i];
  W[(long)p * natom * npmax + i] = mkc<V>(sx * g, sy * g);
}

// ---------------------------------------------------------------------------
// z pencils: fine FFT z, fold to coarse (IP_f2c), add kinetic, coarse IFFT z
// ---------------------------------------------------------------------------
template <typename T, int NZ, int NZF, int TX>
__global__ void __launch_bounds__(PENCIL_THREADS, sizeof(T) == 4 ? 4 : 2)
k_zfold(const VT<T>* __restrict__ C, const VT<T>* __restrict__ K, VT<T>* __restrict__ D, int n0, int n1,
        const VT<T>* twz_g, const VT<T>* twzf_g, int deriv = 0, T gfac = 0, int cplx = 0,
        const T* __restrict__ fmask = nullptr) {
  using V = VT<T>;
  constexpr int PI = 2 * TX + 1;
  constexpr int PA = TX + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* in = reinterpret_cast<V*>(smraw);    // [NZF][PI]
  V* acc = in + NZF * PI;                 // [NZ][PA]
  V* twz = acc + NZ * PA;
  V* twzf = twz + NZ;
  __shared__ int colofs[2 * TX];          // slot offset of input column c in a fine plane, -1 if unused
  load_tw(twz, twz_g, NZ);
  load_tw(twzf, twzf_g, NZF);
  const int ky = blockIdx.x, kx0 = blockIdx.y * TX, p = blockIdx.z;
  const int tw = min(TX, n0 - kx0);
  const ColMap m = colmap<TX>(ky, kx0, tw, n0, n1);
  const int nsx = n0 + 1, nsy = n1 + 1;
  if (threadIdx.x < 2 * TX) {
    const int c = threadIdx.x;
    const bool valid = c < m.ncols && !(c < TX && c >= tw) && !(m.nyy && c >= TX && c - TX >= tw);
    int ky_s = 0, kx_s = 0;
    col_slot<TX>(m, c, ky, kx0, n0, n1, ky_s, kx_s);
    colofs[c] = valid ? ky_s * nsx + kx_s : -1;
  }
  __syncthreads();
  const V* Cp = C + (long)p * NZF * nsy * nsx;
  const long fplane = (long)nsy * nsx;
  // columns the FFT reads but no slot feeds (c < ncols, not in the compact list)
  if (tw < TX) {
    for (int i = threadIdx.x; i < NZF * 2 * TX; i += blockDim.x) {
      const int zf = i / (2 * TX), c = i - zf * (2 * TX);
      if (c < m.ncols && colofs[c] < 0) in[zf * PI + c] = mkc<V>(0, 0);
    }
  }
  for_rows_cols(NZF, ncompact(m, tw), [&](int zf, int j) {
    const int c = compact_col<TX>(j, tw);
    cp_async(&in[zf * PI + c], &Cp[zf * fplane + colofs[c]]);
  });
  // the kinetic term of this tile, needed after the fine transform
  const long nplane = (long)n0 * n1;
  const V* Kp = K ? K + (long)p * NZ * nplane + (long)ky * n0 + kx0 : nullptr;
  V* ks = acc;   // staged in the accumulator array itself
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int kz = i / TX, c = i - kz * TX;
    if (Kp && c < tw) cp_async(&ks[kz * PA + c], &Kp[kz * nplane + c]);
    else ks[kz * PA + c] = mkc<V>(0, 0);
  }
  cp_async_wait_all();
  __syncthreads();
  // only the fine rows that fold onto the coarse spectrum are read afterwards
  smem_fft_cb<NZF, -1, PI, 1, false, 0u, dead_outputs<NZF, Split<NZF>::n1, NZF / Split<NZF>::n1>()>(in, m.ncols,
                                                                                                 twzf);
  __syncthreads();
  if (deriv == 3) {
    // spectral d/dz before the fold: multiply by i G_z of the fine frequency
    for (int i = threadIdx.x; i < NZF * 2 * TX; i += blockDim.x) {
      const int zf = i / (2 * TX), c = i - zf * (2 * TX);
      if (c >= m.ncols) continue;
      const T g = gfac * (T)sgn_idx(zf, NZF);
      const V v = in[zf * PI + c];
      in[zf * PI + c] = mkc<V>(-g * v.y, g * v.x);
    }
    __syncthreads();
  }
  const bool splitrow = m.nyy;
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int kz = i / TX, c = i - kz * TX;
    if (c >= tw) { acc[kz * PA + c] = mkc<V>(0, 0); continue; }
    V v = acc[kz * PA + c];   // staged kinetic term
    const bool nyz = (kz == NZ / 2);
    const int fz = kz <= NZ / 2 ? kz : kz + (NZF - NZ);
    const bool split = splitrow || (c == m.nyx_i);
    if (cplx) {
      // complex bands: the "+" fine position only (idxFineGrid pick)
      v = cadd(v, in[fz * PI + c]);
    } else if (!split) {
      if (nyz) v = cadd(v, cscale(cadd(in[(NZ / 2) * PI + c], in[(NZF - NZ / 2) * PI + c]), (T)0.5));
      else v = cadd(v, in[fz * PI + c]);
    } else {
      const int cp = c, cm = splitrow ? TX + c : TX;
      if (nyz) v = cadd(v, cscale(cadd(in[(NZ / 2) * PI + cp], in[(NZF - NZ / 2) * PI + cm]), (T)0.5));
      else v = cadd(v, cscale(cadd(in[fz * PI + cp], in[fz * PI + cm]), (T)0.5));
    }
    // wavefunction cut-off filter (MultSpinor's exit filter): coefficients with
    // |G|^2/2 above the cut-off are zero in the output spectrum
    if (fmask && fmask[(long)kz * nplane + (long)ky * n0 + kx0 + c] == (T)0) v = mkc<V>(0, 0);
    acc[kz * PA + c] = v;
  }
  __syncthreads();
  smem_fft_cb<NZ, +1, PA, 1>(acc, tw, twz);
  __syncthreads();
  V* Dp = D + (long)p * NZ * nplane + (long)ky * n0 + kx0;
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int z = i / TX, c = i - z * TX;
    if (c < tw) Dp[z * nplane + c] = acc[z * PA + c];
  }
}

// z pencils for the Teter preconditioner: FFT z, * teter / N_c, IFFT z
template <typename T, int NZ, int TX>
__global__ void __launch_bounds__(PENCIL_THREADS, sizeof(T) == 4 ? 4 : 1)
k_zteter(VT<T>* __restrict__ A, const T* __restrict__ teter, int n0, int n1, T inv_nc, const VT<T>* twz_g) {
  using V = VT<T>;
  constexpr int PI = TX + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* in = reinterpret_cast<V*>(smraw);
  V* twz = in + NZ * PI;
  load_tw(twz, twz_g, NZ);
  const int ky = blockIdx.x, kx0 = blockIdx.y * TX, p = blockIdx.z;
  const int tw = min(TX, n0 - kx0);
  const long nplane = (long)n0 * n1;
  V* Ap = A + (long)p * NZ * nplane;
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int z = i / TX, c = i - z * TX;
    in[z * PI + c] = (c < tw) ? Ap[z * nplane + (long)ky * n0 + kx0 + c] : mkc<V>(0, 0);
  }
  __syncthreads();
  smem_fft_cb<NZ, -1, PI, 1>(in, tw, twz);
  __syncthreads();
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int kz = i / TX, c = i - kz * TX;
    if (c < tw) in[kz * PI + c] = cscale(in[kz * PI + c], teter[kz * nplane + (long)ky * n0 + kx0 + c] * inv_nc);
  }
  __syncthreads();
  smem_fft_cb<NZ, +1, PI, 1>(in, tw, twz);
  __syncthreads();
  for (int i = threadIdx.x; i < NZ * TX; i += blockDim.x) {
    const int z = i / TX, c = i - z * TX;
    if (c < tw) Ap[z * nplane + (long)ky * n0 + kx0 + c] = in[z * PI + c];
  }
}

// ---------------------------------------------------------------------------
// Sphere-cut (G-space) mode, Spinor::AddMultSpinorFineR2C complex overload
// (src/SCF/spinor.cpp:528-680).  A band is its coefficients c_s on the half
// sphere 1/2|G|^2 < Ecut in the reference's order (idxCoarseCut,
// src/SCF/fourier.cpp:542-640), complex, sqrt(2) convention (c_0 at G = 0,
// sqrt(2) psi(G) elsewhere).  The G-space grid N is the fine grid of the
// slot box n = N/2, so the sphere (|m_d| <= n_d/2) sits in the same
// [pair][z][ky slot][kx slot] layout the fine-plane kernel works on.  The
// pair field is Z(G) = psi_a(G) + i psi_b(G) over the whole sphere, the
// stored half giving Z(G) = a' + i b' and the mirrored half
// Z(-G) = conj(a') + i conj(b') (a' = c_a / sqrt(2), c_0 real).
//
// Per-row entry lists (built with the context, CSR by block):
//   scatter list, one block per slot row ky: {s+1 at G_s or -(s+1) at -G_s,
//     shared-memory offset fine_z * (n0+1) + kx_slot}
//   gather list, one block per slot row r <= n1/2 and its mirror row: {s,
//     offset of G_s | offset of -G_s << 16} in the block's two-row layout
// ---------------------------------------------------------------------------
// First-pass lane maps of the scatter (FI) and gather (FF) z transforms at the
// fixed pitches n0+1 and 2(n0+1)+1 the entry lists are built for; on the 96
// grid the transform-fastest map saves 7 % / 13 % (FP64) and 4 % (FP32
// gather) of the shared-memory wavefronts in the bank model.
template <typename T, int NZF> struct GsLanes { static constexpr bool FI = false, FF = false; };
template <> struct GsLanes<float, 96> { static constexpr bool FI = false, FF = true; };
template <> struct GsLanes<double, 96> { static constexpr bool FI = true, FF = true; };

__device__ __forceinline__ int mirror_slot(int s, int n) {
  return s == 0 ? 0 : (s == n / 2 ? n : (s == n ? n / 2 : n - s));
}

// sphere scatter + inverse z transform of one slot row (all kx slots) of a pair
template <typename T, int N0, int N1, int NZF>
__global__ void __launch_bounds__(PENCIL_THREADS, sizeof(T) == 4 ? 4 : 2)
k_gs_zinv(const T* __restrict__ psi, int ld, int nband, int band0, const int* __restrict__ rows,
          const int2* __restrict__ ent, VT<T>* __restrict__ B, const VT<T>* twzf_g) {
  using V = VT<T>;
  constexpr int nsx = N0 + 1, nsy = N1 + 1;
  constexpr int PI = nsx;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* in = reinterpret_cast<V*>(smraw);   // [NZF][PI]
  V* twz = in + NZF * PI;
  load_tw(twz, twzf_g, NZF);
  const int ky = blockIdx.x, p = blockIdx.y;
  const int ba = band0 + 2 * p, bb = ba + 1;
  const bool hb = bb < nband;
  const V* pa = reinterpret_cast<const V*>(psi + (long)ba * ld);
  const V* pb = reinterpret_cast<const V*>(psi + (long)(hb ? bb : ba) * ld);
  for (int i = threadIdx.x; i < NZF * PI; i += blockDim.x) in[i] = mkc<V>(0, 0);
  __syncthreads();
  const T r2 = (T)0.70710678118654752440;
  const int e1 = rows[ky + 1];
  for (int e = rows[ky] + threadIdx.x; e < e1; e += blockDim.x) {
    const int2 en = ent[e];
    const int m = en.x;
    const int s = (m > 0 ? m : -m) - 1;
    V a = pa[s];
    V b = hb ? pb[s] : mkc<V>(0, 0);
    T f = r2;
    if (s == 0) { a.y = 0; b.y = 0; f = 1; }
    V z;
    if (m > 0) z = mkc<V>(f * (a.x - b.y), f * (a.y + b.x));
    else z = mkc<V>(f * (a.x + b.y), f * (b.x - a.y));
    in[en.y] = z;
  }
  __syncthreads();
  smem_fft_cb<NZF, +1, PI, 1, GsLanes<T, NZF>::FI>(in, nsx, twz);
  __syncthreads();
  V* Bp = B + (long)p * NZF * nsy * nsx + (long)ky * nsx;
  for_rows_cols(NZF, nsx, [&](int z, int kx) { Bp[(long)z * nsy * nsx + kx] = in[z * PI + kx]; });
}

// forward z transform of a slot row and its mirror row, pair unpack at the
// stored sphere points, sqrt(2) and the kinetic term ekin_s c_s:
// out_s (+)= ekin_s c_s + f_s (Vpsi)(G_s),  f_0 = 1, f_s = sqrt(2)
template <typename T, int N0, int N1, int NZF>
__global__ void __launch_bounds__(PENCIL_THREADS)
k_gs_zfwd(const VT<T>* __restrict__ B, const T* __restrict__ psi, int ld, T* __restrict__ out, int ldo, int nband,
          int band0, int accumulate, const int* __restrict__ rows, const int2* __restrict__ ent,
          const T* __restrict__ ekin, const VT<T>* twzf_g) {
  using V = VT<T>;
  constexpr int nsx = N0 + 1, nsy = N1 + 1;
  constexpr int PI = 2 * nsx + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* in = reinterpret_cast<V*>(smraw);   // [NZF][PI]: row r in columns [0, nsx), its mirror in [nsx, 2 nsx)
  V* twz = in + NZF * PI;
  load_tw(twz, twzf_g, NZF);
  const int r = blockIdx.x, p = blockIdx.y;
  const int rm = mirror_slot(r, N1);
  const int nrow = (rm == r) ? 1 : 2;
  const V* Bp = B + (long)p * NZF * nsy * nsx;
  for_rows_cols(NZF, nrow * nsx, [&](int z, int j) {
    const int row = j < nsx ? r : rm, kx = j < nsx ? j : j - nsx;
    cp_async(&in[z * PI + j], &Bp[((long)z * nsy + row) * nsx + kx]);
  });
  cp_async_wait_all();
  __syncthreads();
  smem_fft_cb<NZF, -1, PI, 1, GsLanes<T, NZF>::FF>(in, nrow * nsx, twz);
  __syncthreads();
  const int ba = band0 + 2 * p, bb = ba + 1;
  const bool hb = bb < nband;
  const V* pa = reinterpret_cast<const V*>(psi + (long)ba * ld);
  const V* pb = reinterpret_cast<const V*>(psi + (long)(hb ? bb : ba) * ld);
  V* oa = reinterpret_cast<V*>(out + (long)ba * ldo);
  V* ob = reinterpret_cast<V*>(out + (long)(hb ? bb : ba) * ldo);
  const T sq2 = (T)1.41421356237309504880;
  const int e1 = rows[r + 1];
  for (int e = rows[r] + threadIdx.x; e < e1; e += blockDim.x) {
    const int2 en = ent[e];
    const int s = en.x;
    // G_s and its mirror -G_s (in the other row of the block, or the same row for r == rm)
    const V y = in[en.y & 0xffff];
    const V ym = in[(unsigned)en.y >> 16];
    const T f = s == 0 ? (T)1 : sq2;
    const T hf = (T)0.5 * f;
    const T ek = ekin[s];
    const V ca = pa[s];
    V va = mkc<V>(hf * (y.x + ym.x) + ek * ca.x, hf * (y.y - ym.y) + ek * ca.y);
    if (accumulate) va = cadd(va, oa[s]);
    oa[s] = va;
    if (hb) {
      const V cb = pb[s];
      V vb = mkc<V>(hf * (y.y + ym.y) + ek * cb.x, hf * (ym.x - y.x) + ek * cb.y);
      if (accumulate) vb = cadd(vb, ob[s]);
      ob[s] = vb;
    }
  }
}

// ---------------------------------------------------------------------------
// coarse plane inverse: D -> hpsi (two real bands)
// ---------------------------------------------------------------------------
template <typename T, int N0, int N1, bool CPLX = false>
__global__ void __launch_bounds__(PLANE_THREADS)
k_cxy_inv(const VT<T>* __restrict__ D, T* __restrict__ out, int ldo, int nband, int band0, int accumulate,
          const VT<T>* twx_g, const VT<T>* twy_g) {
  using V = VT<T>;
  using PL = PlaneLayout<T, N0, N1>;
  constexpr int P0 = PL::P0;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* pl = reinterpret_cast<V*>(smraw);
  V* twx = pl + N1 * P0;
  V* twy = twx + N0;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  const int z = blockIdx.x, p = blockIdx.y;
  const int N2 = gridDim.x;
  const long ntot_plane = (long)N0 * N1;
  const V* Dp = D + ((long)p * N2 + z) * ntot_plane;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
    const int y = i / N0, x = i - y * N0;
    cp_async(&pl[y * P0 + x], &Dp[i]);
  }
  cp_async_wait_all();
  __syncthreads();
  smem_fft_cb<N1, +1, P0, 1, PL::FC>(pl, N0, twy);
  __syncthreads();
  smem_fft_cb<N0, +1, 1, P0, PL::FR>(pl, N1, twx);
  __syncthreads();
  if (CPLX) {
    V* oc = reinterpret_cast<V*>(out) + (long)(band0 + p) * ldo + z * ntot_plane;
    for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
      const int y = i / N0, x = i - y * N0;
      const V v = pl[y * P0 + x];
      oc[i] = accumulate ? cadd(oc[i], v) : v;
    }
    return;
  }
  const int ba = band0 + 2 * p, bb = ba + 1;
  T* oa = out + (long)ba * ldo + z * ntot_plane;
  T* ob = (bb < nband) ? out + (long)bb * ldo + z * ntot_plane : nullptr;
  for (int i = threadIdx.x; i < N0 * N1; i += blockDim.x) {
    const int y = i / N0, x = i - y * N0;
    const V v = pl[y * P0 + x];
    if (accumulate) {
      oa[i] += v.x;
      if (ob) ob[i] += v.y;
    } else {
      oa[i] = v.x;
      if (ob) ob[i] = v.y;
    }
  }
}

// ---------------------------------------------------------------------------
// host-side launch plan for one (precision, grid) instantiation
// ---------------------------------------------------------------------------
// Records a launch; when profiling is on, brackets it with events on the stream.

template <typename T> static int fplane_cr(int NXF, int NYF) {
  // rows per chunk so that S + R (+ twiddles) fit in ~200 KB of shared memory
  const size_t vs = sizeof(T) * 2;
  const size_t S = (size_t)NYF * (NXF / 2 + 1) * vs;
  const size_t budget = 200 * 1024;
  int best = 1;
  for (int cr = 1; cr <= NYF; ++cr) {
    if (NYF % cr) continue;
    if (S + (size_t)cr * (NXF + 1) * vs + (NXF + NYF) * vs <= budget) best = cr;
  }
  return best;
}

template <typename T, int N0, int N1, int N2>
struct Plan {
  static constexpr int TX = PencilTile<T, N0>::v;
  static constexpr int TXF = TX;   // z-fold tile width
  using V = VT<T>;
  static constexpr int NF0 = 2 * N0, NF1 = 2 * N1, NF2 = 2 * N2;

  static int chunk_rows() { return fplane_cr<T>(NF0, NF1); }

  static size_t sm_cxy() { return sizeof(V) * (N1 * PlaneLayout<T, N0, N1>::P0 + N0 + N1); }
  static size_t sm_zpad() { return sizeof(V) * (N2 * (TX + 1) + NF2 * (2 * TX + 1) + N2 + NF2); }
  static size_t sm_zfold() { return sizeof(V) * (NF2 * (2 * TXF + 1) + N2 * (TXF + 1) + N2 + NF2); }
  static size_t sm_zteter() { return sizeof(V) * (N2 * (TX + 1) + N2); }
  static size_t sm_exx_inv() { return sm_cxy() + sizeof(T) * N0 * N1; }
  static size_t sm_floc() {
    return sizeof(V) * ((size_t)NF1 * (N0 + 1) + NF0 + NF1 + (size_t)(FLOC_THREADS / 32) * FftGroup<NF0>::f * (NF0 + 1));
  }
  template <int VAR = 0> static size_t sm_floc2() {
    using LY = FlocLayoutVar<T, NF0, NF1, VAR>;
    return sizeof(V) * ((size_t)floc_s_size<LY, NF1, NF1 / SplitVar<NF1, VAR>::n1>() + NF0 + NF1 +
                        (size_t)(FLOC_THREADS / 32) * (32 / SplitVar<NF0, VAR>::n1) * LY::PR);
  }
  // the fused fine-plane kernel in the context's radix decomposition
  static void launch_floc2(pw_ctx* c, V* BC, const T* vt, T inv_nf, int nblk, cudaStream_t st) {
    const T* vp = reinterpret_cast<const T*>(c->vperm.p);
    if (c->fft_variant == 2 && (vp || !VpermLayout<T, NF0, NF1>::OK))
      k_floc2<T, NF0, NF1, 2><<<dim3(NF2, nblk), FLOC_THREADS, sm_floc2<2>(), st>>>(BC, vt, inv_nf, tw(c, 3), tw(c, 4),
                                                                                   vp);
    else if (c->fft_variant == 1)
      k_floc2<T, NF0, NF1, 1><<<dim3(NF2, nblk), FLOC_THREADS, sm_floc2<1>(), st>>>(BC, vt, inv_nf, tw(c, 3), tw(c, 4),
                                                                                   nullptr);
    else
      k_floc2<T, NF0, NF1, 0><<<dim3(NF2, nblk), FLOC_THREADS, sm_floc2<0>(), st>>>(BC, vt, inv_nf, tw(c, 3), tw(c, 4),
                                                                                   nullptr);
  }
  // pw_ctx::vperm from pw_ctx::vtot (the lane order of VpermLayout)
  static int vperm_build(pw_ctx* c, cudaStream_t st) {
    using PL = VpermLayout<T, NF0, NF1>;
    if (!PL::OK || !c->vtot.p) return PW_OK;
    int rc = c->vperm.alloc((size_t)PL::PLANE * NF2 * sizeof(T));
    if (rc) return rc;
    k_vperm<T, NF0, NF1><<<148 * 4, 256, 0, st>>>(reinterpret_cast<const T*>(c->vtot.p),
                                                   reinterpret_cast<T*>(c->vperm.p), NF2);
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }
  static size_t sm_fplane(int cr) {
    return sizeof(V) * ((size_t)NF1 * (N0 + 1) + (size_t)cr * (NF0 + 1) + NF0 + NF1);
  }

  static int set_attrs() {
    static PerDeviceOnce once;
    if (once.done()) return PW_OK;
    const int cr = chunk_rows();
    PWB_CUDA(cudaFuncSetAttribute(k_fplane<T, NF0, NF1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_fplane(cr)));
    PWB_CUDA(cudaFuncSetAttribute(k_fplane<T, NF0, NF1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_fplane(cr)));
    PWB_CUDA(cudaFuncSetAttribute(k_zpad<T, N2, NF2, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_zpad()));
    PWB_CUDA(cudaFuncSetAttribute(k_zfold<T, N2, NF2, TXF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_zfold()));
    PWB_CUDA(cudaFuncSetAttribute(k_cxy_fwd<T, N0, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
    PWB_CUDA(cudaFuncSetAttribute(k_cxy_inv<T, N0, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
    PWB_CUDA(cudaFuncSetAttribute(k_zteter<T, N2, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_zteter()));
    PWB_CUDA(cudaFuncSetAttribute(k_floc<T, NF0, NF1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc()));
    PWB_CUDA(cudaFuncSetAttribute(k_floc2<T, NF0, NF1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc2<0>()));
    PWB_CUDA(cudaFuncSetAttribute(k_floc2<T, NF0, NF1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc2<1>()));
    PWB_CUDA(cudaFuncSetAttribute(k_floc2<T, NF0, NF1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc2<2>()));
    PWB_CUDA(cudaFuncSetAttribute(k_floc<T, NF0, NF1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc()));
    once.mark();
    return PW_OK;
  }

  static const V* tw(pw_ctx* c, int i) { return reinterpret_cast<const V*>(c->tw[i].p); }

  // one batch of npair band pairs starting at band0
  static int hpsi_batch(pw_ctx* c, const T* psi, int ld, T* out, int ldo, int nband, int band0, int npair,
                        int accumulate, cudaStream_t st) {
    int rc = set_attrs();
    if (rc) return rc;
    // MultSpinor's exit filter applies to an overwriting call (a3 = P H psi)
    const bool filt = c->wfn_filter && !accumulate;
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    V* K = reinterpret_cast<V*>(c->s_k.p);
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    V* Wp = reinterpret_cast<V*>(c->s_wp.p);
    V* W = reinterpret_cast<V*>(c->s_w.p);
    const T inv_nc = (T)(1.0 / (double)c->ntot);
    const T inv_nf = (T)(1.0 / (double)c->ntotf);
    const int ntx = (N0 + TX - 1) / TX;
    // dense projector mode: Q D Q^T psi depends on psi only, so its GEMMs run
    // on a second stream while the FFT chain runs (their first output goes to
    // the rows of out, which k_cxy_inv then accumulates into after the join);
    // with pw_profile on they run after it, so each kernel is timed alone
    const int nbnl = std::min(2 * npair, nband - band0);
    const bool dense_nl = c->nl_mode == PW_NL_DENSE && c->have_nl && c->nproj > 0 && nbnl > 0;
    cudaStream_t sn = nullptr;
    if (dense_nl && c->nl_overlap && !c->prof_on) {
      if (!c->nl_st) PWB_CUDA(cudaStreamCreateWithFlags(&c->nl_st, cudaStreamNonBlocking));
      if (!c->nl_fork) PWB_CUDA(cudaEventCreateWithFlags(&c->nl_fork, cudaEventDisableTiming));
      if (!c->nl_join) PWB_CUDA(cudaEventCreateWithFlags(&c->nl_join, cudaEventDisableTiming));
      sn = c->nl_st;
      PWB_CUDA(cudaEventRecord(c->nl_fork, st));
      PWB_CUDA(cudaStreamWaitEvent(sn, c->nl_fork, 0));
      if ((rc = dense_apply(c, nl_set(c, filt), psi + (long)band0 * ld, ld, out + (long)band0 * ldo, ldo, nbnl, sn,
                            accumulate))) {
        cudaStreamWaitEvent(st, c->nl_fork, 0);
        return rc;
      }
      PWB_CUDA(cudaEventRecord(c->nl_join, sn));
    }
    { Launch L_(c, st, KK_CXY_FWD);
    k_cxy_fwd<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(psi, ld, nband, band0, AD, tw(c, 0), tw(c, 1)); }
    { Launch L_(c, st, KK_ZPAD);
    k_zpad<T, N2, NF2, TX><<<dim3(N1, ntx, npair), PENCIL_THREADS, sm_zpad(), st>>>(
        AD, K, BC, reinterpret_cast<const T*>(c->ekin.p), N0, N1, inv_nc, tw(c, 2), tw(c, 5)); }
    if (c->nl_mode == PW_NL_DENSE) {
      { Launch L_(c, st, KK_FPLANE_APPLY);
      launch_floc2(c, BC, reinterpret_cast<const T*>(c->vtot.p), inv_nf, npair, st); }
      { Launch L_(c, st, KK_ZFOLD);
      k_zfold<T, N2, NF2, TXF><<<dim3(N1, (N0 + TXF - 1) / TXF, npair), PENCIL_THREADS, sm_zfold(), st>>>(
          BC, K, AD, N0, N1, tw(c, 2), tw(c, 5), 0, (T)0, 0, filt ? reinterpret_cast<const T*>(c->wmask.p) : nullptr); }
      if (sn) PWB_CUDA(cudaStreamWaitEvent(st, c->nl_join, 0));
      { Launch L_(c, st, KK_CXY_INV);
      k_cxy_inv<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(AD, out, ldo, nband, band0,
                                                                          sn ? 1 : accumulate, tw(c, 0), tw(c, 1)); }
      PWB_CUDA(cudaGetLastError());
      if (dense_nl && !sn)
        if ((rc = dense_apply(c, nl_set(c, filt), psi + (long)band0 * ld, ld, out + (long)band0 * ldo, ldo, nbnl, st)))
          return rc;
      return exchange_batch(c, psi, ld, out, ldo, nband, band0, npair, st, filt);
    }
    NLArgs nl{};
    const int cr = chunk_rows();
    nl.cr = cr;
    nl.nchunk = NF1 / cr;
    nl.present = c->have_nl && c->nl.nent > 0;
    int natom = 0, nslot = 0;
    if (nl.present) {
      nl.ent_xy = reinterpret_cast<const int*>(c->nl.ent_xy.p);
      nl.ent_beta = c->nl.ent_beta.p;
      nl.tile_slot = reinterpret_cast<const int*>(c->nl.tile_slot.p);
      nl.slot_atom = reinterpret_cast<const int*>(c->nl.slot_atom.p);
      nl.slot_ent = reinterpret_cast<const int*>(c->nl.slot_ent.p);
      nl.nent = c->nl.nent;
      nl.npmax = c->nl.npmax;
      natom = c->nl.natom;
      nslot = c->nl.nslot;
      if (c->nl.cr != cr) { set_error("projector tables built for another chunk size"); return PW_EINVAL; }
      { Launch L_(c, st, KK_FPLANE_GATHER);
    k_fplane<T, NF0, NF1, false><<<dim3(NF2, npair), PLANE_THREADS, sm_fplane(cr), st>>>(
          BC, reinterpret_cast<const T*>(c->vtot.p), nl, Wp, W, natom, nslot, inv_nf, tw(c, 3), tw(c, 4)); }
      const int nthr = 128;
      { Launch L_(c, st, KK_NL_REDUCE);
    k_nl_reduce<T><<<dim3((natom * nl.npmax + nthr - 1) / nthr, npair), nthr, 0, st>>>(
          Wp, W, reinterpret_cast<const int*>(c->nl.atom_slot.p), reinterpret_cast<const int*>(c->nl.atom_slot_list.p),
          reinterpret_cast<const T*>(c->nl.wgt.p), natom, nslot, nl.npmax); }
    }
    { Launch L_(c, st, KK_FPLANE_APPLY);
    k_fplane<T, NF0, NF1, true><<<dim3(NF2, npair), PLANE_THREADS, sm_fplane(cr), st>>>(
        BC, reinterpret_cast<const T*>(c->vtot.p), nl, Wp, W, natom, nslot, inv_nf, tw(c, 3), tw(c, 4)); }
    { Launch L_(c, st, KK_ZFOLD);
    k_zfold<T, N2, NF2, TXF><<<dim3(N1, (N0 + TXF - 1) / TXF, npair), PENCIL_THREADS, sm_zfold(), st>>>(
        BC, K, AD, N0, N1, tw(c, 2), tw(c, 5), 0, (T)0, 0, filt ? reinterpret_cast<const T*>(c->wmask.p) : nullptr); }
    { Launch L_(c, st, KK_CXY_INV);
    k_cxy_inv<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(AD, out, ldo, nband, band0, accumulate, tw(c, 0), tw(c, 1)); }
    PWB_CUDA(cudaGetLastError());
    return exchange_batch(c, psi, ld, out, ldo, nband, band0, npair, st, filt);
  }

  // exact exchange of the batch's bands: the ACE operator (two GEMMs) or the
  // full pair-FFT exchange, depending on the context's hybrid mode
  static int exchange_batch(pw_ctx* c, const T* psi, int ld, T* out, int ldo, int nband, int band0, int npair,
                            cudaStream_t st, bool filt = false) {
    const int nb = std::min(2 * npair, nband - band0);
    if (nb <= 0 || c->exx_mode == PW_EXX_OFF) return PW_OK;
    if (c->exx_mode == PW_EXX_ACE) {
      if (c->ace_n == 0) return PW_OK;
      return dense_apply(c, ace_set(c, filt), psi + (long)band0 * ld, ld, out + (long)band0 * ldo, ldo, nb, st);
    }
    if (c->gs) return gs_exx_apply(c, psi + (long)band0 * ld, ld, nb, out + (long)band0 * ldo, ldo, 1, st);
    int rc = exx_apply(c, psi + (long)band0 * ld, ld, nb, out + (long)band0 * ldo, ldo, 1, st);
    if (rc || !filt) return rc;
    // the pair-FFT exchange has no fused filter: one explicit P pass over the
    // batch's output bands (the local, kinetic and projector parts are already
    // in the filtered space, and P is idempotent)
    const void* saved = c->teter_tab;
    c->teter_tab = c->wmask.p;
    rc = teter_batch(c, out, ldo, out, ldo, nband, band0, npair, 0, st);
    c->teter_tab = saved;
    return rc;
  }

  // the projector matrix; with the filter the accumulating product reads P Q
  static DenseSet nl_set(pw_ctx* c, bool filt = false) {
    return DenseSet{c->q.p, c->qd.p, c->q_bf.p, filt ? c->qtf_bf.p : c->qt_bf.p, c->nproj, c->nproj_pad,
                    filt ? c->qf.p : c->q.p};
  }
  static DenseSet ace_set(pw_ctx* c, bool filt = false) {
    return DenseSet{c->ace_xi.p, c->ace_qd.p, c->ace_bf.p, filt ? c->acef_t_bf.p : c->ace_t_bf.p, c->ace_n,
                    c->ace_npad, filt ? c->acef_xi.p : c->ace_xi.p};
  }

  // out (+)= V_x psi, AddMultSpinorEXX (src/SCF/spinor.cpp:682-781): for every
  // band k and exchange orbital j, out_k -= alpha f_j phi_j (1/N_c) IFFT(v FFT(psi_k phi_j)).
  // Two orbitals share one complex field (v is real and even, so the real and
  // imaginary parts stay separate); batches of (band, orbital pair) fields.
  static int exx_apply(pw_ctx* c, const T* psi, int ld, int nb, T* out, int ldo, int accumulate, cudaStream_t st) {
    int rc = set_attrs();
    if (rc) return rc;
    static PerDeviceOnce attr;
    if (!attr.done()) {
      PWB_CUDA(cudaFuncSetAttribute(k_exx_fwd<T, N0, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
      PWB_CUDA(cudaFuncSetAttribute(k_exx_inv<T, N0, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_exx_inv()));
      attr.mark();
    }
    const int nphi = c->exx_nphi;
    if (nphi == 0 || nb == 0) {
      if (!accumulate && nb > 0)
        PWB_CUDA(cudaMemset2DAsync(out, (size_t)ldo * sizeof(T), 0, (size_t)c->ntot * sizeof(T), nb, st));
      return PW_OK;
    }
    const long nt = c->ntot;
    const int njp = (nphi + 1) / 2;
    const long cap = std::max<long>(1, (long)(c->exx_scratch_bytes / ((size_t)nt * sizeof(V))));
    const int jc = (int)std::min<long>(njp, std::max<long>(1, cap / nb));
    const int kc = (int)std::max<long>(1, std::min<long>(nb, cap / jc));
    if ((rc = c->s_exx.alloc((size_t)kc * jc * nt * sizeof(V)))) return rc;
    V* A = reinterpret_cast<V*>(c->s_exx.p);
    const T* phi = reinterpret_cast<const T*>(c->exx_phi.p);
    const T* wj = reinterpret_cast<const T*>(c->exx_w.p);
    const T* kern = reinterpret_cast<const T*>(c->exx_kern.p);
    const T inv_nc = (T)(1.0 / (double)nt);
    const int ntx = (N0 + TX - 1) / TX;
    for (int k0 = 0; k0 < nb; k0 += kc) {
      const int nk = std::min(kc, nb - k0);
      for (int jp0 = 0; jp0 < njp; jp0 += jc) {
        const int nj = std::min(jc, njp - jp0);
        { Launch L_(c, st, KK_EXX);
        k_exx_fwd<T, N0, N1><<<dim3(N2, nk * nj), PLANE_THREADS, sm_cxy(), st>>>(
            psi, ld, k0, phi, (int)nt, 2 * jp0, nphi, nj, A, tw(c, 0), tw(c, 1)); }
        { Launch L_(c, st, KK_EXX);
        k_zteter<T, N2, TX><<<dim3(N1, ntx, nk * nj), PENCIL_THREADS, sm_zteter(), st>>>(A, kern, N0, N1, inv_nc, tw(c, 2)); }
        { Launch L_(c, st, KK_EXX);
        k_exx_inv<T, N0, N1><<<dim3(N2, nk), PLANE_THREADS, sm_exx_inv(), st>>>(
            A, nj, phi, (int)nt, 2 * jp0, nphi, wj, out, ldo, k0, (accumulate || jp0 > 0) ? 1 : 0, tw(c, 0),
            tw(c, 1)); }
        PWB_CUDA(cudaGetLastError());
      }
    }
    return PW_OK;
  }

  // H psi += Q diag(qd) Q^T psi  for nb bands (column-major, ld); Q is the
  // coarse projector matrix or the ACE vectors (qd = -1)
  // out (+)= Q D Q^T psi: acc 1 accumulates into out, 0 overwrites it
  static int dense_apply(pw_ctx* c, const DenseSet& ds, const T* psi, int ld, T* out, int ldo, int nb,
                         cudaStream_t st, int acc = 1) {
    if constexpr (std::is_same<T, float>::value) {
      return dense_apply_tc(c, ds, psi, ld, out, ldo, nb, st, acc);
    } else {
    cublasHandle_t h = (cublasHandle_t)c->blas;
    if (cublasSetStream(h, st) != CUBLAS_STATUS_SUCCESS) { set_error("cublasSetStream failed"); return PW_ECUDA; }
    const int np = ds.np, nt = (int)c->ntot;
    int rc;
    if ((rc = c->s_wq.alloc((size_t)np * nb * sizeof(T)))) return rc;
    T* W = reinterpret_cast<T*>(c->s_wq.p);
    const T* Q = reinterpret_cast<const T*>(ds.q);
    const T one = 1, zero = 0;
    cublasStatus_t r;
    { Launch L_(c, st, KK_LIBGEMM);
      r = cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, np, nb, nt, &one, Q, nt, psi, ld, &zero, W, np); }
    if (r != CUBLAS_STATUS_SUCCESS) { set_error("projector GEMM (Q^T psi) failed"); return PW_ECUDA; }
    { Launch L_(c, st, KK_MISC);
    k_scale_rows<T><<<(unsigned)(((long)np * nb + 255) / 256), 256, 0, st>>>(W, reinterpret_cast<const T*>(ds.qd), np, nb); }
    const T* Qs = reinterpret_cast<const T*>(ds.q_st ? ds.q_st : ds.q);
    { Launch L_(c, st, KK_LIBGEMM);
      r = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nt, nb, np, &one, Qs, nt, W, np, acc ? &one : &zero, out, ldo); }
    if (r != CUBLAS_STATUS_SUCCESS) { set_error("projector GEMM (Q W) failed"); return PW_ECUDA; }
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
    }
  }

  // rho += sum over the batch's bands of w_b |psi_b,fine|^2 (unnormalised)
  static int density_batch(pw_ctx* c, const T* psi, int ld, int nband, int band0, int npair, const double* w,
                           double* rho, cudaStream_t st) {
    int rc = set_attrs();
    if (rc) return rc;
    static PerDeviceOnce attr;
    if (!attr.done()) {
      PWB_CUDA(cudaFuncSetAttribute(k_fdens<T, NF0, NF1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc()));
      attr.mark();
    }
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    const T inv_nc = (T)(1.0 / (double)c->ntot);
    const int ntx = (N0 + TX - 1) / TX;
    { Launch L_(c, st, KK_DENSITY);
    k_cxy_fwd<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(psi, ld, nband, band0, AD, tw(c, 0), tw(c, 1)); }
    { Launch L_(c, st, KK_DENSITY);
    k_zpad<T, N2, NF2, TX><<<dim3(N1, ntx, npair), PENCIL_THREADS, sm_zpad(), st>>>(
        AD, nullptr, BC, reinterpret_cast<const T*>(c->ekin.p), N0, N1, inv_nc, tw(c, 2), tw(c, 5)); }
    const int ppc = std::max(1, std::min(8, npair));
    { Launch L_(c, st, KK_DENSITY);
    k_fdens<T, NF0, NF1><<<dim3(NF2, (npair + ppc - 1) / ppc), FLOC_THREADS, sm_floc(), st>>>(
        BC, npair, ppc, w + 2 * (band0 / 2), rho, tw(c, 3), tw(c, 4)); }
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }

  // FP32 context: split-BF16 tcgen05 GEMMs
  static int dense_apply_tc(pw_ctx* c, const DenseSet& ds, const float* psi, int ld, float* out, int ldo, int nb,
                            cudaStream_t st, int acc = 1) {
    const int np = ds.np, nt = (int)c->ntot, npp = ds.npp;
    // bf16 row stride: a multiple of 8 elements (16-byte TMA rows); the tensor
    // maps cover K = nt, so the pad is never read
    const long ntp = (nt + 7) / 8 * 8;
    int rc;
    if ((rc = c->s_psi_bf.alloc((size_t)2 * nb * ntp * 2))) return rc;
    if ((rc = c->s_w_bf.alloc((size_t)2 * nb * npp * 2))) return rc;
    char* pb = (char*)c->s_psi_bf.p;
    char* wb = (char*)c->s_w_bf.p;
    { Launch L_(c, st, KK_MISC);
    if ((rc = split_bf16(psi, ld, nt, nb, pb, pb + (size_t)nb * ntp * 2, ntp, 1.0f, st))) return rc; }
    // W^T[b][l] = d_l * sum_g Q[l][g] psi[b][g]   (split-K, deterministic reduce)
    SplitOperand A{ds.q_bf, (const char*)ds.q_bf + (size_t)np * ntp * 2, np, ntp};
    SplitOperand B{pb, pb + (size_t)nb * ntp * 2, nb, ntp};
    ReduceOut ro;
    ro.transpose = 1;
    ro.row_scale = reinterpret_cast<const float*>(ds.qd);
    ro.bf_hi = wb;
    ro.bf_lo = wb + (size_t)nb * npp * 2;
    ro.ldb = npp;
    { Launch L_(c, st, KK_GRAM);
    if ((rc = gemm_tn_reduce(A, B, nt, c->gemm_terms, c->s_ws, ro, st, c->gemm_bn))) return rc; }
    // out[b][g] += sum_l QT[g][l] W^T[b][l]  (tile rows = grid points: coalesced stores)
    SplitOperand W{wb, wb + (size_t)nb * npp * 2, nb, npp};
    SplitOperand QT{ds.qt_bf, (const char*)ds.qt_bf + (size_t)nt * npp * 2, nt, npp};
    { Launch L_(c, st, KK_GRAM);
    if ((rc = gemm_tn_store(QT, W, np, c->gemm_terms, out, ldo, acc, st, 1, c->gemm_bn_store))) return rc; }
    return PW_OK;
  }

  // complex bands at Bloch vector k (Spinor::AddMultSpinorFine, complex
  // version, src/SCF/spinor_complex.cpp:292-542): one band per complex field,
  // idxFineGrid placement, kinetic 1/2 |k+G|^2, projectors with the Bloch phase
  static int hpsi_batch_k(pw_ctx* c, const V* psi, int ld, V* out, int ldo, int band0, int nb, int accumulate,
                          cudaStream_t st, int fpk = 1 << 30, const T* ekin_all = nullptr, const V* qk_all = nullptr) {
    int rc = set_attrs();
    if (rc) return rc;
    static PerDeviceOnce attr;
    if (!attr.done()) {
      PWB_CUDA(cudaFuncSetAttribute(k_cxy_fwd<T, N0, N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
      PWB_CUDA(cudaFuncSetAttribute(k_cxy_inv<T, N0, N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
      attr.mark();
    }
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    V* K = reinterpret_cast<V*>(c->s_k.p);
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    const T inv_nc = (T)(1.0 / (double)c->ntot);
    const T inv_nf = (T)(1.0 / (double)c->ntotf);
    const int ntx = (N0 + TX - 1) / TX;
    const T* pr = reinterpret_cast<const T*>(psi);
    { Launch L_(c, st, KK_CXY_FWD);
    k_cxy_fwd<T, N0, N1, true><<<dim3(N2, nb), PLANE_THREADS, sm_cxy(), st>>>(pr, ld, 0, band0, AD, tw(c, 0), tw(c, 1)); }
    { Launch L_(c, st, KK_ZPAD);
    k_zpad<T, N2, NF2, TX><<<dim3(N1, ntx, nb), PENCIL_THREADS, sm_zpad(), st>>>(
        AD, K, BC, ekin_all ? ekin_all : reinterpret_cast<const T*>(c->ekin_k.p), N0, N1, inv_nc, tw(c, 2), tw(c, 5),
        1, band0, fpk, ekin_all ? c->ntot : 0); }
    { Launch L_(c, st, KK_FPLANE_APPLY);
    launch_floc2(c, BC, reinterpret_cast<const T*>(c->vtot.p), inv_nf, nb, st); }
    { Launch L_(c, st, KK_ZFOLD);
    k_zfold<T, N2, NF2, TXF><<<dim3(N1, (N0 + TXF - 1) / TXF, nb), PENCIL_THREADS, sm_zfold(), st>>>(
        BC, K, AD, N0, N1, tw(c, 2), tw(c, 5), 0, (T)0, 1); }
    { Launch L_(c, st, KK_CXY_INV);
    k_cxy_inv<T, N0, N1, true><<<dim3(N2, nb), PLANE_THREADS, sm_cxy(), st>>>(AD, reinterpret_cast<T*>(out), ldo, 0,
                                                                              band0, accumulate, tw(c, 0), tw(c, 1)); }
    PWB_CUDA(cudaGetLastError());
    if (c->nproj == 0 || !(qk_all ? qk_all : c->qk.p)) return PW_OK;
    // V_nl psi = Q diag(d) Q^H psi with the complex coarse projector matrix Q of
    // each k-point, one GEMM pair per k segment of the batch
    const size_t kq_per = kq_bf_bytes(c);
    for (int f = band0; f < band0 + nb;) {
      const int kk = f / fpk;
      const int f1 = (int)std::min<long>(band0 + nb, (long)(kk + 1) * fpk);
      const V* Qk = qk_all ? qk_all + (long)kk * c->nproj * c->ntot : reinterpret_cast<const V*>(c->qk.p);
      const void* qbf = qk_all ? (c->qkb_bf.p ? (const char*)c->qkb_bf.p + (size_t)kk * kq_per : nullptr)
                               : c->qk_bf.p;
      if ((rc = nl_k(c, Qk, qbf, psi + (long)f * ld, ld, out + (long)f * ldo, ldo, f1 - f, st))) return rc;
      f = f1;
    }
    return PW_OK;
  }

  // FP32, tensor cores: V_nl psi as two real split-BF16 GEMMs over the
  // interleaved (re, im) view.  [Re W; Im W] = d o (A1 psi) (K = 2 ntot, split-K
  // reduced, written as the bf16 operand of the next product), then
  // psi_out += A2 [Re W; Im W] (K = 2 nproj) on the grid-major rows.
  static int nl_k_tc(pw_ctx* c, const void* qbf, const float* x, int ld, float* y, int ldo, int nb, cudaStream_t st) {
    const int np = c->nproj, np2 = c->nkp2;
    const long nt = c->ntot, nt2 = 2 * nt;
    const char* a1h = (const char*)qbf;
    const char* a1l = a1h + (size_t)2 * np * nt2 * 2;
    const char* a2h = a1l + (size_t)2 * np * nt2 * 2;
    const char* a2l = a2h + (size_t)nt2 * np2 * 2;
    int rc;
    if ((rc = c->s_psi_bf.alloc((size_t)2 * nb * nt2 * 2))) return rc;
    if ((rc = c->s_w_bf.alloc((size_t)2 * nb * np2 * 2))) return rc;
    char* pb = (char*)c->s_psi_bf.p;
    char* wb = (char*)c->s_w_bf.p;
    PWB_CUDA(cudaMemsetAsync(wb, 0, (size_t)2 * nb * np2 * 2, st));
    { Launch L_(c, st, KK_MISC);
    if ((rc = split_bf16(x, 2L * ld, (int)nt2, nb, pb, pb + (size_t)nb * nt2 * 2, nt2, 1.0f, st))) return rc; }
    SplitOperand A{a1h, a1l, 2 * np, nt2};
    SplitOperand B{pb, pb + (size_t)nb * nt2 * 2, nb, nt2};
    ReduceOut ro;
    ro.transpose = 1;
    ro.row_scale = reinterpret_cast<const float*>(c->qdk2.p);
    ro.bf_hi = wb;
    ro.bf_lo = wb + (size_t)nb * np2 * 2;
    ro.ldb = np2;
    { Launch L_(c, st, KK_GRAM);
    if ((rc = gemm_tn_reduce(A, B, (int)nt2, c->gemm_terms, c->s_ws, ro, st, c->gemm_bn))) return rc; }
    SplitOperand W{wb, wb + (size_t)nb * np2 * 2, nb, np2};
    SplitOperand QT{a2h, a2l, (int)nt2, np2};
    { Launch L_(c, st, KK_GRAM);
    if ((rc = gemm_tn_store(QT, W, 2 * np, c->gemm_terms, y, 2L * ldo, 1, st, 1, c->gemm_bn_store))) return rc; }
    return PW_OK;
  }

  static int nl_k(pw_ctx* c, const V* Q, const void* qbf, const V* x, int ld, V* y, int ldo, int nb,
                  cudaStream_t st) {
    int rc;
    if constexpr (std::is_same<T, float>::value) {
      if (!qbf) { set_error("k-point projector bf16 copies missing"); return PW_ENOTREADY; }
      return nl_k_tc(c, qbf, reinterpret_cast<const float*>(x), ld, reinterpret_cast<float*>(y), ldo, nb, st);
    } else {
    cublasHandle_t h = (cublasHandle_t)c->blas;
    if (cublasSetStream(h, st) != CUBLAS_STATUS_SUCCESS) { set_error("cublasSetStream failed"); return PW_ECUDA; }
    const int np = c->nproj, nt = (int)c->ntot;
    if ((rc = c->s_wq.alloc((size_t)np * nb * sizeof(V)))) return rc;
    V* W = reinterpret_cast<V*>(c->s_wq.p);
    cublasStatus_t r;
    { Launch L_(c, st, KK_LIBGEMM);
      const cuDoubleComplex one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
      r = cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, np, nb, nt, &one, (const cuDoubleComplex*)Q, nt,
                      (const cuDoubleComplex*)x, ld, &zero, (cuDoubleComplex*)W, np); }
    if (r != CUBLAS_STATUS_SUCCESS) { set_error("projector GEMM (Q^H psi) failed"); return PW_ECUDA; }
    { Launch L_(c, st, KK_MISC);
    k_scale_rows_c<T><<<(unsigned)(((long)np * nb + 255) / 256), 256, 0, st>>>(W, reinterpret_cast<const T*>(c->qdk.p),
                                                                                np, nb); }
    { Launch L_(c, st, KK_LIBGEMM);
      const cuDoubleComplex one = make_cuDoubleComplex(1, 0);
      r = cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nt, nb, np, &one, (const cuDoubleComplex*)Q, nt,
                      (const cuDoubleComplex*)W, np, &one, (cuDoubleComplex*)y, ldo); }
    if (r != CUBLAS_STATUS_SUCCESS) { set_error("projector GEMM (Q W) failed"); return PW_ECUDA; }
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
    }
  }

  // complex coarse projectors at Bloch vector k: q_l = T(conj(e^{i k.d}) beta_l),
  // one projector per complex field, into Qout (complex, leading dimension ntot)
  static int build_q_k(pw_ctx* c, const int* d_idx, const double* d_beta, const double* d_disp, const long* d_pio,
                       const long* d_pbo, const int* d_pnp, int nproj, const double kv[3], V* Qout, cudaStream_t st) {
    int rc = set_attrs();
    if (rc) return rc;
    static PerDeviceOnce attr;
    if (!attr.done()) {
      PWB_CUDA(cudaFuncSetAttribute(k_cxy_inv<T, N0, N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cxy()));
      attr.mark();
    }
    const int cap = c->pair_cap;                 // complex fields per pass
    const long nf = c->ntotf;
    DevBuf fields;
    if ((rc = fields.alloc((size_t)2 * cap * nf * sizeof(T)))) return rc;
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    const T inv_nf = (T)(1.0 / (double)c->ntotf);
    for (int l0 = 0; l0 < nproj; l0 += cap) {
      const int nl = std::min(cap, nproj - l0);
      PWB_CUDA(cudaMemsetAsync(fields.p, 0, (size_t)2 * nl * nf * sizeof(T), st));
      k_scatter_beta_k<T><<<dim3(64, nl), 256, 0, st>>>(reinterpret_cast<T*>(fields.p), nf, d_idx, d_beta, d_disp, d_pio,
                                                         d_pbo, d_pnp, l0, nproj, kv[0], kv[1], kv[2]);
      k_floc<T, NF0, NF1, 1><<<dim3(NF2, nl), FLOC_THREADS, sm_floc(), st>>>(
          BC, nullptr, reinterpret_cast<const T*>(fields.p), nf, inv_nf, tw(c, 3), tw(c, 4));
      k_zfold<T, N2, NF2, TXF><<<dim3(N1, (N0 + TXF - 1) / TXF, nl), PENCIL_THREADS, sm_zfold(), st>>>(
          BC, nullptr, AD, N0, N1, tw(c, 2), tw(c, 5), 0, (T)0, 1);
      k_cxy_inv<T, N0, N1, true><<<dim3(N2, nl), PLANE_THREADS, sm_cxy(), st>>>(
          AD, reinterpret_cast<T*>(Qout), (int)c->ntot, 0, l0, 0, tw(c, 0), tw(c, 1));
      PWB_CUDA(cudaGetLastError());
    }
    PWB_CUDA(cudaStreamSynchronize(st));
    return PW_OK;
  }

  // Build q_l = T(beta_l) for all projectors with the fine->coarse half of
  // the pipeline, two projectors per complex field.
  static int build_q(pw_ctx* c, const int* d_idx, const double* d_beta, const long* d_pio, const long* d_pbo,
                     const int* d_pnp, int nproj, cudaStream_t st, int deriv = 0, T* Qout = nullptr) {
    int rc = set_attrs();
    if (rc) return rc;
    const int cap = c->pair_cap;                 // pairs per pass
    const long nf = c->ntotf;
    DevBuf fields;
    if ((rc = fields.alloc((size_t)2 * cap * nf * sizeof(T)))) return rc;
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    T* Q = Qout ? Qout : reinterpret_cast<T*>(c->q.p);
    const T inv_nf = (T)(1.0 / (double)c->ntotf);
    const T gx = (T)(2 * M_PI / c->L[0]), gy = (T)(2 * M_PI / c->L[1]), gz = (T)(2 * M_PI / c->L[2]);
    for (int l0 = 0; l0 < nproj; l0 += 2 * cap) {
      const int nl = std::min(2 * cap, nproj - l0);
      const int npair = (nl + 1) / 2;
      PWB_CUDA(cudaMemsetAsync(fields.p, 0, (size_t)2 * npair * nf * sizeof(T), st));
      k_scatter_beta<T><<<dim3(64, nl), 256, 0, st>>>(reinterpret_cast<T*>(fields.p), nf, d_idx, d_beta, d_pio, d_pbo, d_pnp, l0, nproj);
      k_floc<T, NF0, NF1, 1><<<dim3(NF2, npair), FLOC_THREADS, sm_floc(), st>>>(
          BC, nullptr, reinterpret_cast<const T*>(fields.p), nf, inv_nf, tw(c, 3), tw(c, 4), deriv,
          deriv == 1 ? gx : gy);
      k_zfold<T, N2, NF2, TXF><<<dim3(N1, (N0 + TXF - 1) / TXF, npair), PENCIL_THREADS, sm_zfold(), st>>>(BC, nullptr, AD, N0, N1, tw(c, 2),
                                                                                     tw(c, 5), deriv, gz);
      k_cxy_inv<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(AD, Q, (int)c->ntot, nproj, l0, 0, tw(c, 0), tw(c, 1));
      PWB_CUDA(cudaGetLastError());
    }
    PWB_CUDA(cudaStreamSynchronize(st));
    return PW_OK;
  }

  static int teter_batch(pw_ctx* c, const T* r, int ld, T* out, int ldo, int nband, int band0, int npair,
                         int accumulate, cudaStream_t st) {
    int rc = set_attrs();
    if (rc) return rc;
    V* AD = reinterpret_cast<V*>(c->s_ad.p);
    const T inv_nc = (T)(1.0 / (double)c->ntot);
    const int ntx = (N0 + TX - 1) / TX;
    { Launch L_(c, st, KK_CXY_FWD);
    k_cxy_fwd<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(r, ld, nband, band0, AD, tw(c, 0), tw(c, 1)); }
    { Launch L_(c, st, KK_ZTETER);
    k_zteter<T, N2, TX><<<dim3(N1, ntx, npair), PENCIL_THREADS, sm_zteter(), st>>>(
        AD, reinterpret_cast<const T*>(c->teter_tab ? c->teter_tab : c->teter.p), N0, N1, inv_nc, tw(c, 2)); }
    { Launch L_(c, st, KK_CXY_INV);
    k_cxy_inv<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(AD, out, ldo, nband, band0, accumulate, tw(c, 0), tw(c, 1)); }
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }

  // Teter preconditioner with caller-provided device scratch (npair complex
  // coarse fields); launches kernels only, allocates nothing.
  static int teter_batch_scratch(pw_ctx* c, const T* r, int ld, T* out, int ldo, int nband, int band0, int npair,
                                 int accumulate, cudaStream_t st, void* scratch) {
    int rc = set_attrs();
    if (rc) return rc;
    V* AD = reinterpret_cast<V*>(scratch);
    const T inv_nc = (T)(1.0 / (double)c->ntot);
    const int ntx = (N0 + TX - 1) / TX;
    c->launches += 3;
    k_cxy_fwd<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(r, ld, nband, band0, AD, tw(c, 0), tw(c, 1));
    k_zteter<T, N2, TX><<<dim3(N1, ntx, npair), PENCIL_THREADS, sm_zteter(), st>>>(
        AD, reinterpret_cast<const T*>(c->teter.p), N0, N1, inv_nc, tw(c, 2));
    k_cxy_inv<T, N0, N1><<<dim3(N2, npair), PLANE_THREADS, sm_cxy(), st>>>(AD, out, ldo, nband, band0, accumulate,
                                                                            tw(c, 0), tw(c, 1));
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }
  // ---- sphere-cut (G-space) contexts: the G-space grid is (NF0, NF1, NF2) ----
  static size_t sm_gs_zinv() { return sizeof(V) * ((size_t)NF2 * (N0 + 1) + NF2); }
  static size_t sm_gs_zfwd() { return sizeof(V) * ((size_t)NF2 * (2 * (N0 + 1) + 1) + NF2); }
  static int set_attrs_gs() {
    static PerDeviceOnce once;
    if (once.done()) return PW_OK;
    int rc = set_attrs();
    if (rc) return rc;
    PWB_CUDA(cudaFuncSetAttribute(k_gs_zinv<T, N0, N1, NF2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm_gs_zinv()));
    PWB_CUDA(cudaFuncSetAttribute(k_gs_zfwd<T, N0, N1, NF2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm_gs_zfwd()));
    PWB_CUDA(cudaFuncSetAttribute(k_fdens<T, NF0, NF1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_floc()));
    once.mark();
    return PW_OK;
  }

  // H c for one batch of npair band pairs of sphere coefficients (real view:
  // 2 ns reals per band): local + kinetic through the slot layout, then the
  // nonlocal V (wgt o Re(V^H c)) (EigenSolver::NonlocalMultX,
  // src/EigenSolver/eigensolver.cpp:471-515) as the dense projector GEMMs on
  // the real view
  static int hpsi_gs_batch(pw_ctx* c, const T* psi, int ld, T* out, int ldo, int nband, int band0, int npair,
                           int accumulate, cudaStream_t st) {
    int rc = set_attrs_gs();
    if (rc) return rc;
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    const int* rows_i = reinterpret_cast<const int*>(c->gs_rows_inv.p);
    const int2* ent_i = reinterpret_cast<const int2*>(c->gs_ent_inv.p);
    const T inv_n = (T)(1.0 / (double)c->ntotf);
    { Launch L_(c, st, KK_ZPAD);
    k_gs_zinv<T, N0, N1, NF2><<<dim3(N1 + 1, npair), PENCIL_THREADS, sm_gs_zinv(), st>>>(
        psi, ld, nband, band0, rows_i, ent_i, BC, tw(c, 5)); }
    { Launch L_(c, st, KK_FPLANE_APPLY);
    launch_floc2(c, BC, reinterpret_cast<const T*>(c->vtot.p), inv_n, npair, st); }
    { Launch L_(c, st, KK_ZFOLD);
    k_gs_zfwd<T, N0, N1, NF2><<<dim3(N1 / 2 + 1, npair), PENCIL_THREADS, sm_gs_zfwd(), st>>>(
        BC, psi, ld, out, ldo, nband, band0, accumulate, reinterpret_cast<const int*>(c->gs_rows_fwd.p),
        reinterpret_cast<const int2*>(c->gs_ent_fwd.p), reinterpret_cast<const T*>(c->gs_ekin.p), tw(c, 5)); }
    PWB_CUDA(cudaGetLastError());
    const int nb = std::min(2 * npair, nband - band0);
    if (c->have_nl && c->nproj > 0 && nb > 0 &&
        (rc = dense_apply(c, nl_set(c), psi + (long)band0 * ld, ld, out + (long)band0 * ldo, ldo, nb, st)))
      return rc;
    return exchange_batch(c, psi, ld, out, ldo, nband, band0, npair, st);
  }

  // rho += sum of w_b |psi_b(r)|^2 from sphere coefficients (CalculateDensity
  // sphere branch, src/SCF/hamiltonian.cpp:2508-2547, unnormalised)
  static int density_gs_batch(pw_ctx* c, const T* psi, int ld, int nband, int band0, int npair, const double* w,
                              double* rho, cudaStream_t st) {
    int rc = set_attrs_gs();
    if (rc) return rc;
    V* BC = reinterpret_cast<V*>(c->s_bc.p);
    { Launch L_(c, st, KK_DENSITY);
    k_gs_zinv<T, N0, N1, NF2><<<dim3(N1 + 1, npair), PENCIL_THREADS, sm_gs_zinv(), st>>>(
        psi, ld, nband, band0, reinterpret_cast<const int*>(c->gs_rows_inv.p),
        reinterpret_cast<const int2*>(c->gs_ent_inv.p), BC, tw(c, 5)); }
    const int ppc = std::max(1, std::min(8, npair));
    { Launch L_(c, st, KK_DENSITY);
    k_fdens<T, NF0, NF1><<<dim3(NF2, (npair + ppc - 1) / ppc), FLOC_THREADS, sm_floc(), st>>>(
        BC, npair, ppc, w + 2 * (band0 / 2), rho, tw(c, 3), tw(c, 4)); }
    PWB_CUDA(cudaGetLastError());
    return PW_OK;
  }
};


// ---------------------------------------------------------------------------
// dispatch over the instantiated grids
// ---------------------------------------------------------------------------

template <typename T, int N0, int N1, int N2>
static int hpsi_thunk(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int nband, int band0, int npair,
                      int acc, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::hpsi_batch(c, (const T*)psi, ld, (T*)out, ldo, nband, band0, npair, acc, st);
}
template <typename T, int N0, int N1, int N2>
static int teter_thunk(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int nband, int band0, int npair,
                       int acc, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::teter_batch(c, (const T*)psi, ld, (T*)out, ldo, nband, band0, npair, acc, st);
}
template <typename T, int N0, int N1, int N2> static int cr_thunk() { return Plan<T, N0, N1, N2>::chunk_rows(); }
template <typename T, int N0, int N1, int N2>
static int teter_scratch_thunk(pw_ctx* c, const void* r, int ld, void* out, int ldo, int nband, int band0, int npair,
                               int acc, cudaStream_t st, void* scratch) {
  return Plan<T, N0, N1, N2>::teter_batch_scratch(c, (const T*)r, ld, (T*)out, ldo, nband, band0, npair, acc, st,
                                                  scratch);
}
template <typename T, int N0, int N1, int N2>
static int dens_thunk(pw_ctx* c, const void* psi, int ld, int nband, int band0, int npair, const double* w, double* rho,
                      cudaStream_t st) {
  return Plan<T, N0, N1, N2>::density_batch(c, (const T*)psi, ld, nband, band0, npair, w, rho, st);
}
template <typename T, int N0, int N1, int N2>
static int buildq_thunk(pw_ctx* c, const int* a, const double* b, const long* d, const long* e, const int* f, int n,
                        cudaStream_t st, int deriv, void* out) {
  return Plan<T, N0, N1, N2>::build_q(c, a, b, d, e, f, n, st, deriv, (T*)out);
}

template <typename T, int N0, int N1, int N2>
static int exx_thunk(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int acc, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::exx_apply(c, (const T*)psi, ld, nb, (T*)out, ldo, acc, st);
}

template <typename T, int N0, int N1, int N2>
static int ace_thunk(pw_ctx* c, const void* psi, int ld, int nb, void* out, int ldo, int acc, cudaStream_t st) {
  (void)acc;
  return Plan<T, N0, N1, N2>::dense_apply(c, Plan<T, N0, N1, N2>::ace_set(c), (const T*)psi, ld, (T*)out, ldo, nb,
                                          st);
}

template <typename T, int N0, int N1, int N2>
static int hpsik_thunk(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int band0, int nb, int acc,
                       cudaStream_t st) {
  using V = VT<T>;
  return Plan<T, N0, N1, N2>::hpsi_batch_k(c, (const V*)psi, ld, (V*)out, ldo, band0, nb, acc, st);
}
template <typename T, int N0, int N1, int N2>
static int hpsikb_thunk(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int band0, int nb, int acc,
                        cudaStream_t st, int fpk, const void* ekin_all, const void* qk_all) {
  using V = VT<T>;
  return Plan<T, N0, N1, N2>::hpsi_batch_k(c, (const V*)psi, ld, (V*)out, ldo, band0, nb, acc, st, fpk,
                                           (const T*)ekin_all, (const V*)qk_all);
}
template <typename T, int N0, int N1, int N2>
static int hpsigs_thunk(pw_ctx* c, const void* psi, int ld, void* out, int ldo, int nband, int band0, int npair,
                        int acc, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::hpsi_gs_batch(c, (const T*)psi, ld, (T*)out, ldo, nband, band0, npair, acc, st);
}
template <typename T, int N0, int N1, int N2>
static int densgs_thunk(pw_ctx* c, const void* psi, int ld, int nband, int band0, int npair, const double* w,
                        double* rho, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::density_gs_batch(c, (const T*)psi, ld, nband, band0, npair, w, rho, st);
}
template <typename T, int N0, int N1, int N2> static int vperm_thunk(pw_ctx* c, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::vperm_build(c, st);
}
template <typename T, int N0, int N1, int N2>
static int buildqk_thunk(pw_ctx* c, const int* a, const double* b, const double* d, const long* e, const long* f,
                         const int* g, int n, const double* kv, void* out, cudaStream_t st) {
  return Plan<T, N0, N1, N2>::build_q_k(c, a, b, d, e, f, g, n, kv, (VT<T>*)out, st);
}

#define PWB_GRID_ENTRY(a, b, c)                                                                          \
  {a, b, c, {hpsi_thunk<double, a, b, c>, hpsi_thunk<float, a, b, c>},                             \
   {teter_thunk<double, a, b, c>, teter_thunk<float, a, b, c>},                                    \
   {cr_thunk<double, a, b, c>, cr_thunk<float, a, b, c>},                                          \
   {buildq_thunk<double, a, b, c>, buildq_thunk<float, a, b, c>},                                  \
   {dens_thunk<double, a, b, c>, dens_thunk<float, a, b, c>},                                      \
   {teter_scratch_thunk<double, a, b, c>, teter_scratch_thunk<float, a, b, c>},                    \
   {exx_thunk<double, a, b, c>, exx_thunk<float, a, b, c>},                                        \
   {ace_thunk<double, a, b, c>, ace_thunk<float, a, b, c>},                                        \
   {hpsik_thunk<double, a, b, c>, hpsik_thunk<float, a, b, c>},                                    \
   {buildqk_thunk<double, a, b, c>, buildqk_thunk<float, a, b, c>},                                \
   {hpsikb_thunk<double, a, b, c>, hpsikb_thunk<float, a, b, c>},                                  \
   {hpsigs_thunk<double, a, b, c>, hpsigs_thunk<float, a, b, c>},                                  \
   {densgs_thunk<double, a, b, c>, densgs_thunk<float, a, b, c>},                                  \
   {vperm_thunk<double, a, b, c>, vperm_thunk<float, a, b, c>}}

}  // namespace pwb
