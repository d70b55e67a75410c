// Split-BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
//
//   C[m][n] = sum_k A[m][k] * B[n][k]        (both operands K-major)
//
// Each FP32 operand x is split into x_hi = bf16(x), x_lo = bf16(x - x_hi);
// the kernel accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi (optionally
// + A_lo B_lo) in FP32 in tensor memory.  With the operands' bf16 pair
// carrying ~16 mantissa bits this reproduces an FP32 product to ~1e-5
// relative per term.
//
// A persistent CTA (one per SM) walks 128 x BN tiles over K ranges: warp 0
// issues TMA loads into a ring of shared-memory stages, warp 1 issues the
// UMMAs (one elected thread) and commits each stage back to the producer,
// warps 2-5 read the accumulator from TMEM and write the tile.  Two TMEM
// accumulators alternate between tiles so the epilogue of one tile overlaps
// the loads and MMAs of the next.  Two epilogues: a split-K
// partial (deterministically reduced by a second kernel) and a direct
// row-major (optionally accumulating) store.  No cluster multicast is used.
// Every mbarrier wait is bounded: on timeout the kernel records an error code,
// drains its own copies and frees its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "common.hpp"
#include "gemm.hpp"

namespace pwb {

constexpr int GM = 128;             // tile rows (UMMA M)
constexpr int GK = 64;              // K per stage (one 128-byte swizzle row of bf16)
constexpr int GEMM_THREADS = 192;   // 6 warps
constexpr unsigned long long WAIT_NS = 2000000000ull;   // 2 s per wait (default, and the floor of drain waits)

__device__ int g_gemm_error = 0;
// limit of the pipeline waits on this device (pw_set_wait_limit); the drain
// waits at the end of a CTA keep at least WAIT_NS so issued copies always land
__device__ unsigned long long g_wait_ns = WAIT_NS;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// bounded wait; returns false (and records code) on timeout.  drain: a wait
// for copies or MMAs this CTA issued itself, which must finish before exit
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int code, bool drain = false) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long lim = drain ? max(g_wait_ns, WAIT_NS) : g_wait_ns;
  const unsigned long long t0 = gtimer();
  for (unsigned it = 1;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255) == 0 && gtimer() - t0 > lim) break;
  }
  atomicCAS(&g_gemm_error, 0, code);
  return false;
}

// The failure path of the bounded waits, exercised without a fault: one
// thread waits on an mbarrier that nothing arrives on, with the given limit,
// records code 7 when it gives up and returns.
__global__ void k_wait_probe(unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const unsigned long long t0 = gtimer();
  for (unsigned it = 1;; ++it) {
    if (mbar_try(&bar, 0)) return;
    if ((it & 255) == 0 && gtimer() - t0 > limit_ns) break;
  }
  atomicCAS(&g_gemm_error, 0, 7);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1 << 46;                 // descriptor version (sm100)
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}

template <int BN> __host__ __device__ constexpr uint32_t umma_idesc() {
  // F32 accumulate, BF16 A and B, both K-major, N = BN, M = 128
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

template <int BN> struct GemmSmem {
  static constexpr int A_BYTES = GM * GK * 2;          // one bf16 tile of A
  static constexpr int B_BYTES = BN * GK * 2;
  static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int NSTAGE = (3 * STAGE + 2048 <= 226 * 1024) ? 3 : 2;
  static constexpr int BYTES = NSTAGE * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  // two accumulators (double-buffered across the tiles of a persistent CTA)
  static constexpr int TMEM_COLS = 2 * BN <= 64 ? 64 : 2 * BN <= 128 ? 128 : 2 * BN <= 256 ? 256 : 512;
};

struct GemmArgs {
  int M, N, K;           // full problem
  int kchunk;            // K per split (multiple of GK)
  int nsplit;            // K splits
  int nterms;            // 3 or 4 split products
  int epi;               // 0: split-K partial, 1: row-major store, 2: transposed store
  float* ws;             // epi 0: [split][N][M]
  float* C;              // epi 1: C[m*ldc + n], epi 2: C[n*ldc + m]
  long ldc;
  int accumulate;        // epi 1 / 2: C += tile
  int sym;               // symmetric product (A = B): only tiles not strictly below the diagonal
  int ntiles;            // sym: number of those tiles
};

// tiles of column block nt that are not strictly below the diagonal of a
// symmetric product (row tile m0 < n0 + BN)
__host__ __device__ __forceinline__ int sym_tiles_in_col(int nt, int bn, int tilesM) {
  return min(tilesM, ((nt + 1) * bn + GM - 1) / GM);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Persistent CTA: tile t = (m tile, n tile, K split), m fastest, strided by
// gridDim.x.  The stage ring runs across tiles; the accumulator alternates
// between two TMEM buffers so that the epilogue of one tile overlaps the
// loads and MMAs of the next.
template <int BN>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
k_gemm_tn(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
          const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo, GemmArgs g) {
  using SM = GemmSmem<BN>;
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + SM::NSTAGE * SM::STAGE);
  uint64_t* empty = full + SM::NSTAGE;
  uint64_t* tfull = empty + SM::NSTAGE;      // [2] accumulator ready
  uint64_t* tempty = tfull + 2;              // [2] accumulator drained (4 epilogue warps)
  uint64_t* final_bar = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(final_bar + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tilesM = (g.M + GM - 1) / GM, tilesN = (g.N + BN - 1) / BN;
  const int total = (g.sym ? g.ntiles : tilesM * tilesN) * g.nsplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < SM::NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    mbar_init(final_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(SM::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  auto coords = [&](int t, int& m0, int& n0, int& split, int& kbeg, int& nkb) {
    int mt, ntl;
    if (g.sym) {
      // the upper tiles, column block by column block
      int idx = t % g.ntiles;
      split = t / g.ntiles;
      ntl = 0;
      for (int c = sym_tiles_in_col(0, BN, tilesM); idx >= c; c = sym_tiles_in_col(ntl, BN, tilesM)) {
        idx -= c;
        ++ntl;
      }
      mt = idx;
    } else {
      mt = t % tilesM;
      const int r = t / tilesM;
      ntl = r % tilesN;
      split = r / tilesN;
    }
    m0 = mt * GM;
    n0 = ntl * BN;
    kbeg = split * g.kchunk;
    const int kend = min(g.K, kbeg + g.kchunk);
    nkb = (kend > kbeg) ? (kend - kbeg + GK - 1) / GK : 0;
  };

  if (warp == 0) {
    if (lane == 0) {
      long it = 0;
      bool stop = false;
      for (int t = blockIdx.x; t < total && !stop; t += gridDim.x) {
        int m0, n0, split, kbeg, nkb;
        coords(t, m0, n0, split, kbeg, nkb);
        for (int kb = 0; kb < nkb; ++kb) {
          const int s = (int)(it % SM::NSTAGE);
          if (it >= SM::NSTAGE && !mbar_wait(&empty[s], (uint32_t)(((it / SM::NSTAGE) - 1) & 1), 1)) {
            *abort_flag = 1;
            stop = true;
            break;
          }
          if (*abort_flag) { stop = true; break; }
          unsigned char* st = base + s * SM::STAGE;
          mbar_expect_tx(&full[s], SM::STAGE);
          const int kx = kbeg + kb * GK;
          tma_load_2d(st, &tmA_hi, &full[s], kx, m0);
          tma_load_2d(st + SM::A_BYTES, &tmA_lo, &full[s], kx, m0);
          tma_load_2d(st + 2 * SM::A_BYTES, &tmB_hi, &full[s], kx, n0);
          tma_load_2d(st + 2 * SM::A_BYTES + SM::B_BYTES, &tmB_lo, &full[s], kx, n0);
          ++it;
        }
      }
      // drain: every issued stage must have landed before the CTA exits
      for (long k = (it > SM::NSTAGE ? it - SM::NSTAGE : 0); k < it; ++k)
        mbar_wait(&full[k % SM::NSTAGE], (uint32_t)((k / SM::NSTAGE) & 1), 2, true);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = umma_idesc<BN>();
      long it = 0;
      int lt = 0;
      bool ok = true, any = false;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++lt) {
        int m0, n0, split, kbeg, nkb;
        coords(t, m0, n0, split, kbeg, nkb);
        const int buf = lt & 1;
        if (lt >= 2 && !mbar_wait(&tempty[buf], (uint32_t)(((lt >> 1) - 1) & 1), 5)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t acc = tmem + (uint32_t)(buf * BN);
        for (int kb = 0; kb < nkb; ++kb, ++it) {
          const int s = (int)(it % SM::NSTAGE);
          if (!mbar_wait(&full[s], (uint32_t)((it / SM::NSTAGE) & 1), 3)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t sa = smem_u32(base + s * SM::STAGE);
          const uint32_t ahi = sa, alo = sa + SM::A_BYTES;
          const uint32_t bhi = sa + 2 * SM::A_BYTES, blo = bhi + SM::B_BYTES;
#pragma unroll
          for (int kk = 0; kk < GK / 16; ++kk) {
            const uint32_t off = kk * 32;   // 16 bf16 along K inside the swizzled 128-byte row
            const uint32_t acc0 = (kb > 0 || kk > 0) ? 1u : 0u;
            umma_bf16(acc, umma_desc(ahi + off), umma_desc(bhi + off), idesc, acc0);
            umma_bf16(acc, umma_desc(ahi + off), umma_desc(blo + off), idesc, 1u);
            umma_bf16(acc, umma_desc(alo + off), umma_desc(bhi + off), idesc, 1u);
            if (g.nterms > 3) umma_bf16(acc, umma_desc(alo + off), umma_desc(blo + off), idesc, 1u);
          }
          umma_commit(&empty[s]);
          any = true;
        }
        if (!ok) break;
        if (nkb > 0) umma_commit(&tfull[buf]);
        else mbar_arrive(&tfull[buf]);
      }
      if (!ok) *abort_flag = 1;
      // every issued MMA must have completed before the tensor memory is freed
      if (any) {
        umma_commit(final_bar);
        mbar_wait(final_bar, 0, 6, true);
      }
    }
  } else {
    // epilogue warps 2..5: TMEM lanes 32*(warp%4) .. +31
    const int q = warp & 3;
    int lt = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++lt) {
      int m0, n0, split, kbeg, nkb;
      coords(t, m0, n0, split, kbeg, nkb);
      const int buf = lt & 1;
      int ok = 1;
      if (lane == 0) ok = mbar_wait(&tfull[buf], (uint32_t)((lt >> 1) & 1), 4) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      const int ab = __shfl_sync(0xffffffffu, *abort_flag, 0);
      if (!ok || ab) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int row = m0 + q * 32 + lane;
      const bool rowok = row < g.M;
      for (int c0 = 0; c0 < BN; c0 += 32) {
        const int nc = g.N - (n0 + c0);    // valid columns in this chunk (may be <= 0)
        float* dst;
        long cs;                            // column stride of the destination
        if (g.epi == 0) {
          dst = g.ws + ((long)split * g.N + n0 + c0) * g.M + row;
          cs = g.M;
        } else if (g.epi == 2) {
          dst = g.C + (long)(n0 + c0) * g.ldc + row;
          cs = g.ldc;
        } else {
          dst = g.C + (long)row * g.ldc + n0 + c0;
          cs = 1;
        }
        float cv[32];
        const bool acc = g.epi != 0 && g.accumulate;
        if (acc && rowok) {
          // issue the destination loads before the TMEM read so their latencies overlap
#pragma unroll
          for (int j = 0; j < 32; ++j) cv[j] = (j < nc) ? dst[(long)j * cs] : 0.0f;
        }
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr + 16u));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (rowok) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (j < nc) {
              const float v = nkb > 0 ? __uint_as_float(r[j]) : 0.0f;
              dst[(long)j * cs] = acc ? cv[j] + v : v;
            }
          }
        }
      }
      // hand the accumulator back to the MMA warp
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(SM::TMEM_COLS));
  }
}

// fp32 -> (bf16 hi, bf16 lo): nrow rows of ncol values (row stride ld_in) into
// packed rows of stride ld_out; 4 values per thread when the rows allow it
__global__ void k_split_bf16(const float* __restrict__ x, long ld_in, int ncol, int nrow, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo, long ld_out, float scale) {
  const int r = blockIdx.y;
  const float* xr = x + (long)r * ld_in;
  __nv_bfloat16* hr = hi + (long)r * ld_out;
  __nv_bfloat16* lr = lo + (long)r * ld_out;
  const bool vec = ((ncol & 3) == 0) && ((ld_in & 3) == 0) && ((ld_out & 3) == 0) &&
                   (((uintptr_t)x & 15) == 0) && (((uintptr_t)hi & 7) == 0) && (((uintptr_t)lo & 7) == 0);
  if (vec) {
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) * 4; c < ncol; c += gridDim.x * blockDim.x * 4) {
      const float4 v = *reinterpret_cast<const float4*>(xr + c);
      const float a[4] = {v.x * scale, v.y * scale, v.z * scale, v.w * scale};
      __nv_bfloat16 h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        h[j] = __float2bfloat16_rn(a[j]);
        l[j] = __float2bfloat16_rn(a[j] - __bfloat162float(h[j]));
      }
      *reinterpret_cast<uint2*>(hr + c) = *reinterpret_cast<const uint2*>(h);
      *reinterpret_cast<uint2*>(lr + c) = *reinterpret_cast<const uint2*>(l);
    }
  } else {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += gridDim.x * blockDim.x) {
      const float v = xr[c] * scale;
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      hr[c] = h;
      lr[c] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
  }
}

// transpose + split: x is nrow x ncol (row stride ld_in); writes the ncol x nrow
// transpose as bf16 hi/lo with row stride ld_out
__global__ void k_split_bf16_t(const float* __restrict__ x, long ld_in, int ncol, int nrow, __nv_bfloat16* __restrict__ hi,
                               __nv_bfloat16* __restrict__ lo, long ld_out) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    tile[j][threadIdx.x] = (r < nrow && c < ncol) ? x[(long)r * ld_in + c] : 0.f;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (c < ncol && r < nrow) {
      const float v = tile[threadIdx.x][j];
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      hi[(long)c * ld_out + r] = h;
      lo[(long)c * ld_out + r] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
  }
}

// out = sum over splits of ws[split][M][N], with optional per-row / per-column
// scale, written as double or float, directly or transposed.
__global__ void k_splitk_reduce(const float* __restrict__ ws, int nsplit, int M, int N, const float* __restrict__ rs,
                                const float* __restrict__ cs, int transpose, int out_f64, void* out, long ldo,
                                __nv_bfloat16* bhi, __nv_bfloat16* blo, long ldb, int sym_bn) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)M * N) return;
  const int n = (int)(i / M), m = (int)(i - (long)n * M);
  // symmetric product: an entry of a tile strictly below the diagonal was not
  // computed; its mirror (n, m) was
  const bool mirror = sym_bn > 0 && (n / sym_bn) * sym_bn + sym_bn <= (m / GM) * GM;
  const long src = mirror ? (long)m * M + n : (long)n * M + m;
  // four interleaved partial sums (a fixed order: deterministic), eight loads in flight
  const long stride = (long)N * M;
  double s4[4] = {0, 0, 0, 0};
  int k = 0;
#pragma unroll 2
  for (; k + 4 <= nsplit; k += 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) s4[q] += (double)ws[(long)(k + q) * stride + src];
  }
  for (; k < nsplit; ++k) s4[0] += (double)ws[(long)k * stride + src];
  double s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
  if (rs) s *= rs[m];
  if (cs) s *= cs[n];
  const long o = transpose ? (long)n * ldo + m : (long)m * ldo + n;
  if (out) {
    if (out_f64) reinterpret_cast<double*>(out)[o] = s;
    else reinterpret_cast<float*>(out)[o] = (float)s;
  }
  if (bhi) {
    const long ob = transpose ? (long)n * ldb + m : (long)m * ldb + n;
    const float v = (float)s;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    bhi[ob] = h;
    blo[ob] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 2-D bf16 tensor map over rows x K (K contiguous, row stride ld elements), box GK x box_rows
static int make_tmap(CUtensorMap* m, const void* ptr, long rows, long K, long ld, int box_rows) {
  auto enc = get_encode();
  PWB_CHECK(enc, PW_ECUDA, "cuTensorMapEncodeTiled unavailable");
  PWB_CHECK(((uintptr_t)ptr & 15) == 0 && (ld * 2) % 16 == 0, PW_EINVAL, "TMA operand not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  cuuint32_t box[2] = {(cuuint32_t)GK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PWB_CHECK(r == CUDA_SUCCESS, PW_ECUDA, "cuTensorMapEncodeTiled failed");
  return PW_OK;
}

static int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

template <int BN> static int launch_bn(const SplitOperand& A, const SplitOperand& B, const GemmArgs& g, int nsplit,
                                       cudaStream_t st) {
  using SM = GemmSmem<BN>;
  static PerDeviceOnce attr;
  if (!attr.done()) {
    PWB_CUDA(cudaFuncSetAttribute(k_gemm_tn<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM::BYTES));
    attr.mark();
  }
  CUtensorMap ah, al, bh, bl;
  int rc;
  if ((rc = make_tmap(&ah, A.hi, A.rows, g.K, A.ld, GM)) || (rc = make_tmap(&al, A.lo, A.rows, g.K, A.ld, GM)) ||
      (rc = make_tmap(&bh, B.hi, B.rows, g.K, B.ld, BN)) || (rc = make_tmap(&bl, B.lo, B.rows, g.K, B.ld, BN)))
    return rc;
  GemmArgs ga = g;
  ga.nsplit = nsplit;
  const int tilesM = (g.M + GM - 1) / GM, tilesN = (g.N + BN - 1) / BN;
  if (ga.sym) {
    ga.ntiles = 0;
    for (int nt = 0; nt < tilesN; ++nt) ga.ntiles += sym_tiles_in_col(nt, BN, tilesM);
  }
  const long total = (long)(ga.sym ? ga.ntiles : tilesM * tilesN) * nsplit;
  const int grid = (int)std::min<long>(total, num_sms());
  k_gemm_tn<BN><<<grid, GEMM_THREADS, SM::BYTES, st>>>(ah, al, bh, bl, ga);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

static int launch(const SplitOperand& A, const SplitOperand& B, const GemmArgs& g, int BN, int nsplit,
                  cudaStream_t st) {
  switch (BN) {
    case 32: return launch_bn<32>(A, B, g, nsplit, st);
    case 64: return launch_bn<64>(A, B, g, nsplit, st);
    case 96: return launch_bn<96>(A, B, g, nsplit, st);
    case 128: return launch_bn<128>(A, B, g, nsplit, st);
    case 160: return launch_bn<160>(A, B, g, nsplit, st);
    case 192: return launch_bn<192>(A, B, g, nsplit, st);
    case 256: return launch_bn<256>(A, B, g, nsplit, st);
    default: set_error("unsupported GEMM tile width"); return PW_EUNSUPPORTED;
  }
}

static int pick_bn(int N) {
  static const int cands[] = {32, 64, 96, 128, 160, 192, 256};
  // smallest padding waste, then widest tile
  int best = 256;
  long bestw = -1;
  for (int bn : cands) {
    const long pad = ((N + bn - 1) / bn) * (long)bn;
    if (bestw < 0 || pad < bestw || (pad == bestw && bn > best)) { bestw = pad; best = bn; }
  }
  return best;
}

int set_wait_limit_ns(unsigned long long ns) {
  PWB_CUDA(cudaMemcpyToSymbol(g_wait_ns, &ns, sizeof(ns)));
  return PW_OK;
}

int wait_probe(unsigned long long limit_ns, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(limit_ns);
  PWB_CUDA(cudaGetLastError());
  PWB_CUDA(cudaStreamSynchronize(st));
  return gemm_error_check();
}

int gemm_error_check() {
  int h = 0;
  PWB_CUDA(cudaMemcpyFromSymbol(&h, g_gemm_error, sizeof(int)));
  if (h) {
    int z = 0;
    cudaMemcpyToSymbol(g_gemm_error, &z, sizeof(int));
    set_error("tensor-core GEMM pipeline wait timed out (code " + std::to_string(h) + ")");
    return PW_ETIMEOUT;
  }
  return PW_OK;
}

int split_bf16(const float* x, long ld_in, int ncol, int nrow, void* hi, void* lo, long ld_out, float scale,
               cudaStream_t st) {
  if ((long)nrow * ncol == 0) return PW_OK;
  const int bx = std::max(1, std::min((ncol + 1023) / 1024, 64));
  k_split_bf16<<<dim3(bx, nrow), 256, 0, st>>>(x, ld_in, ncol, nrow, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ld_out,
                                                scale);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

int split_bf16_t(const float* x, long ld_in, int ncol, int nrow, void* hi, void* lo, long ld_out, cudaStream_t st) {
  if ((long)nrow * ncol == 0) return PW_OK;
  dim3 grid((ncol + 31) / 32, (nrow + 31) / 32);
  k_split_bf16_t<<<grid, dim3(32, 8), 0, st>>>(x, ld_in, ncol, nrow, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ld_out);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

int gemm_tn_reduce(const SplitOperand& A, const SplitOperand& B, int K, int nterms, DevBuf& ws,
                   const ReduceOut& out, cudaStream_t st, int bn, int sym) {
  const int M = A.rows, N = B.rows;
  if (M == 0 || N == 0) return PW_OK;
  const int BN = bn > 0 ? bn : pick_bn(N);
  sym = sym && M == N;
  int tiles = ((M + GM - 1) / GM) * ((N + BN - 1) / BN);
  if (sym) {
    tiles = 0;
    for (int nt = 0; nt < (N + BN - 1) / BN; ++nt) tiles += sym_tiles_in_col(nt, BN, (M + GM - 1) / GM);
  }
  // enough CTAs to fill the GPU twice over, each with >= 4 K-blocks
  int nsplit = std::max(1, (2 * num_sms() + tiles - 1) / tiles);
  const int maxsplit = std::max(1, (K + 4 * GK - 1) / (4 * GK));
  nsplit = std::min(nsplit, maxsplit);
  // at most KCHUNK_MAX per tensor-memory accumulator: the accumulation of the
  // UMMA partial sums loses low-order bits, so its error grows with the number
  // of k-steps summed in one accumulator (measured: a 124k-long chunk at
  // K = 373,248 was off by 8e-4 relative, 64-block chunks stay below 3e-5)
  constexpr int KCHUNK_MAX = 64 * GK;
  nsplit = std::max(nsplit, (K + KCHUNK_MAX - 1) / KCHUNK_MAX);
  int kchunk = ((K + nsplit - 1) / nsplit + GK - 1) / GK * GK;
  nsplit = (K + kchunk - 1) / kchunk;
  int rc = ws.alloc((size_t)nsplit * M * N * sizeof(float));
  if (rc) return rc;
  GemmArgs g{};
  g.M = M; g.N = N; g.K = K; g.kchunk = kchunk; g.nterms = nterms; g.epi = 0;
  g.ws = reinterpret_cast<float*>(ws.p);
  g.sym = sym;
  if ((rc = launch(A, B, g, BN, nsplit, st))) return rc;
  const long tot = (long)M * N;
  k_splitk_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(
      g.ws, nsplit, M, N, out.row_scale, out.col_scale, out.transpose, out.f64, out.out, out.ldo,
      (__nv_bfloat16*)out.bf_hi, (__nv_bfloat16*)out.bf_lo, out.ldb, sym ? BN : 0);
  PWB_CUDA(cudaGetLastError());
  return PW_OK;
}

int gemm_tn_store(const SplitOperand& A, const SplitOperand& B, int K, int nterms, float* C, long ldc, int accumulate,
                  cudaStream_t st, int transposed, int bn) {
  const int M = A.rows, N = B.rows;
  if (M == 0 || N == 0) return PW_OK;
  const int BN = bn > 0 ? bn : (N >= 256 ? 256 : pick_bn(N));
  GemmArgs g{};
  g.M = M; g.N = N; g.K = K; g.kchunk = ((K + GK - 1) / GK) * GK; g.nterms = nterms; g.epi = transposed ? 2 : 1;
  g.C = C; g.ldc = ldc; g.accumulate = accumulate;
  return launch(A, B, g, BN, 1, st);
}

}  // namespace pwb
