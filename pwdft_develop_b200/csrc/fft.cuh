// Shared-memory / register FFT building blocks for sm_100a.
//
// A length-N transform (N = N1*N2, both <= 16) runs as a two-level
// "four-step" FFT inside shared memory: pass 1 does N2 register DFTs of
// length N1 on strided elements and applies the W_N^{j2 k1} twiddles in
// place, pass 2 does N1 register DFTs of length N2 and writes the natural
// order result.  One warp owns F = 32/N1 transforms at a time, so the only
// synchronisation inside a transform is __syncwarp().  Register DFTs are
// fully unrolled at compile time; their twiddles are literal constants.
#pragma once
#include <cuda_runtime.h>
#include <type_traits>

namespace pwb {

template <typename T> struct C2;
template <> struct C2<float> { using t = float2; };
template <> struct C2<double> { using t = double2; };

template <typename V> struct RealOf;
template <> struct RealOf<float2> { using t = float; };
template <> struct RealOf<double2> { using t = double; };

template <typename V> __device__ __forceinline__ V mkc(typename RealOf<V>::t a, typename RealOf<V>::t b) {
  V r; r.x = a; r.y = b; return r;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mkc<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mkc<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  return mkc<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cscale(V a, typename RealOf<V>::t s) { return mkc<V>(a.x * s, a.y * s); }
// multiply by i*sgn
template <int SGN, typename V> __device__ __forceinline__ V cmuli(V a) {
  return SGN > 0 ? mkc<V>(-a.y, a.x) : mkc<V>(a.y, -a.x);
}

template <int R> struct TwR;
#include "twiddle_consts.inc"

template <int I> using ic = std::integral_constant<int, I>;
template <int B, int E, typename F> __device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) { f(ic<B>{}); sfor<B + 1, E>(f); }
}

// W_R^m with sign DIR (DIR=-1 forward e^{-2 pi i m/R}, DIR=+1 backward)
template <int R, int M, int DIR, typename V> __device__ __forceinline__ V twmul(V a) {
  using T = typename RealOf<V>::t;
  constexpr int m = M % R;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (4 * m == R) {
    return cmuli<DIR>(a);
  } else if constexpr (2 * m == R) {
    return mkc<V>(-a.x, -a.y);
  } else if constexpr (4 * m == 3 * R) {
    return cmuli<-DIR>(a);
  } else {
    constexpr double c = TwR<R>::c[m];
    constexpr double s = DIR * TwR<R>::s[m];
    return mkc<V>(a.x * (T)c - a.y * (T)s, a.x * (T)s + a.y * (T)c);
  }
}

// p[k] = w^k for k = 1 .. R-1 (even k: the square of w^{k/2}, odd k: w^{k-1} w),
// each power at most about 2 log2(R) rounded products from w
template <int R, typename V> __device__ __forceinline__ void twiddle_powers(V w, V* p) {
  p[1] = w;
  sfor<2, R>([&](auto kI) {
    constexpr int k = decltype(kI)::value;
    if constexpr (k % 2 == 0) {
      const V h = p[k / 2];
      p[k] = mkc<V>(h.x * h.x - h.y * h.y, (h.x + h.x) * h.y);
    } else {
      p[k] = cmul(p[k - 1], w);
    }
  });
}

template <int R> struct FirstFactor {
  static constexpr int v = (R % 4 == 0 && R != 4) ? 4
                         : (R % 2 == 0 && R != 2) ? 2
                         : (R % 3 == 0 && R != 3) ? 3
                         : (R % 5 == 0 && R != 5) ? 5 : R;
};

// In-place DFT of R elements in registers, natural order in and out.
template <int R, int DIR, typename V> struct DFT {
  static __device__ __forceinline__ void run(V* v) {
    constexpr int A = FirstFactor<R>::v;
    if constexpr (A == R) {
      // prime length: direct O(R^2) with literal twiddles
      V out[R];
      sfor<0, R>([&](auto kI) {
        constexpr int k = decltype(kI)::value;
        V acc = v[0];
        sfor<1, R>([&](auto nI) {
          constexpr int n = decltype(nI)::value;
          acc = cadd(acc, twmul<R, n * k, DIR>(v[n]));
        });
        out[k] = acc;
      });
      sfor<0, R>([&](auto kI) { v[decltype(kI)::value] = out[decltype(kI)::value]; });
    } else {
      constexpr int B = R / A;
      V t[R];
      sfor<0, B>([&](auto bI) {
        constexpr int b = decltype(bI)::value;
        V a_[A];
        sfor<0, A>([&](auto aI) { a_[decltype(aI)::value] = v[B * decltype(aI)::value + b]; });
        DFT<A, DIR, V>::run(a_);
        sfor<0, A>([&](auto kaI) {
          constexpr int ka = decltype(kaI)::value;
          t[ka * B + b] = twmul<R, b * ka, DIR>(a_[ka]);
        });
      });
      sfor<0, A>([&](auto kaI) {
        constexpr int ka = decltype(kaI)::value;
        V c_[B];
        sfor<0, B>([&](auto bI) { c_[decltype(bI)::value] = t[ka * B + decltype(bI)::value]; });
        DFT<B, DIR, V>::run(c_);
        sfor<0, B>([&](auto kbI) { v[ka + A * decltype(kbI)::value] = c_[decltype(kbI)::value]; });
      });
    }
  }
};
template <int DIR, typename V> struct DFT<1, DIR, V> {
  static __device__ __forceinline__ void run(V*) {}
};
template <int DIR, typename V> struct DFT<2, DIR, V> {
  static __device__ __forceinline__ void run(V* v) {
    V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int DIR, typename V> struct DFT<3, DIR, V> {
  static __device__ __forceinline__ void run(V* v) {
    using T = typename RealOf<V>::t;
    const T s = (T)0.8660254037844386;
    V t1 = cadd(v[1], v[2]);
    V t2 = csub(v[0], cscale(t1, (T)0.5));
    V t3 = cscale(csub(v[1], v[2]), s);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, cmuli<DIR>(t3));
    v[2] = csub(t2, cmuli<DIR>(t3));
  }
};
template <int DIR, typename V> struct DFT<4, DIR, V> {
  static __device__ __forceinline__ void run(V* v) {
    V a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    V c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, cmuli<DIR>(d));
    v[3] = csub(b, cmuli<DIR>(d));
  }
};
template <int DIR, typename V> struct DFT<5, DIR, V> {
  static __device__ __forceinline__ void run(V* v) {
    using T = typename RealOf<V>::t;
    const T c1 = (T)TwR<5>::c[1], c2 = (T)TwR<5>::c[2];
    const T s1 = (T)TwR<5>::s[1], s2 = (T)TwR<5>::s[2];
    V a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    V b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    V x0 = v[0];
    V r1 = mkc<V>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    V r2 = mkc<V>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    V i1 = mkc<V>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
    V i2 = mkc<V>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(r1, cmuli<DIR>(i1));
    v[4] = csub(r1, cmuli<DIR>(i1));
    v[2] = cadd(r2, cmuli<DIR>(i2));
    v[3] = csub(r2, cmuli<DIR>(i2));
  }
};

// DFT of R elements in registers whose inputs in the bit mask ZM are known,
// at compile time, to be zero (the padded slots of a coarse spectrum): the
// butterflies that would add a known zero are not emitted.  Same result as
// DFT<R, DIR, V> up to the sign of zero results.
template <int R, int DIR, typename V, unsigned ZM> struct DFTZ {
  static constexpr unsigned ALL = (1u << R) - 1u;
  static constexpr unsigned Z = ZM & ALL;
  static __device__ __forceinline__ void run(V* v) {
    if constexpr (Z == 0) {
      DFT<R, DIR, V>::run(v);
    } else if constexpr (Z == ALL) {
      sfor<0, R>([&](auto kI) { v[decltype(kI)::value] = mkc<V>(0, 0); });
    } else if constexpr (R == 2) {
      // one of the two inputs is zero
      if constexpr (Z & 1u) {
        const V b = v[1];
        v[0] = b;
        v[1] = mkc<V>(-b.x, -b.y);
      } else {
        v[1] = v[0];
      }
    } else if constexpr (FirstFactor<R>::v == R) {
      // prime length: direct sum over the inputs that can be nonzero
      V out[R];
      sfor<0, R>([&](auto kI) {
        constexpr int k = decltype(kI)::value;
        V acc = mkc<V>(0, 0);
        bool first = true;
        sfor<0, R>([&](auto nI) {
          constexpr int n = decltype(nI)::value;
          if constexpr (!((Z >> n) & 1u)) {
            const V term = twmul<R, n * k, DIR>(v[n]);
            acc = first ? term : cadd(acc, term);
            first = false;
          }
        });
        out[k] = acc;
      });
      sfor<0, R>([&](auto kI) { v[decltype(kI)::value] = out[decltype(kI)::value]; });
    } else {
      constexpr int A = FirstFactor<R>::v;
      constexpr int B = R / A;
      V t[R];
      sfor<0, B>([&](auto bI) {
        constexpr int b = decltype(bI)::value;
        constexpr unsigned sub = [] {
          unsigned m = 0;
          for (int a = 0; a < A; ++a)
            if ((Z >> (B * a + b)) & 1u) m |= 1u << a;
          return m;
        }();
        V a_[A];
        sfor<0, A>([&](auto aI) { a_[decltype(aI)::value] = v[B * decltype(aI)::value + b]; });
        DFTZ<A, DIR, V, sub>::run(a_);
        sfor<0, A>([&](auto kaI) {
          constexpr int ka = decltype(kaI)::value;
          t[ka * B + b] = twmul<R, b * ka, DIR>(a_[ka]);
        });
      });
      // a first-stage transform whose inputs were all zero gives zeros
      constexpr unsigned zb = [] {
        unsigned m = 0;
        for (int b = 0; b < B; ++b) {
          bool all = true;
          for (int a = 0; a < A; ++a) all = all && ((Z >> (B * a + b)) & 1u);
          if (all) m |= 1u << b;
        }
        return m;
      }();
      sfor<0, A>([&](auto kaI) {
        constexpr int ka = decltype(kaI)::value;
        V c_[B];
        sfor<0, B>([&](auto bI) { c_[decltype(bI)::value] = t[ka * B + decltype(bI)::value]; });
        DFTZ<B, DIR, V, zb>::run(c_);
        sfor<0, B>([&](auto kbI) { v[ka + A * decltype(kbI)::value] = c_[decltype(kbI)::value]; });
      });
    }
  }
};

// Length split used for each supported 1D size (N1 <= 16, N2 <= 16).
template <int N> struct Split;
#define PWB_SPLIT(N_, N1_) template <> struct Split<N_> { static constexpr int n1 = N1_; };
PWB_SPLIT(8, 2) PWB_SPLIT(12, 3) PWB_SPLIT(16, 4) PWB_SPLIT(20, 4) PWB_SPLIT(24, 4) PWB_SPLIT(30, 5)
PWB_SPLIT(32, 4) PWB_SPLIT(36, 6) PWB_SPLIT(40, 5) PWB_SPLIT(48, 6) PWB_SPLIT(60, 6) PWB_SPLIT(64, 8)
PWB_SPLIT(72, 8) PWB_SPLIT(80, 8) PWB_SPLIT(96, 8) PWB_SPLIT(120, 10) PWB_SPLIT(128, 8) PWB_SPLIT(144, 12)
#undef PWB_SPLIT

// `count` in-place transforms of length N on shared memory.  Element e of
// transform b sits at base[b*bs + e*es].  tw[m] = exp(-2 pi i m / N) for
// m < N, in shared memory.  All threads of the block must call this.
// Explicit work split: warp `warp` of `nw` cooperating warps (a single warp
// with warp = 0, nw = 1 runs a warp-private batch without block barriers).
template <int N, int DIR, typename V>
__device__ __forceinline__ void smem_fft_w(V* base, int count, int es, int bs, const V* tw, int warp, int nw) {
  constexpr int N1 = Split<N>::n1;
  constexpr int N2 = N / N1;
  static_assert(N1 * N2 == N && N1 <= 32, "bad split");
  constexpr int F = 32 / N1;
  const int lane = threadIdx.x & 31;
  for (int g = warp * F; g < count; g += nw * F) {
    // pass 1: DFT_N1 over j1 for each (f, j2), twiddle, store in place
    for (int it = lane; it < F * N2; it += 32) {
      const int f = it / N2, j2 = it - f * N2;
      const int b = g + f;
      if (b < count) {
        V* p = base + (long)b * bs;
        V t[N1];
#pragma unroll
        for (int j1 = 0; j1 < N1; ++j1) t[j1] = p[(N2 * j1 + j2) * es];
        DFT<N1, DIR, V>::run(t);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) {
          V w = tw[j2 * k1];
          if (DIR > 0) w.y = -w.y;
          t[k1] = cmul(t[k1], w);
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) p[(N2 * k1 + j2) * es] = t[k1];
      }
    }
    __syncwarp();
    // pass 2: DFT_N2 over j2 for each (f, k1); natural-order output
    const int f = lane / N1, k1 = lane - f * N1;
    const bool act = (lane < F * N1) && (g + f < count);
    V u[N2];
    V* p = base + (long)(g + f) * bs;
    if (act) {
#pragma unroll
      for (int j2 = 0; j2 < N2; ++j2) u[j2] = p[(N2 * k1 + j2) * es];
      DFT<N2, DIR, V>::run(u);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) p[(k1 + N1 * k2) * es] = u[k2];
    }
    __syncwarp();
  }
}

template <int N, int DIR, typename V>
__device__ __forceinline__ void smem_fft(V* base, int count, int es, int bs, const V* tw) {
  smem_fft_w<N, DIR>(base, count, es, bs, tw, (int)(threadIdx.x >> 5), (int)(blockDim.x >> 5));
}

// Same transform with compile-time element stride ES and batch stride BS:
// addresses fold to 32-bit immediates.  FB puts the transform index on the
// fastest lanes of the first pass (lane -> (f = it % F, j2 = it / F)), which
// spreads a warp's accesses over more banks when BS is small against ES.
// ZIN: first-pass inputs j1 (elements N2 j1 + j2) known to be zero for every
// j2, not read and pruned from the register transforms; DOUT: second-pass
// outputs k2 (elements k1 + N1 k2) never read afterwards, not written (and so
// not computed).  Both 0: the plain transform.
template <int N, int DIR, int ES, int BS, bool FB = false, unsigned ZIN = 0u, unsigned DOUT = 0u, typename V>
__device__ __forceinline__ void smem_fft_c(V* base, int count, const V* tw, int warp, int nw) {
  constexpr int N1 = Split<N>::n1;
  constexpr int N2 = N / N1;
  constexpr int F = 32 / N1;
  constexpr int R1 = (F * N2 + 31) / 32;   // pass-1 rounds per group
  const int lane = threadIdx.x & 31;
  const int f2 = lane / N1, k1_2 = lane - f2 * N1;
  for (int g = warp * F; g < count; g += nw * F) {
#pragma unroll
    for (int r = 0; r < R1; ++r) {
      const int it = lane + 32 * r;
      const int f = FB ? it % F : it / N2, j2 = FB ? it / F : it - f * N2;
      const int b = g + f;
      if (it < F * N2 && b < count) {
        V* p = base + b * BS + j2 * ES;
        V t[N1];
        sfor<0, N1>([&](auto jI) {
          constexpr int j1 = decltype(jI)::value;
          if constexpr ((ZIN >> j1) & 1u) t[j1] = mkc<V>(0, 0);
          else t[j1] = p[N2 * j1 * ES];
        });
        DFTZ<N1, DIR, V, ZIN>::run(t);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) {
          V w = tw[j2 * k1];
          if (DIR > 0) w.y = -w.y;
          t[k1] = cmul(t[k1], w);
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) p[N2 * k1 * ES] = t[k1];
      }
    }
    __syncwarp();
    const bool act = (lane < F * N1) && (g + f2 < count);
    V u[N2];
    V* p = base + (g + f2) * BS;
    if (act) {
#pragma unroll
      for (int j2 = 0; j2 < N2; ++j2) u[j2] = p[(N2 * k1_2 + j2) * ES];
      DFT<N2, DIR, V>::run(u);
    }
    __syncwarp();
    if (act) {
      sfor<0, N2>([&](auto kI) {
        constexpr int k2 = decltype(kI)::value;
        if constexpr (!((DOUT >> k2) & 1u)) p[(k1_2 + N1 * k2) * ES] = u[k2];
      });
    }
    __syncwarp();
  }
}

template <int N, int DIR, int ES, int BS, bool FB = false, unsigned ZIN = 0u, unsigned DOUT = 0u, typename V>
__device__ __forceinline__ void smem_fft_cb(V* base, int count, const V* tw) {
  smem_fft_c<N, DIR, ES, BS, FB, ZIN, DOUT>(base, count, tw, (int)(threadIdx.x >> 5), (int)(blockDim.x >> 5));
}

// Second radix decomposition N = n1 x (N / n1) of the longer lengths, the
// alternative the autotuner times against Split (the fine-plane kernel takes
// either; the other lengths have one).
template <int N> struct SplitAlt { static constexpr int n1 = Split<N>::n1; };
#define PWB_SPLIT_ALT(N_, N1_) template <> struct SplitAlt<N_> { static constexpr int n1 = N1_; };
PWB_SPLIT_ALT(48, 8) PWB_SPLIT_ALT(60, 10) PWB_SPLIT_ALT(64, 16) PWB_SPLIT_ALT(72, 12) PWB_SPLIT_ALT(80, 10)
PWB_SPLIT_ALT(96, 12) PWB_SPLIT_ALT(120, 12) PWB_SPLIT_ALT(128, 16) PWB_SPLIT_ALT(144, 16)
#undef PWB_SPLIT_ALT
template <int N, int VAR> struct SplitVar { static constexpr int n1 = VAR == 1 ? SplitAlt<N>::n1 : Split<N>::n1; };

// Number of transforms one warp processes together for length N.
template <int N> struct FftGroup {
  static constexpr int f = 32 / Split<N>::n1;
};

// Runtime-length dispatch over the supported sizes.  Returns false when N is
// not supported (the host validates sizes before launching).
template <int DIR, typename V>
__device__ __forceinline__ bool smem_fft_rt(int N, V* base, int count, int es, int bs, const V* tw) {
  switch (N) {
#define PWB_CASE(n) case n: smem_fft<n, DIR, V>(base, count, es, bs, tw); return true;
    PWB_CASE(8) PWB_CASE(12) PWB_CASE(16) PWB_CASE(20) PWB_CASE(24) PWB_CASE(30) PWB_CASE(32)
    PWB_CASE(36) PWB_CASE(40) PWB_CASE(48) PWB_CASE(60) PWB_CASE(64) PWB_CASE(72) PWB_CASE(80)
    PWB_CASE(96) PWB_CASE(120) PWB_CASE(128) PWB_CASE(144)
#undef PWB_CASE
    default: return false;
  }
}

__host__ __device__ inline bool fft_len_supported(int n) {
  switch (n) {
    case 8: case 12: case 16: case 20: case 24: case 30: case 32: case 36: case 40: case 48:
    case 60: case 64: case 72: case 80: case 96: case 120: case 128: case 144: return true;
    default: return false;
  }
}

}  // namespace pwb
