// fft_plan.cuh -- FFTs with compile-time plans.
//
// For the grid lengths of the tuned shapes every stage's radix, block length
// and strides are template constants, so index arithmetic folds into
// immediates and each stage is a fully unrolled register DFT.  Radices up to
// 32 are register codelets built from the prime cores of fft_engine.cuh by a
// Cooley-Tukey split with constant twiddles (Dft<N> below), which cuts the
// number of shared-memory passes to two per axis for lengths up to 256.
// Same conventions as fft_engine.cuh: forward = decimation in frequency
// (output digit-reversed), inverse = decimation in time (input
// digit-reversed), unnormalised.
#pragma once

#include <type_traits>

#include "fft_engine.cuh"

namespace dda {

// ---------------------------------------------- compile-time constants ----
// cos/sin of 2 pi k/n from the Taylor series on |x| <= pi/4 after reduction
// by the octant symmetries, in long double: exact to double precision.
__host__ __device__ constexpr long double ct_sin_small(long double x) {
  long double term = x, sum = x;
  for (int i = 1; i < 14; i++) {
    term *= -x * x / ((2 * i) * (2 * i + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr long double ct_cos_small(long double x) {
  long double term = 1, sum = 1;
  for (int i = 1; i < 14; i++) {
    term *= -x * x / ((2 * i - 1) * (2 * i));
    sum += term;
  }
  return sum;
}
// angle 2 pi k / n, k reduced to [0, n); returns {cos, sin}
struct CtCS {
  long double c, s;
};
__host__ __device__ constexpr CtCS ct_cossin(long long k, long long n) {
  k %= n;
  if (k < 0) k += n;
  // work in units of n/8: octant o and remainder r, angle = (o + r/(n/8)) pi/4
  const long double kPi4 = 0.78539816339744830961566084581987572L;
  const long long k8 = 8 * k;
  const long long o = k8 / n;
  const long double frac = (long double)(k8 - o * n) / (long double)n;  // in [0,1)
  long double x = frac * kPi4;                                           // [0, pi/4)
  long double c = 0, s = 0;
  // angle = o*pi/4 + x
  switch (o) {
    case 0: c = ct_cos_small(x); s = ct_sin_small(x); break;
    case 1: c = ct_sin_small(kPi4 - x); s = ct_cos_small(kPi4 - x); break;
    case 2: c = -ct_sin_small(x); s = ct_cos_small(x); break;
    case 3: c = -ct_cos_small(kPi4 - x); s = ct_sin_small(kPi4 - x); break;
    case 4: c = -ct_cos_small(x); s = -ct_sin_small(x); break;
    case 5: c = -ct_sin_small(kPi4 - x); s = -ct_cos_small(kPi4 - x); break;
    case 6: c = ct_sin_small(x); s = -ct_cos_small(x); break;
    default: c = ct_cos_small(kPi4 - x); s = -ct_sin_small(kPi4 - x); break;
  }
  return CtCS{c, s};
}

template <int I, int N, typename F>
__host__ __device__ __forceinline__ void sfor(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    sfor<I + 1, N>(f);
  }
}

// multiply by exp(-/+ 2 pi i e / n) with compile-time e, n
template <int E, int N, bool INV, typename T2>
__host__ __device__ __forceinline__ T2 cmul_tw(T2 v) {
  typedef decltype(v.x) T;
  constexpr int e = ((E % N) + N) % N;
  if constexpr (e == 0) {
    return v;
  } else if constexpr (4 * e == N) {
    return mul_mi<INV>(v);  // exp(-i pi/2)
  } else if constexpr (2 * e == N) {
    v.x = -v.x; v.y = -v.y;
    return v;
  } else if constexpr (4 * e == 3 * N) {
    return mul_mi<!INV>(v);
  } else {
    constexpr CtCS cs = ct_cossin(-e, N);
    constexpr double c = (double)cs.c;
    constexpr double s = INV ? -(double)cs.s : (double)cs.s;
    T2 w;
    w.x = (T)c;
    w.y = (T)s;
    return cmul(v, w);
  }
}

// ---------------------------------------------- composite codelets --------
__host__ __device__ constexpr bool is_base_radix(int n) { return n == 2 || n == 3 || n == 4 || n == 5 || n == 7 || n == 8; }
__host__ __device__ constexpr int first_factor(int n) {
  return n % 4 == 0 && n != 4 ? 4 : n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n % 5 == 0 ? 5 : 7;
}

// DFT of N values in registers, natural order in and out.  Base radices use
// the cores of fft_engine.cuh; composite N = A*B splits as
// X[k1 + A k2] = sum_n2 w_N^(n2 k1) w_B^(n2 k2) sum_n1 x[B n1 + n2] w_A^(n1 k1).
template <int N, bool INV, typename T2, bool BASE = is_base_radix(N)>
struct DftN;

template <int N, bool INV, typename T2>
struct DftN<N, INV, T2, true> {
  static __host__ __device__ __forceinline__ void run(T2* v) { Dft<N, INV, T2>::run(v); }
};

template <int N, bool INV, typename T2>
struct DftN<N, INV, T2, false> {
  static constexpr int A = first_factor(N);
  static constexpr int B = N / A;
  static __host__ __device__ __forceinline__ void run(T2* x) {
    T2 y[N];
    sfor<0, B>([&](auto n2c) {
      constexpr int n2 = decltype(n2c)::value;
      T2 t[A];
#pragma unroll
      for (int n1 = 0; n1 < A; n1++) t[n1] = x[B * n1 + n2];
      DftN<A, INV, T2>::run(t);
      sfor<0, A>([&](auto k1c) {
        constexpr int k1 = decltype(k1c)::value;
        y[n2 + B * k1] = cmul_tw<n2 * k1, N, INV>(t[k1]);
      });
    });
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      T2 t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; n2++) t[n2] = y[n2 + B * k1];
      DftN<B, INV, T2>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) x[k1 + A * k2] = t[k2];
    }
  }
};

// ------------------------------------------------------------- plans -----
template <int... Rs> struct Plan {
  static constexpr int K = sizeof...(Rs);
  static constexpr int r[K] = {Rs...};
  static __host__ __device__ constexpr int n() {
    int p = 1;
    for (int i = 0; i < K; i++) p *= r[i];
    return p;
  }
  static constexpr int N = n();
  // block length of stage i: N / (R_0 ... R_{i-1})
  static __host__ __device__ constexpr int L(int i) {
    int l = N;
    for (int k = 0; k < i; k++) l /= r[k];
    return l;
  }
  // frequency held at position p after the forward pass
  static __host__ __device__ __forceinline__ int freq_of(int p) {
    constexpr int rr[K] = {Rs...};
    int k = 0, unit = N, mul = 1;
#pragma unroll
    for (int i = 0; i < K; i++) {
      unit /= rr[i];
      const int d = p / unit;
      p -= d * unit;
      k += d * mul;
      mul *= rr[i];
    }
    return k;
  }
  // mixed-radix digit reversal: frequency -> position after the forward pass
  static __host__ __device__ constexpr int pos(int k) {
    int p = 0, rem = k, unit = N;
    for (int i = 0; i < K; i++) {
      unit /= r[i];
      p += (rem % r[i]) * unit;
      rem /= r[i];
    }
    return p;
  }
};

// One stage of plan P applied to one butterfly: R = P::r[I], block length
// L, stride S = L/R; v holds the R elements base + m*S.  Twiddle exponents
// j*m*(N/L) index the length-N table tw (shared memory).
template <typename P, int I, bool INV, typename T2>
__device__ __forceinline__ void butterfly(T2* v, int j, const T2* tw) {
  constexpr int R = P::r[I];
  constexpr int L = P::L(I);
  constexpr int TS = P::N / L;
  if constexpr (L == R) {  // last forward / first inverse stage: no twiddles
    DftN<R, INV, T2>::run(v);
  } else if constexpr (INV) {
    if (j) {
#pragma unroll
      for (int m = 1; m < R; m++) {
        T2 w = tw[j * m * TS];
        w.y = -w.y;
        v[m] = cmul(v[m], w);
      }
    }
    DftN<R, INV, T2>::run(v);
  } else {
    DftN<R, INV, T2>::run(v);
    if (j) {
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = cmul(v[m], tw[j * m * TS]);
    }
  }
}

// Stage-0 twiddles of plan P in butterfly-major order for two-stage plans,
// whose last stage needs none: entry (m - 1) S0 + j = exp(-2 pi i j m / N)
// for m in [1, R0), j in [0, S0), copied from the plan's length-N table (the
// same values as tw[j m]).  Threads that run butterflies j, j+1, ... then
// read consecutive words instead of words j m apart, which fall into the same
// shared-memory banks for even m.
template <typename T, int NT, typename P>
__device__ __forceinline__ void stage_twiddles0(int off, const FftPlanDev& pl) {
  constexpr int R = P::r[0], S0 = P::N / R;
  const typename C2<T>::t* src = reinterpret_cast<const typename C2<T>::t*>(pl.tw);
  typename C2<T>::t* dst = smem_at<T>(off);
  for (int i = threadIdx.x; i < (R - 1) * S0; i += NT) {
    const int m = 1 + i / S0, j = i - (m - 1) * S0;
    dst[i] = src[j * m];
  }
}

// butterfly<P, 0, INV> with the twiddles of stage_twiddles0.
template <typename P, bool INV, typename T2>
__device__ __forceinline__ void butterfly0(T2* v, int j, const T2* t0) {
  constexpr int R = P::r[0];
  constexpr int S0 = P::N / R;
  static_assert(P::K == 2, "butterfly-major stage-0 twiddles are staged for two-stage plans");
  if constexpr (INV) {
    if (j) {
#pragma unroll
      for (int m = 1; m < R; m++) {
        T2 w = t0[(m - 1) * S0 + j];
        w.y = -w.y;
        v[m] = cmul(v[m], w);
      }
    }
    DftN<R, INV, T2>::run(v);
  } else {
    DftN<R, INV, T2>::run(v);
    if (j) {
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = cmul(v[m], t0[(m - 1) * S0 + j]);
    }
  }
}

// Stage I of plan P on nl lines by a group of G threads (tid in [0, G)).
// Element e of line l is at shared offset soff + l*ls + e*es.  Work items are
// (line, butterfly) pairs with the line fastest, so a line tile and a column
// tile both keep every lane busy.
// DIV = 2 (stages I >= 1 only): the line's first half, positions [0, N/2),
// which holds whole blocks of these stages when the first radix is even.
template <typename T, typename P, int I, bool INV, int G, int DIV = 1>
__device__ __forceinline__ void pstage(int soff, int nl, int ls, int es, int twoff, int tid, int bar = 0) {
  typedef typename C2<T>::t T2;
  constexpr int R = P::r[I];
  constexpr int L = P::L(I);
  constexpr int S = L / R;
  constexpr int NB = P::N / R / DIV;  // butterflies per line
  static_assert(DIV == 1 || (I >= 1 && P::r[0] % DIV == 0), "half lines need stage >= 1 and an even first radix");
  T2* s = smem_at<T>(0);
  const T2* tw = s + twoff;
  const int total = nl * NB;
  const int mstep = S * es;
#pragma unroll 2
  for (int b = tid; b < total; b += G) {
    const int t = b / nl, l = b - t * nl;
    const int blk = t / S, j = t - blk * S;
    const int base = soff + l * ls + (blk * L + j) * es;
    T2 v[R];
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = s[base + m * mstep];
    butterfly<P, I, INV>(v, j, tw);
#pragma unroll
    for (int m = 0; m < R; m++) s[base + m * mstep] = v[m];
  }
  group_sync<G>(bar);
}

// Stages [I0, I1) of P, forward in order or inverse in reverse order.
template <typename T, typename P, bool INV, int G, int I0, int I1, int DIV = 1>
__device__ __forceinline__ void pstages(int soff, int nl, int ls, int es, int twoff, int tid, int bar = 0) {
  if constexpr (I0 < I1) {
    if constexpr (!INV) {
      pstage<T, P, I0, false, G, DIV>(soff, nl, ls, es, twoff, tid, bar);
      pstages<T, P, false, G, I0 + 1, I1, DIV>(soff, nl, ls, es, twoff, tid, bar);
    } else {
      pstage<T, P, I1 - 1, true, G, DIV>(soff, nl, ls, es, twoff, tid, bar);
      pstages<T, P, true, G, I0, I1 - 1, DIV>(soff, nl, ls, es, twoff, tid, bar);
    }
  }
}

// Whole transform of nlines lines shared by the CTA's warps (contiguous
// runs; CTA-wide when there are fewer lines than warps), ending with a CTA
// barrier.
// Stages [I0, I1) of P on nlines lines with the whole CTA (one barrier per
// stage), ending with a CTA barrier.
template <typename T, typename P, int NT, bool INV, int I0 = 0, int I1 = P::K>
__device__ __forceinline__ void plines(int soff, int nlines, int ls, int es, int twoff) {
  pstages<T, P, INV, NT, I0, I1>(soff, nlines, ls, es, twoff, threadIdx.x);
}

}  // namespace dda
