// fft_engine.cuh -- shared-memory mixed-radix FFT for sm_100a.
//
// Lines of a batched transform are staged in shared memory by the calling
// kernel; fft_smem() then runs every radix stage of a Stockham autosort FFT
// on them with all threads of the CTA.  Each stage reads its butterfly inputs
// into registers, synchronises, and writes the outputs back in place, so a
// transform needs no second shared-memory buffer.  Lengths are products of
// 2, 3, 4, 5, 7 and 8 (every even 2,3,5,7-smooth FFT grid the DDA grid rule
// produces, DDA/DDAParams.cpp:45-90).
//
// Sign convention: forward = exp(-2 pi i jk/n), inverse = exp(+2 pi i jk/n),
// both unnormalised (the convention of the FFT plans the reference drives,
// LinAlg/GpuFFTPlan.hpp:176-186 and LinAlg/FFTWPlan.cpp:82,113).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dda {

template <typename T> struct C2;
template <> struct C2<float> { typedef float2 t; };
template <> struct C2<double> { typedef double2 t; };

template <typename T2> __device__ __forceinline__ T2 czero() {
  T2 r; r.x = 0; r.y = 0; return r;
}
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) {
  T2 r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) {
  T2 r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
template <typename T2> __device__ __forceinline__ T2 cconj(T2 a) {
  a.y = -a.y; return a;
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename T2> __device__ __forceinline__ T2 mul_mi(T2 a) {
  T2 r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

constexpr int kMaxStages = 16;

// Device-side description of one transform length.
struct FftPlanDev {
  int n;
  int nst;
  int radix[kMaxStages];
  const void* tw;  // exp(-2 pi i k / n), k = 0..n-1, as float2 or double2
};

// ------------------------------------------------------------ DFT cores ----
template <int R, bool INV, typename T2> struct Dft;

template <bool INV, typename T2> struct Dft<2, INV, T2> {
  static __device__ __forceinline__ void run(T2* v) {
    T2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV, typename T2> struct Dft<4, INV, T2> {
  static __device__ __forceinline__ void run(T2* v) {
    T2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    T2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV, typename T2> struct Dft<8, INV, T2> {
  static __device__ __forceinline__ void run(T2* v) {
    typedef decltype(v[0].x) T;
    const T h = (T)0.7071067811865475244008444;
    T2 e[4] = {v[0], v[2], v[4], v[6]};
    T2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV, T2>::run(e);
    Dft<4, INV, T2>::run(o);
    // o[k] *= w8^k, w8 = exp(-/+ i pi/4)
    T2 w1, w3;
    w1.x = h; w1.y = INV ? h : -h;
    w3.x = -h; w3.y = INV ? h : -h;
    o[1] = cmul(o[1], w1);
    o[2] = mul_mi<INV>(o[2]);
    o[3] = cmul(o[3], w3);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

// Odd prime radix via symmetric pairs: y_k = a0 + sum_m C(mk) t_m -/+ i sum_m S(mk) u_m.
template <int R> struct OddConst;
template <> struct OddConst<3> {
  static __device__ __forceinline__ double c(int j) { return -0.5; }
  static __device__ __forceinline__ double s(int j) {
    return j == 1 ? 0.8660254037844386467637232 : -0.8660254037844386467637232;
  }
};
template <> struct OddConst<5> {
  static __device__ __forceinline__ double c(int j) {
    return (j == 1 || j == 4) ? 0.3090169943749474241022934 : -0.8090169943749474241022934;
  }
  static __device__ __forceinline__ double s(int j) {
    return j == 1 ? 0.9510565162951535721164393
         : j == 2 ? 0.587785252292473129168706
         : j == 3 ? -0.587785252292473129168706
                  : -0.9510565162951535721164393;
  }
};
template <> struct OddConst<7> {
  static __device__ __forceinline__ double c(int j) {
    return (j == 1 || j == 6) ? 0.6234898018587335305250049
         : (j == 2 || j == 5) ? -0.2225209339563144042889026
                              : -0.9009688679024191262361023;
  }
  static __device__ __forceinline__ double s(int j) {
    return j == 1 ? 0.7818314824680298087084445
         : j == 2 ? 0.9749279121818236070181317
         : j == 3 ? 0.4338837391175581204757683
         : j == 4 ? -0.4338837391175581204757683
         : j == 5 ? -0.9749279121818236070181317
                  : -0.7818314824680298087084445;
  }
};

template <int R, bool INV, typename T2> struct DftOdd {
  // In place: the pair sums/differences replace v[1..R-1] before the outputs
  // are written back, so no second output array is live.
  static __device__ __forceinline__ void run(T2* v) {
    typedef decltype(v[0].x) T;
    constexpr int H = (R - 1) / 2;
    T2 t[H], u[H];
#pragma unroll
    for (int m = 1; m <= H; m++) {
      t[m - 1] = cadd(v[m], v[R - m]);
      u[m - 1] = csub(v[m], v[R - m]);
    }
    const T2 a0 = v[0];
#pragma unroll
    for (int m = 0; m < H; m++) v[0] = cadd(v[0], t[m]);
#pragma unroll
    for (int k = 1; k <= H; k++) {
      T2 re = a0, im;
      im.x = 0; im.y = 0;
#pragma unroll
      for (int m = 1; m <= H; m++) {
        const T c = (T)OddConst<R>::c((m * k) % R);
        const T s = (T)OddConst<R>::s((m * k) % R);
        re.x += c * t[m - 1].x; re.y += c * t[m - 1].y;
        im.x += s * u[m - 1].x; im.y += s * u[m - 1].y;
      }
      // forward: y_k = re - i im, y_{R-k} = re + i im
      const T2 mi = mul_mi<INV>(im);  // -i*im (fwd) or +i*im (inv)
      v[k] = cadd(re, mi);
      v[R - k] = csub(re, mi);
    }
  }
};
template <bool INV, typename T2> struct Dft<3, INV, T2> : DftOdd<3, INV, T2> {};
template <bool INV, typename T2> struct Dft<5, INV, T2> : DftOdd<5, INV, T2> {};
template <bool INV, typename T2> struct Dft<7, INV, T2> : DftOdd<7, INV, T2> {};

// ------------------------------------------------------------- stages ----
// One Stockham stage on lines [l0, l0+nl) of the shared-memory tile.  Element
// e of line l lives at s[l*ls + e*es].  Butterfly b maps to (line, j) with the
// line index fastest when `line_fast` (column tiles: neighbouring threads touch
// neighbouring addresses) and j fastest otherwise (row tiles).
template <typename T, int NT, int MAXE, bool INV, int R>
__device__ __forceinline__ void fft_stage(typename C2<T>::t* s, int l0, int nl, int ls, int es,
                                          bool line_fast, int n, int Ns,
                                          const typename C2<T>::t* __restrict__ tw) {
  typedef typename C2<T>::t T2;
  constexpr int MB = (MAXE + R - 1) / R;
  const int nb = n / R;
  const int total = nl * nb;
  const int tstride = n / (Ns * R);
  T2 v[MB][R];
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (b < total) {
      int l, j;
      if (line_fast) { l = b % nl; j = b / nl; } else { j = b % nb; l = b / nb; }
      const T2* line = s + (size_t)(l0 + l) * ls;
#pragma unroll
      for (int r = 0; r < R; r++) v[q][r] = line[(j + r * nb) * es];
      if (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; r++) {
          T2 w = tw[k * r * tstride];
          if (INV) w.y = -w.y;
          v[q][r] = cmul(v[q][r], w);
        }
      }
      Dft<R, INV, T2>::run(v[q]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (b < total) {
      int l, j;
      if (line_fast) { l = b % nl; j = b / nl; } else { j = b % nb; l = b / nb; }
      T2* line = s + (size_t)(l0 + l) * ls;
      const int k = j % Ns;
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) line[(base + r * Ns) * es] = v[q][r];
    }
  }
  __syncthreads();
}

// Transforms `nlines` lines of length pl.n held in shared memory (layout as
// for fft_stage).  Lines are processed in chunks of at most NT*MAXE elements
// so every thread holds at most about MAXE elements per stage.  Must be called
// by all NT threads of the CTA after the tile is complete in shared memory
// (the caller's __syncthreads); returns after a final __syncthreads.
template <typename T, int NT, int MAXE, bool INV>
__device__ __noinline__ void fft_smem(typename C2<T>::t* s, int nlines, int ls, int es,
                                      bool line_fast, const FftPlanDev& pl) {
  typedef typename C2<T>::t T2;
  const T2* tw = reinterpret_cast<const T2*>(pl.tw);
  const int n = pl.n;
  int chunk = (NT * MAXE) / n;
  if (chunk < 1) chunk = 1;
#pragma unroll 1
  for (int l0 = 0; l0 < nlines; l0 += chunk) {
    const int nl = min(chunk, nlines - l0);
    int Ns = 1;
#pragma unroll 1
    for (int st = 0; st < pl.nst; st++) {
      const int R = pl.radix[st];
      switch (R) {
        case 2: fft_stage<T, NT, MAXE, INV, 2>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
        case 3: fft_stage<T, NT, MAXE, INV, 3>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
        case 4: fft_stage<T, NT, MAXE, INV, 4>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
        case 5: fft_stage<T, NT, MAXE, INV, 5>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
        case 7: fft_stage<T, NT, MAXE, INV, 7>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
        default: fft_stage<T, NT, MAXE, INV, 8>(s, l0, nl, ls, es, line_fast, n, Ns, tw); break;
      }
      Ns *= R;
    }
  }
}

template <typename T, int NT, int MAXE>
__device__ __forceinline__ void fft_smem_dir(typename C2<T>::t* s, int nlines, int ls, int es,
                                             bool line_fast, const FftPlanDev& pl, bool inverse) {
  if (inverse)
    fft_smem<T, NT, MAXE, true>(s, nlines, ls, es, line_fast, pl);
  else
    fft_smem<T, NT, MAXE, false>(s, nlines, ls, es, line_fast, pl);
}

}  // namespace dda
