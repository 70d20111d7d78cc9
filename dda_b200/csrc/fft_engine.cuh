// fft_engine.cuh -- shared-memory mixed-radix FFT for sm_100a.
//
// Lines of a batched transform are staged in shared memory by the calling
// kernel; fft_lines() then runs every radix stage on them in place.  Forward
// transforms are decimation in frequency: natural-order input, output in
// mixed-radix digit-reversed order.  Inverse transforms are decimation in
// time: digit-reversed input, natural-order output.  A forward transform, a
// pointwise product in the permuted order and an inverse transform thus form
// a convolution with no reordering pass; wherever the actual frequency index
// is needed (the D-matrix lookup) it comes from the plan's position table.
// Each butterfly reads and writes the same R shared-memory slots, so threads
// need only R complex registers and one barrier per stage.  Lengths are
// products of 2, 3, 4, 5, 7 and 8 (every even 2,3,5,7-smooth FFT grid the
// DDA grid rule produces, DDA/DDAParams.cpp:45-90).
//
// Sign convention: forward = exp(-2 pi i jk/n), inverse = exp(+2 pi i jk/n),
// both unnormalised (the convention of the FFT plans the reference drives,
// LinAlg/GpuFFTPlan.hpp:176-186 and LinAlg/FFTWPlan.cpp:82,113).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

// sm_100 issues two FP32 lanes per instruction (__fadd2_rn, __ffma2_rn on
// float2): complex adds and real-scalar multiply-adds of complex64 values use
// them, halving the FP32 instruction count of the DFT codelets.  Per lane the
// rounding is that of the scalar operation.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
#define DDA_F32X2 1
#endif

namespace dda {

template <typename T> struct C2;
template <> struct C2<float> { typedef float2 t; };
template <> struct C2<double> { typedef double2 t; };

template <typename T2> __host__ __device__ __forceinline__ T2 czero() {
  T2 r; r.x = 0; r.y = 0; return r;
}
template <typename T2> __host__ __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T2> __host__ __device__ __forceinline__ T2 cadd(T2 a, T2 b) {
#ifdef DDA_F32X2
  if constexpr (std::is_same<T2, float2>::value) return __fadd2_rn(a, b);
#endif
  T2 r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename T2> __host__ __device__ __forceinline__ T2 csub(T2 a, T2 b) {
#ifdef DDA_F32X2
  if constexpr (std::is_same<T2, float2>::value) return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);  // exact -b
#endif
  T2 r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
// acc + c t for a real c
template <typename T, typename T2> __host__ __device__ __forceinline__ T2 caxr(T2 acc, T c, T2 t) {
#ifdef DDA_F32X2
  if constexpr (std::is_same<T2, float2>::value) return __ffma2_rn(make_float2(c, c), t, acc);
#endif
  acc.x += c * t.x; acc.y += c * t.y; return acc;
}
// a complex value in another precision (round to nearest)
template <typename T2, typename S2> __host__ __device__ __forceinline__ T2 cvt(S2 a) {
  T2 r; r.x = a.x; r.y = a.y; return r;
}
template <typename T2> __host__ __device__ __forceinline__ T2 cconj(T2 a) {
  a.y = -a.y; return a;
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename T2> __host__ __device__ __forceinline__ T2 mul_mi(T2 a) {
  T2 r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

constexpr int kMaxStages = 16;

// Device-side description of one transform length.
struct FftPlanDev {
  int n;
  int nst;
  const void* tw;    // exp(-2 pi i k / n), k = 0..n-1, as float2 or double2
  const int* freq;  // frequency index held at each position after a forward transform
  uint32_t packed;  // radices 4 bits each, stage 0 in the low bits (nst <= 8)
};

// ------------------------------------------------------------ DFT cores ----
template <int R, bool INV, typename T2> struct Dft;

template <bool INV, typename T2> struct Dft<2, INV, T2> {
  static __host__ __device__ __forceinline__ void run(T2* v) {
    T2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV, typename T2> struct Dft<4, INV, T2> {
  static __host__ __device__ __forceinline__ void run(T2* v) {
    T2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    T2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV, typename T2> struct Dft<8, INV, T2> {
  static __host__ __device__ __forceinline__ void run(T2* v) {
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
  static __host__ __device__ __forceinline__ double c(int j) { return -0.5; }
  static __host__ __device__ __forceinline__ double s(int j) {
    return j == 1 ? 0.8660254037844386467637232 : -0.8660254037844386467637232;
  }
};
template <> struct OddConst<5> {
  static __host__ __device__ __forceinline__ double c(int j) {
    return (j == 1 || j == 4) ? 0.3090169943749474241022934 : -0.8090169943749474241022934;
  }
  static __host__ __device__ __forceinline__ double s(int j) {
    return j == 1 ? 0.9510565162951535721164393
         : j == 2 ? 0.587785252292473129168706
         : j == 3 ? -0.587785252292473129168706
                  : -0.9510565162951535721164393;
  }
};
template <> struct OddConst<7> {
  static __host__ __device__ __forceinline__ double c(int j) {
    return (j == 1 || j == 6) ? 0.6234898018587335305250049
         : (j == 2 || j == 5) ? -0.2225209339563144042889026
                              : -0.9009688679024191262361023;
  }
  static __host__ __device__ __forceinline__ double s(int j) {
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
  static __host__ __device__ __forceinline__ void run(T2* v) {
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
        re = caxr(re, c, t[m - 1]);
        im = caxr(im, s, u[m - 1]);
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
// All kernels of the library share one dynamic shared-memory window; the FFT
// engine addresses it by element offset so every access is a 32-bit shared
// load/store even though the engine functions are not inlined.
extern __shared__ __align__(16) unsigned char dda_smem[];

template <typename T>
__device__ __forceinline__ typename C2<T>::t* smem_at(int off) {
  return reinterpret_cast<typename C2<T>::t*>(dda_smem) + off;
}

// floor(a / d) for 0 <= a < 2^20 from an FP32 reciprocal: the fraction of
// (a + 0.5)/d stays 0.5/d away from an integer, above the rounding error.
__device__ __forceinline__ int fdiv_i(int a, float rcp) { return (int)(((float)a + 0.5f) * rcp); }

// Barrier of a group of G threads: the warp (G == 32), the CTA (bar == 0),
// or the named barrier `bar` (1..15) shared by G threads of the CTA.
template <int G> __device__ __forceinline__ void group_sync(int bar = 0) {
  if (G == 32) __syncwarp();
  else if (bar == 0) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(G) : "memory");
}

// One radix-R stage over nl lines by a group of G threads (one warp, or the
// whole CTA when G == blockDim.x).  Element e of line l is at shared offset
// soff + l*ls + e*es; the length-n table exp(-2 pi i k/n) is at shared
// offset twoff.  L is the stage's block length: butterfly (block, j) works
// on elements block*L + j + m*L/R, m < R.  Forward (DIF): DFT, then twiddle
// w_L^(j m).  Inverse (DIT): conjugate twiddle, then inverse DFT.  With `lf`
// neighbouring threads take neighbouring lines (column tiles), otherwise
// neighbouring butterflies of one line (row tiles).
template <typename T, int G, bool INV, int R>
__device__ __forceinline__ void stage(int soff, int nl, int ls, int es, bool lf, int n, int L,
                                      int twoff, int tid) {
  typedef typename C2<T>::t T2;
  T2* s = smem_at<T>(0);
  const int S = L / R;
  const int nb = n / R;
  const int total = nl * nb;
  const int tstride = n / L;
  const float rd = 1.0f / (float)(lf ? nl : nb);
  const float rs = 1.0f / (float)S;
  const int mstep = S * es;
#pragma unroll 2
  for (int b = tid; b < total; b += G) {
    const int qq = fdiv_i(b, rd);
    int l, t;
    if (lf) { t = qq; l = b - qq * nl; } else { l = qq; t = b - qq * nb; }
    const int blk = fdiv_i(t, rs);
    const int j = t - blk * S;
    const int base = soff + l * ls + (blk * L + j) * es;
    T2 v[R];
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = s[base + m * mstep];
    if (INV) {
      if (j) {
#pragma unroll
        for (int m = 1; m < R; m++) {
          T2 w = s[twoff + j * m * tstride];
          w.y = -w.y;
          v[m] = cmul(v[m], w);
        }
      }
      Dft<R, true, T2>::run(v);
    } else {
      Dft<R, false, T2>::run(v);
      if (j) {
#pragma unroll
        for (int m = 1; m < R; m++) v[m] = cmul(v[m], s[twoff + j * m * tstride]);
      }
    }
#pragma unroll
    for (int m = 0; m < R; m++) s[base + m * mstep] = v[m];
  }
  group_sync<G>();
}

template <typename T, int G, bool INV>
__device__ __forceinline__ void stage_r(int R, int soff, int nl, int ls, int es, bool lf, int n, int L,
                                        int twoff, int tid) {
  switch (R) {
    case 2: stage<T, G, INV, 2>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
    case 3: stage<T, G, INV, 3>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
    case 4: stage<T, G, INV, 4>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
    case 5: stage<T, G, INV, 5>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
    case 7: stage<T, G, INV, 7>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
    default: stage<T, G, INV, 8>(soff, nl, ls, es, lf, n, L, twoff, tid); break;
  }
}

// All stages of one transform of lines [0, nlines) by a group of G threads,
// entered converged; forward stages run first to last, inverse stages last
// to first.
template <typename T, int G, bool INV>
__device__ __noinline__ void fft_group(int soff, int nlines, int ls, int es, bool lf, int n,
                                       uint32_t packed, int nst, int twoff) {
  const int tid = G == 32 ? (threadIdx.x & 31) : threadIdx.x;
  if (!INV) {
    int L = n;
#pragma unroll 1
    for (int st = 0; st < nst; st++) {
      const int R = (packed >> (4 * st)) & 15;
      stage_r<T, G, false>(R, soff, nlines, ls, es, lf, n, L, twoff, tid);
      L /= R;
    }
  } else {
    int L = 1;
#pragma unroll 1
    for (int st = nst - 1; st >= 0; st--) {
      const int R = (packed >> (4 * st)) & 15;
      L *= R;
      stage_r<T, G, true>(R, soff, nlines, ls, es, lf, n, L, twoff, tid);
    }
  }
}

// Transforms `nlines` lines (layout as for stage()) with the whole CTA and
// returns after a CTA barrier.  With at least one line per warp the lines
// are shared out to warps in contiguous runs and transformed without CTA
// barriers; otherwise all NT threads work through each stage together.
template <typename T, int NT, bool INV>
__device__ __forceinline__ void fft_lines(int soff, int nlines, int ls, int es, bool lf,
                                          const FftPlanDev& pl, int twoff) {
  constexpr int NW = NT / 32;
  if (nlines >= NW) {
    const int w = threadIdx.x >> 5;
    const int per = (nlines + NW - 1) / NW;
    const int l0 = min(nlines, w * per), l1 = min(nlines, l0 + per);
    if (l1 > l0)
      fft_group<T, 32, INV>(soff + l0 * ls, l1 - l0, ls, es, lf, pl.n, pl.packed, pl.nst, twoff);
  } else {
    fft_group<T, NT, INV>(soff, nlines, ls, es, lf, pl.n, pl.packed, pl.nst, twoff);
  }
  __syncthreads();
}

template <typename T, int NT>
__device__ __forceinline__ void fft_lines_dir(int soff, int nlines, int ls, int es, bool lf,
                                              const FftPlanDev& pl, int twoff, bool inverse) {
  if (inverse) fft_lines<T, NT, true>(soff, nlines, ls, es, lf, pl, twoff);
  else fft_lines<T, NT, false>(soff, nlines, ls, es, lf, pl, twoff);
}

// Copies the twiddle table of a plan to shared offset `off` (caller syncs).
template <typename T, int NT>
__device__ __forceinline__ void stage_twiddles(int off, const FftPlanDev& pl) {
  const typename C2<T>::t* src = reinterpret_cast<const typename C2<T>::t*>(pl.tw);
  typename C2<T>::t* dst = smem_at<T>(off);
  for (int i = threadIdx.x; i < pl.n; i += NT) dst[i] = src[i];
}

}  // namespace dda
