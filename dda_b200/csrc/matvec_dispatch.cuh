// matvec_dispatch.cuh -- selection of the matvec kernels for a context: the
// compile-time-planned kernels of matvec_planned.cuh when every grid edge has
// a tuned plan, the runtime-planned kernels of matvec_kernels.cuh otherwise.
#pragma once

#include "matvec_kernels.cuh"
#include "matvec_planned.cuh"
#include "matvec_slot.cuh"
#include "matvec_pair.cuh"

namespace dda {

template <typename T> struct MvKernels {
  typedef typename C2<T>::t T2;
  // x passes over vectors of element type A2 (T2, or double2 for FP64
  // Krylov vectors around an FP32 convolution)
  template <typename A2>
  using XfwdF = void (*)(const A2*, T2*, const uint32_t*, const uint32_t*, const uint32_t*, const T2*, int,
                         MvGeom, FftPlanDev, KrylovState*, int, XPre);
  template <typename A2>
  using XinvF = void (*)(const A2*, A2*, const T2*, const uint32_t*, const uint32_t*, const uint32_t*,
                         const T2*, int, MvGeom, FftPlanDev, KrylovState*, KrylovStep, int);
  typedef XfwdF<T2> XfwdFn;
  typedef XinvF<T2> XinvFn;
  typedef void (*YzFn)(T2*, const T2*, MvGeom, YzGeom, FftPlanDev, FftPlanDev, const KrylovState*, int);
  typedef void (*YrowsFn)(T2*, const T2*, MvGeom, YzGeom, FftPlanDev, const KrylovState*, int);
  typedef void (*ColsFn)(const T2*, T2*, ColGeom, FftPlanDev, int, const KrylovState*, int);
  typedef void (*SlotFn)(T2*, const T2*, MvGeom, SlotGeom, const uint32_t*, int, T2*, FftPlanDev, FftPlanDev,
                         const KrylovState*, int);
  XfwdFn xfwd = nullptr;
  XfwdFn xfwd_pre = nullptr;  // with a solver step in the load (XPre)
  XinvFn xinv = nullptr;
  // FP32 engines: the same over FP64 vectors (mixed precision)
  XfwdF<double2> xfwd_m = nullptr, xfwd_m_pre = nullptr;
  XinvF<double2> xinv_m = nullptr;
  YzFn yz = nullptr;        // fused plane kernel (nullptr: none for this shape)
  YzFn yz2 = nullptr;       // the same kernel run as two groups of half the CTA
  YzFn yz4 = nullptr;       // ... and as four groups of a quarter
  YzFn pair[3] = {};        // a plane per cluster of two CTAs (k_yz_pair), 1 / 2 / 4 groups
  YrowsFn yrows = nullptr;  // split path
  ColsFn cols = nullptr;
  SlotFn slot = nullptr;    // cluster plane kernel for planes beyond shared memory
  bool planned = false;
};


inline bool has_tuned_plan(int n) {
  switch (n) {
#define C(N) case N:
    DDA_TUNED_LENGTHS(C)
#undef C
    return true;
    default: return false;
  }
}

// Fused plane kernel for y = z = N; the HALF variant when the box is exactly
// half the grid in y and z and the first radix is even.
template <typename T, int NTYZ, int N, int GR = 1>
typename MvKernels<T>::YzFn fused_kernel(bool half) {
  typedef typename PlanFor<N>::type P;
  if constexpr (P::r[0] % 2 == 0) {
    if (half) return k_yz_p<T, NTYZ, P, P, true, GR>;
  }
  return k_yz_p<T, NTYZ, P, P, false, GR>;
}

// Two-CTA plane kernel for y = z = N (needs an even first radix).
template <typename T, int NTYZ, int N, int GR>
typename MvKernels<T>::YzFn pair_kernel(bool half) {
  typedef typename PlanFor<N>::type P;
  if constexpr (P::r[0] % 2 == 0) {
    if (half) return k_yz_pair<T, NTYZ, P, P, true, GR>;
    return k_yz_pair<T, NTYZ, P, P, false, GR>;
  } else {
    (void)half;
    return nullptr;
  }
}

// Cluster plane kernel for y = z = N, likewise.
template <typename T, int NTYZ, int N>
typename MvKernels<T>::SlotFn slot_kernel(bool half) {
  typedef typename PlanFor<N>::type P;
  if constexpr (P::r[0] % 2 == 0) {
    if (half) return k_yz_slot<T, NTYZ, P, P, true>;
  }
  return k_yz_slot<T, NTYZ, P, P, false>;
}

// The kernel tables are filled in parts, each compiled in its own
// translation unit (mv_inst.cu, built once per part and precision) so the
// several hundred plan instantiations compile in parallel.  Part 0: x passes;
// 1: split path (y rows, z columns) and the runtime-planned kernels; 2: fused
// plane kernels; 3: cluster plane kernels.
// The x passes of one x plan (PX: compile-time plan, or void) over the
// engine's own vectors (M = false) or, for FP32 engines, over FP64 vectors
// (M = true).
template <typename T, int NTX, typename PX, bool M>
void x_kernels(MvKernels<T>& k) {
  typedef typename C2<T>::t T2;
  if constexpr (!M) {
    k.xfwd = k_xfwd<T, NTX, PX, T2, 0>;
    k.xfwd_pre = k_xfwd<T, NTX, PX, T2, 1>;
    k.xinv = k_xinv<T, NTX, PX, T2>;
  } else if constexpr (std::is_same<T, float>::value) {
    k.xfwd_m = k_xfwd<T, NTX, PX, double2, 0>;
    k.xfwd_m_pre = k_xfwd<T, NTX, PX, double2, 1>;
    k.xinv_m = k_xinv<T, NTX, PX, double2>;
  }
}

template <typename T, int NTX, bool M>
void planned_x(MvKernels<T>& k, int gx) {
  switch (gx) {
#define C(N) \
  case N: x_kernels<T, NTX, typename PlanFor<N>::type, M>(k); break;
    DDA_TUNED_LENGTHS(C)
#undef C
    default: break;
  }
}

template <typename T, int NTYZ, int NTC>
void planned_split(MvKernels<T>& k, int gy, int gz) {
  switch (gy) {
#define C(N)                                                           \
  case N: k.yrows = k_yrows_p<T, NTYZ, typename PlanFor<N>::type>; break;
    DDA_TUNED_LENGTHS(C)
#undef C
    default: break;
  }
  switch (gz) {
#define C(N)                                                           \
  case N: k.cols = k_fft_cols<T, NTC, typename PlanFor<N>::type>; break;
    DDA_TUNED_LENGTHS(C)
#undef C
    default: break;
  }
}

template <typename T, int NTYZ>
void planned_fused(MvKernels<T>& k, int gy, int gz, int by, int bz) {
  if (gy != gz) return;
  switch (gy) {
#define C(N)                                                                                     \
  case N:                                                                                       \
    k.yz = fused_kernel<T, NTYZ, N>(2 * by == gy && 2 * bz == gz);                               \
    k.yz2 = fused_kernel<T, NTYZ, N, 2>(2 * by == gy && 2 * bz == gz);                           \
    k.yz4 = fused_kernel<T, NTYZ, N, 4>(2 * by == gy && 2 * bz == gz);                           \
    break;
    DDA_FUSED_LENGTHS(C)
#undef C
    default: break;
  }
}

template <typename T, int NTYZ>
void planned_pair(MvKernels<T>& k, int gy, int gz, int by, int bz) {
  if (gy != gz) return;
  switch (gy) {
#define C(N)                                                                                     \
  case N:                                                                                       \
    k.pair[0] = pair_kernel<T, NTYZ, N, 1>(2 * by == gy && 2 * bz == gz);                        \
    k.pair[1] = pair_kernel<T, NTYZ, N, 2>(2 * by == gy && 2 * bz == gz);                        \
    k.pair[2] = pair_kernel<T, NTYZ, N, 4>(2 * by == gy && 2 * bz == gz);                        \
    break;
    DDA_FUSED_LENGTHS(C)
#undef C
    default: break;
  }
}

template <typename T, int NTYZ>
void planned_slot(MvKernels<T>& k, int gy, int gz, int by, int bz) {
  if (gy != gz) return;
  switch (gy) {
#define C(N)                                                                                        \
  case N: k.slot = slot_kernel<T, NTYZ, N>(2 * by == gy && 2 * bz == gz); break;
    DDA_TUNED_LENGTHS(C)
#undef C
    default: break;
  }
}

template <typename T, int NTX, int NTYZ, int NTC>
void generic_kernels(MvKernels<T>& k) {
  x_kernels<T, NTX, void, false>(k);
  x_kernels<T, NTX, void, true>(k);
  k.yz = k_yz<T, NTYZ>;
  k.yrows = k_yrows<T, NTYZ>;
  k.cols = k_fft_cols<T, NTC>;
  k.slot = k_yz_slot<T, NTYZ, void, void>;
}

// Entry points of the parts (defined in mv_inst.cu).
void mv_part_x(MvKernels<float>& k, int gx);
void mv_part_x(MvKernels<double>& k, int gx);
void mv_part_xm(MvKernels<float>& k, int gx);
void mv_part_xm(MvKernels<double>& k, int gx);
void mv_part_split(MvKernels<float>& k, int gy, int gz, bool generic);
void mv_part_split(MvKernels<double>& k, int gy, int gz, bool generic);
void mv_part_fused(MvKernels<float>& k, int gy, int gz, int by, int bz);
void mv_part_fused(MvKernels<double>& k, int gy, int gz, int by, int bz);
void mv_part_slot(MvKernels<float>& k, int gy, int gz, int by, int bz);
void mv_part_slot(MvKernels<double>& k, int gy, int gz, int by, int bz);
void mv_part_pair(MvKernels<float>& k, int gy, int gz, int by, int bz);
void mv_part_pair(MvKernels<double>& k, int gy, int gz, int by, int bz);

// Kernel table of a context: compile-time-planned kernels for grid
// (gx, gy, gz) and box extents by, bz when every edge is tuned, the
// runtime-planned ones otherwise.
template <typename T>
MvKernels<T> select_kernels(bool planned, int gx, int gy, int gz, int by, int bz) {
  MvKernels<T> k;
  k.planned = planned;
  if (!planned) {
    mv_part_split(k, gy, gz, true);
    return k;
  }
  mv_part_x(k, gx);
  mv_part_xm(k, gx);
  mv_part_split(k, gy, gz, false);
  mv_part_fused(k, gy, gz, by, bz);
  mv_part_pair(k, gy, gz, by, bz);
  mv_part_slot(k, gy, gz, by, bz);
  return k;
}

}  // namespace dda
