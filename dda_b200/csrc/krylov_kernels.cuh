// krylov_kernels.cuh -- fused vector steps of the Krylov solvers.
//
// One launch per solver step does every linear combination of that step in
// a single pass over the vectors and the step's dot products in FP64, then
// the last CTA runs the scalar recurrence (krylov_ops.cuh).  This replaces the
// per-update linComb kernels, the two-stage reductions and the blocking
// scalar reads/writes of GpuLinComb / GpuQmrCs / GpuBicgStab
// (LinAlg/GpuLinCombInst.cl:171-322, DDA/GpuQmrCs.cpp:102-198,
// DDA/GpuBicgStab.cpp:44-125) and the setup kernels of
// DDA/GpuIterativeSolverInst.cl:27-108.
#pragma once

#include <array>
#include <utility>

#include "fft_engine.cuh"
#include "krylov_ops.cuh"
#include "reduce.cuh"

namespace dda {

// (The steps that produce a matvec argument -- BiCGStab's p and s, BiCG's
// and CGNR's p -- run in the matvec's first pass: XPreOp, matvec_kernels.cuh.)
enum VecOp {
  V_SETUP_PVEC = 0,  // v0 = sqrt(cc).v1 (b = sqrt(cc) Einc); n = |v0|^2
  V_START_X,         // v0 = v1 / sqrt(cc)  (start value, DDA/GpuIterativeSolverInst.cl:52-77)
  V_R_INIT,          // v0 = -v1 + v2  (r = b - A x); n = |r|^2
  V_CHOOSE_X0,       // usezero ? (v0 = 0, v1 = v2) : v0 = v2      (x, r, b)
  V_QMR_V0,          // v0 = v1 . betaInv                          (v = r / beta)
  V_QMR_VT,          // v0 = [v0 mBeta] + v1 mAlpha + v2; a = v0.v0, n = |v0|^2   (vt, v, A)
  V_QMR_UPD,         // p/x/v/r update of DDA/QmrCs.cpp:152-167 (first: 1 = iteration 0, 2 = iteration 1)
  V_BIS_INIT,        // v0 = v1 (rt = r); a = v1.conj(v0)
  V_BIS_XR,          // x/r update of DDA/BicgStab.cpp:98-110
  V_BICG_RO,         // a = v0.v0
  V_BICG_XR,         // x += p alpha; r += A mAlpha; n = |r|^2; a = r.r
  V_CGNR_XR,         // x += p alpha; r += A mAlpha; n = |r|^2
  V_RESULT,          // v0 = sqrt(cc).v1  (P = sqrt(cc) x)
  V_NORM,            // n = |v0|^2
  V_COUNT
};

struct VecArgs {
  void* v[6];
  int op;
  int first;  // iteration 0 variant
  int nv, nvs, nmat;
  int nparts;
  const uint8_t* mat;  // material per dipole (caller order)
  const void* ccs;     // [nrhs][nmat][3] complex, scaled by d^-3/2
  double pscale;       // d^3: P = pscale * ccs . x (V_RESULT); x = P / (pscale ccs) (V_START_X)
  KrylovStep step;
};

// Whether the element loop of step OP reads vector k (first: the
// iteration-0 variant flag, skip: the BiCGStab half-step exit).
template <int OP>
__device__ __forceinline__ bool vec_reads(int k, int first, int skip) {
  switch (OP) {
    case V_SETUP_PVEC:
    case V_RESULT:
    case V_START_X:
    case V_QMR_V0:
    case V_BIS_INIT:
      return k == 1;
    case V_R_INIT:
      return k == 1 || k == 2;
    case V_CHOOSE_X0:
      return k == 2;
    case V_QMR_VT:
      return k == 1 || k == 2 || (k == 0 && !first);
    case V_QMR_UPD:
      return k == 0 || k == 3 || k == 4 || k == 5 || (k == 2 && first != 1) || (k == 1 && first == 0);
    case V_BIS_XR:
      return k == 0 || k == 1 || (!skip && (k == 2 || k == 3 || k == 5));
    case V_BICG_RO:
    case V_NORM:
      return k == 0;
    case V_BICG_XR:
    case V_CGNR_XR:
      return k <= 3;
    default:
      return false;
  }
}

// One instantiation per operation OP (va.op == OP), so that each keeps only
// its own registers: the vector steps are streaming kernels, and their speed
// is the number of loads in flight, i.e. the CTAs an SM holds times the loads
// each thread issues before it waits.
template <typename T, int NT, int OP>
__global__ void __launch_bounds__(NT, 3) k_vec(VecArgs va, KrylovState* st) {
  typedef typename C2<T>::t T2;
  const int b = blockIdx.y;
  KrylovState& s = st[b];
  if (s.done && OP != V_RESULT) return;  // the result copy runs after convergence
  const long long len = 3LL * va.nvs;
  const long long chunk = ((len + va.nparts - 1) / va.nparts + 31) / 32 * 32;
  const long long i0 = chunk * blockIdx.x;
  const long long i1 = min(len, i0 + chunk);
  const size_t off = (size_t)b * len;
  T2* v0 = va.v[0] ? reinterpret_cast<T2*>(va.v[0]) + off : nullptr;
  T2* v1 = va.v[1] ? reinterpret_cast<T2*>(va.v[1]) + off : nullptr;
  T2* v2 = va.v[2] ? reinterpret_cast<T2*>(va.v[2]) + off : nullptr;
  T2* v3 = va.v[3] ? reinterpret_cast<T2*>(va.v[3]) + off : nullptr;
  T2* v4 = va.v[4] ? reinterpret_cast<T2*>(va.v[4]) + off : nullptr;
  T2* v5 = va.v[5] ? reinterpret_cast<T2*>(va.v[5]) + off : nullptr;
  const T2* ccs = reinterpret_cast<const T2*>(va.ccs) + (size_t)b * va.nmat * 3;
  // step scalars in working precision
  const T2 mBeta = cvt<T2>(s.mBeta), mAlpha = cvt<T2>(s.mAlpha), alpha = cvt<T2>(s.alpha);
  const T2 betaInv = cvt<T2>(s.betaInv);
  const T2 omega = cvt<T2>(s.omega), tau = cvt<T2>(s.tau), cNOT = cvt<T2>(s.cNOT);
  const T2 zetaInv = cvt<T2>(s.zetaInv), mEtaZeta = cvt<T2>(s.mEtaZeta), mThetaZeta = cvt<T2>(s.mThetaZeta);
  const T2 mOmega = cvt<T2>(dneg(s.omega));
  const T normS = (T)s.normSNew;
  const int skip = s.skipmv, usezero = s.usezero;
  RedSums acc = red_zero();
  // Every element's inputs are loaded for U elements before the first is
  // used: with one element at a time a thread waits out the memory latency
  // once per element and the step runs far below the HBM rate.
  constexpr int U = (sizeof(T) == 4 ? 4 : 2) / (OP == V_QMR_UPD ? 2 : 1);  // six streams: half
  const int first = va.first;
  for (long long base = i0 + threadIdx.x; base < i1; base += (long long)U * NT) {
    T2 in0[U], in1[U], in2[U], in3[U], in4[U], in5[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long i = base + (long long)u * NT;
      if (i < i1) {
        if (vec_reads<OP>(0, first, skip)) in0[u] = v0[i];
        if (vec_reads<OP>(1, first, skip)) in1[u] = v1[i];
        if (vec_reads<OP>(2, first, skip)) in2[u] = v2[i];
        if (vec_reads<OP>(3, first, skip)) in3[u] = v3[i];
        if (vec_reads<OP>(4, first, skip)) in4[u] = v4[i];
        if (vec_reads<OP>(5, first, skip)) in5[u] = v5[i];
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long i = base + (long long)u * NT;
      if (i >= i1) break;
      switch (OP) {
        case V_SETUP_PVEC:
        case V_RESULT:
        case V_START_X: {
          const int c = (int)(i / va.nvs), j = (int)(i % va.nvs);
          T2 o = czero<T2>();
          if (j < va.nv) {
            const T2 cc = ccs[va.mat[j] * 3 + c];
            const T2 x = in1[u];
            if (OP == V_START_X) {
              // x / cc (Smith division in FP64)
              double2 q = ddivc(make_double2(x.x, x.y), make_double2(cc.x, cc.y));
              o = cvt<T2>(dscale(q, 1.0 / va.pscale));
            } else if (OP == V_RESULT) {
              o = cvt<T2>(dscale(dmulc(make_double2(cc.x, cc.y), make_double2(x.x, x.y)), va.pscale));
            } else {
              o = cmul(cc, x);
            }
          }
          v0[i] = o;
          acc.n += (double)o.x * o.x + (double)o.y * o.y;
          break;
        }
        case V_R_INIT: {
          T2 r = csub(in2[u], in1[u]);
          v0[i] = r;
          acc.n += (double)r.x * r.x + (double)r.y * r.y;
          break;
        }
        case V_CHOOSE_X0: {
          const T2 p = in2[u];
          if (usezero) { v0[i] = czero<T2>(); v1[i] = p; }
          else v0[i] = p;
          break;
        }
        case V_QMR_V0:
          v0[i] = cmul(in1[u], betaInv);
          break;
        case V_QMR_VT: {
          T2 t = cadd(cmul(in1[u], mAlpha), in2[u]);
          if (!va.first) t = cadd(cmul(in0[u], mBeta), t);
          v0[i] = t;
          acc.a.x += (double)t.x * t.x - (double)t.y * t.y;
          acc.a.y += 2.0 * (double)t.x * t.y;
          acc.n += (double)t.x * t.x + (double)t.y * t.y;
          break;
        }
        case V_QMR_UPD: {
          // v0 = r, v1 = p_old, v2 = p_new, v3 = v, v4 = vt, v5 = x.  The new
          // search direction goes to p_new in iteration 0 and to p_old after
          // that (the caller then swaps p_old and p_new, DDA/QmrCs.cpp:152-160).
          const T2 v = in3[u];
          T2 pn;
          if (va.first == 1) {
            pn = cmul(v, zetaInv);
            v2[i] = pn;
          } else {
            if (va.first == 2) pn = cadd(cmul(in2[u], mEtaZeta), cmul(v, zetaInv));
            else pn = cadd(cadd(cmul(in1[u], mThetaZeta), cmul(in2[u], mEtaZeta)), cmul(v, zetaInv));
            v1[i] = pn;
          }
          v5[i] = cadd(cmul(pn, tau), in5[u]);
          const T2 vn = cmul(in4[u], betaInv);
          v4[i] = vn;
          const T2 ro = in0[u];
          T2 r;
          r.x = ro.x * normS; r.y = ro.y * normS;
          r = cadd(r, cmul(vn, cNOT));
          v0[i] = r;
          acc.n += (double)r.x * r.x + (double)r.y * r.y;
          break;
        }
        case V_BIS_INIT: {
          const T2 r = in1[u];
          v0[i] = r;
          acc.a.x += (double)r.x * r.x + (double)r.y * r.y;
          break;
        }
        case V_BIS_XR: {
          // v0 = x, v1 = p, v2 = s, v3 = A s, v4 = r, v5 = rt
          if (skip) {
            v0[i] = cadd(cmul(in1[u], alpha), in0[u]);
          } else {
            const T2 sv = in2[u];
            v0[i] = cadd(cadd(cmul(in1[u], alpha), cmul(sv, omega)), in0[u]);
            const T2 r = cadd(cmul(in3[u], mOmega), sv);
            v4[i] = r;
            const T2 rt = in5[u];
            acc.n += (double)r.x * r.x + (double)r.y * r.y;
            acc.a.x += (double)r.x * rt.x + (double)r.y * rt.y;
            acc.a.y += (double)r.y * rt.x - (double)r.x * rt.y;
          }
          break;
        }
        case V_BICG_RO: {
          const T2 r = in0[u];
          acc.a.x += (double)r.x * r.x - (double)r.y * r.y;
          acc.a.y += 2.0 * (double)r.x * r.y;
          break;
        }
        case V_BICG_XR:
        case V_CGNR_XR: {
          // v0 = x, v1 = p, v2 = A, v3 = r
          v0[i] = cadd(cmul(in1[u], alpha), in0[u]);
          const T2 r = cadd(cmul(in2[u], mAlpha), in3[u]);
          v3[i] = r;
          acc.n += (double)r.x * r.x + (double)r.y * r.y;
          acc.a.x += (double)r.x * r.x - (double)r.y * r.y;
          acc.a.y += 2.0 * (double)r.x * r.y;
          break;
        }
        case V_NORM: {
          const T2 r = in0[u];
          acc.n += (double)r.x * r.x + (double)r.y * r.y;
          break;
        }
        default:
          break;
      }
    }
  }
  if (va.step.op != KOP_NONE) {
    RedSums tot;
    if (block_finish<NT>(acc, va.step.red, b, blockIdx.x, tot) && threadIdx.x == 0)
      krylov_finalize(s, va.step, tot);
  }
}

// k_vec<T, NT, op> for a run-time op.
template <typename T, int NT, int... OPS>
__host__ inline auto vec_kernel_table(std::integer_sequence<int, OPS...>) {
  typedef void (*Fn)(VecArgs, KrylovState*);
  return std::array<Fn, sizeof...(OPS)>{{&k_vec<T, NT, OPS>...}};
}
template <typename T, int NT>
__host__ inline void (*vec_kernel(int op))(VecArgs, KrylovState*) {
  static const auto tab = vec_kernel_table<T, NT>(std::make_integer_sequence<int, V_COUNT>{});
  return tab[op];
}

// x64 += e for every right-hand side the refinement loop still runs
// (grid (parts, nrhs)); the FP64 update of mixed-precision refinement.
template <typename E2>
__global__ void __launch_bounds__(256) k_accum(double2* __restrict__ x, const E2* __restrict__ e,
                                             const KrylovState* __restrict__ st, long long len) {
  const int b = blockIdx.y;
  if (st[b].done) return;
  const size_t off = (size_t)b * len;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < len; i += (long long)gridDim.x * 256) {
    const E2 d = e[off + i];
    double2 v = x[off + i];
    v.x += d.x;
    v.y += d.y;
    x[off + i] = v;
  }
}

}  // namespace dda
