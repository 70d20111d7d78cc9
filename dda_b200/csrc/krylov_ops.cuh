// krylov_ops.cuh -- device-resident Krylov scalar state and the scalar
// recurrences of the four solvers, run by the last CTA of each fused
// reduction (see reduce.cuh).  The vector work of each step lives in
// krylov_kernels.cuh and in the matvec epilogue (k_xinv).
//
// Recurrences follow the reference CPU solvers line by line:
//   QMR-CS   DDA/QmrCs.cpp:58-168     (bilinear product, DDA/QmrCs.cpp:48-55)
//   BiCGStab DDA/BicgStab.cpp:59-112  (Hermitian product, DDA/BicgStab.cpp:34-41)
//   BiCG-CS  DDA/BicgCs.cpp:56-84
//   CGNR     DDA/Cgnr.cpp:39-73
// and the shared loop of IterativeSolverBase::getPolVec
// (DDA/IterativeSolverBase.cpp:56-98): stop when the best |r|^2 so far drops
// below epsB = eps^2 |b|^2; fail after maxIter iterations or more than
// maxResIncrease iterations without improvement.  All scalars are FP64
// (the reference's long-double temporaries in BiCGStab become FP64).
#pragma once

#include <cuda_runtime.h>
#include "reduce.cuh"

namespace dda {

enum KStatus {
  KS_RUNNING = 0,
  KS_BREAKDOWN = -5,
  KS_MAXITER = -6,
  KS_NOPROGRESS = -7,
};

// Reductions a step asks of its kernel (over the step's output vector y,
// its input a and an optional third vector w).
enum EpMode {
  EP_YA_BIL = 0,        // a += sum y.a            (bilinear)
  EP_YW_HERM = 1,       // a += sum y.conj(w)
  EP_AY_HERM_NORM = 2,  // a += sum a.conj(y); n += sum |y|^2
  EP_NORM = 3,          // n += sum |y|^2
};

enum KOp {
  KOP_NONE = 0,
  KOP_INIT_PVEC,   // n = |b|^2 -> residScale
  KOP_INIT_R,      // n = |r0|^2 -> choose x0 in {0, b}
  KOP_INIT_START,  // n = |r0|^2 with a loaded start value
  KOP_QMR_INIT,    // a = r.r
  KOP_QMR_ALPHA,   // a = v.Av
  KOP_QMR_GIVENS,  // a = vt.vt, n = |vt|^2
  KOP_QMR_END,     // n = |r|^2
  KOP_BIS_RO,      // a = r.conj(rt)          (first iteration)
  KOP_BIS_ALPHA,   // a = v.conj(rt)
  KOP_BIS_S,       // n = |s|^2
  KOP_BIS_OMEGA,   // a = s.conj(As), n = |As|^2
  KOP_BIS_END,     // n = |r|^2, a = r.conj(rt)
  KOP_BICG_RO,     // a = r.r                 (first iteration)
  KOP_BICG_MU,     // a = p.Ap
  KOP_BICG_END,    // n = |r|^2, a = r.r
  KOP_CGNR_RO,     // n = |A^H r|^2
  KOP_CGNR_ALPHA,  // n = |Ap|^2
  KOP_CGNR_END,    // n = |r|^2
  KOP_NORM,        // n -> last (plain reduction)
};

struct KrylovState {
  int done;       // 1 once converged or failed; kernels skip this rhs
  int status;     // KStatus
  int skipmv;     // BiCGStab half-step exit: skip the second matvec
  int usezero;    // initGeneral chose x0 = 0
  long long count, counter, maxIter, maxResIncrease, histCap;
  double inprodR, residScale, epsB, last, temp;
  double2 alpha, beta, mBeta, omega, ro_new, ro_old, tau, tautilda, s_old, s_new;
  double2 zetaInv, mEtaZeta, mThetaZeta, betaInv, cNOT, mAlpha, bo;
  double omega_old, omega_new, c_old, c_new, normSNew, abs_ro_new, sNorm;
  double* hist;
  // progress-rate stop (inner solves of the mixed refinement): with
  // rateWin > 0 the solve ends with KS_NOPROGRESS when the best |r| has not
  // halved over the last rateWin iterations
  long long rateWin, chkIt;
  double chkR;
};

struct KrylovStep {
  int op;
  int mode;
  const void* w;  // third vector for EP_YW_HERM (same precision as y)
  RedTarget red;
};

__device__ __forceinline__ double2 dc(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 dmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 ddivc(double2 a, double2 b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
__device__ __forceinline__ double dabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double dabsc(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double2 dneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 dconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 dscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// principal square root (std::sqrt of a complex)
__device__ __forceinline__ double2 dsqrtc(double2 z) {
  double r = dabsc(z);
  if (r == 0) return make_double2(0, 0);
  if (z.x >= 0) {
    double t = sqrt(0.5 * (r + z.x));
    return make_double2(t, z.y / (2 * t));
  } else {
    double t = sqrt(0.5 * (r - z.x));
    return make_double2(fabs(z.y) / (2 * t), z.y >= 0 ? t : -t);
  }
}

template <typename T2>
__device__ __forceinline__ RedSums epilogue_terms(RedSums acc, T2 y, T2 a, T2 w, int mode) {
  const double yx = y.x, yy = y.y;
  switch (mode) {
    case EP_YA_BIL:
      acc.a.x += yx * a.x - yy * a.y;
      acc.a.y += yx * a.y + yy * a.x;
      break;
    case EP_YW_HERM:
      acc.a.x += yx * w.x + yy * w.y;
      acc.a.y += yy * w.x - yx * w.y;
      break;
    case EP_AY_HERM_NORM:
      acc.a.x += (double)a.x * yx + (double)a.y * yy;
      acc.a.y += (double)a.y * yx - (double)a.x * yy;
      acc.n += yx * yx + yy * yy;
      break;
    default:
      acc.n += yx * yx + yy * yy;
      break;
  }
  return acc;
}

__device__ __forceinline__ void kfail(KrylovState& s, int code) {
  s.status = code;
  s.done = 1;
}

// IterativeSolverBase loop update (DDA/IterativeSolverBase.cpp:56-98) after
// an iteration returned |r|^2 = next.
// A residual that is not a number ends the solve with KS_BREAKDOWN (the
// reference keeps iterating until maxResIncrease, since no NaN compares as an
// improvement).
__device__ __forceinline__ void loop_update(KrylovState& s, double next) {
  s.count++;
  if (!(next == next)) {
    if (s.hist && s.count - 1 < s.histCap) s.hist[s.count - 1] = next;
    kfail(s, KS_BREAKDOWN);
    return;
  }
  if (next <= s.inprodR) {
    s.inprodR = next;
    s.counter = 0;
  } else {
    s.counter++;
  }
  s.last = next;
  if (s.hist && s.count - 1 < s.histCap) s.hist[s.count - 1] = sqrt(s.residScale * next);
  if (s.rateWin > 0 && s.chkIt == 0 && s.chkR == 0) s.chkR = s.inprodR;
  if (s.inprodR < s.epsB) {
    s.done = 1;
  } else if (s.count >= s.maxIter) {
    kfail(s, KS_MAXITER);
  } else if (s.counter > s.maxResIncrease) {
    kfail(s, KS_NOPROGRESS);
  } else if (s.rateWin > 0 && s.count - s.chkIt >= s.rateWin) {
    if (s.inprodR > 0.25 * s.chkR) {
      kfail(s, KS_NOPROGRESS);
    } else {
      s.chkR = s.inprodR;
      s.chkIt = s.count;
    }
  }
}

// QMR-CS breakdown guard at the start of iteration nr (DDA/QmrCs.cpp:89-93),
// written so that a beta that is not a number fails it as well.
__device__ __forceinline__ void qmr_check_beta(KrylovState& s) {
  double rtmp1 = dabs2(s.beta) * s.residScale;
  if (s.count == 0) {
    if (!(rtmp1 <= 1e+38f)) kfail(s, KS_BREAKDOWN);
  } else if (!(rtmp1 >= 1e-10f && rtmp1 <= 1e+38f)) {
    kfail(s, KS_BREAKDOWN);
  }
}

// BiCGStab start-of-iteration scalars (DDA/BicgStab.cpp:76-88).
__device__ __forceinline__ void bis_start(KrylovState& s, double2 ro) {
  s.ro_new = ro;
  double dtmp = dabsc(ro) / s.inprodR;
  if (!(dtmp >= 1e-16)) { kfail(s, KS_BREAKDOWN); return; }
  if (s.count > 0) {
    double2 rna = dmulc(s.ro_new, s.alpha);
    double2 roo = dmulc(s.ro_old, s.omega);
    if (!(dabsc(roo) / dabsc(rna) >= 10e-10)) { kfail(s, KS_BREAKDOWN); return; }
    s.beta = ddivc(rna, roo);
    s.bo = dneg(dmulc(s.beta, s.omega));
  }
}

// BiCG-CS start-of-iteration scalars (DDA/BicgCs.cpp:65-74).
__device__ __forceinline__ void bicg_start(KrylovState& s, double2 ro) {
  s.ro_new = ro;
  s.abs_ro_new = dabsc(ro);
  double dtmp = s.abs_ro_new / s.inprodR;
  if (dtmp < 1e-10 || dtmp > 1e+10) { kfail(s, KS_BREAKDOWN); return; }
  if (s.count > 0) s.beta = ddivc(s.ro_new, s.ro_old);
}

static __device__ void krylov_finalize(KrylovState& s, const KrylovStep& step, const RedSums& t) {
  switch (step.op) {
    case KOP_INIT_PVEC:
      s.temp = t.n;
      s.residScale = 1.0 / t.n;
      break;
    case KOP_INIT_R:  // DDA/CpuIterativeSolver.cpp:66-86
      s.inprodR = t.n;
      if (s.temp < t.n) {
        s.usezero = 1;
        s.inprodR = s.temp;
      } else {
        s.usezero = 0;
      }
      break;
    case KOP_INIT_START:
      s.inprodR = t.n;
      s.usezero = 0;
      break;
    case KOP_QMR_INIT: {  // DDA/QmrCs.cpp:58-76
      s.omega_old = 0;
      s.beta = dsqrtc(t.a);
      s.mBeta = dneg(s.beta);
      s.omega_new = sqrt(s.inprodR) / dabsc(s.beta);
      s.tautilda = dscale(s.beta, s.omega_new);
      s.c_old = 1; s.c_new = 1;
      s.s_old = dc(0, 0); s.s_new = dc(0, 0);
      s.betaInv = ddivc(dc(1, 0), s.beta);
      qmr_check_beta(s);
      break;
    }
    case KOP_QMR_ALPHA:
      s.alpha = t.a;
      s.mAlpha = dneg(t.a);
      break;
    case KOP_QMR_GIVENS: {  // DDA/QmrCs.cpp:113-148
      const double2 ctmp3 = t.a;
      const double rtmp2 = t.n;
      double2 ctmp1 = dscale(s.beta, s.omega_old);
      double2 ctmp2 = dscale(s.alpha, s.omega_new);
      double2 theta = dmulc(dconj(s.s_old), ctmp1);
      double2 eta = dadd2(dscale(ctmp1, s.c_old * s.c_new), dmulc(dconj(s.s_new), ctmp2));
      double2 zetatilda = dadd2(dscale(ctmp2, s.c_new), dneg(dscale(dmulc(s.s_new, ctmp1), s.c_old)));
      s.beta = dsqrtc(ctmp3);
      s.mBeta = dneg(s.beta);
      s.omega_old = s.omega_new;
      s.omega_new = sqrt(rtmp2) / dabsc(s.beta);
      double zetaabs = sqrt(dabs2(zetatilda) + rtmp2);
      double rtmp3 = sqrt(dabs2(zetatilda));
      double2 zeta;
      if (rtmp3 < 1e-40f) zeta = dc(zetaabs, 0);
      else zeta = dscale(zetatilda, zetaabs / rtmp3);
      s.c_old = s.c_new;
      s.c_new = rtmp3 / zetaabs;
      s.s_old = s.s_new;
      s.s_new = dscale(ddivc(s.beta, zeta), s.omega_new);
      s.tau = dscale(s.tautilda, s.c_new);
      s.tautilda = dneg(dmulc(s.s_new, s.tautilda));
      s.zetaInv = ddivc(dc(1, 0), zeta);
      s.mEtaZeta = dneg(ddivc(eta, zeta));
      s.mThetaZeta = dneg(ddivc(theta, zeta));
      s.betaInv = ddivc(dc(1, 0), s.beta);
      s.normSNew = dabs2(s.s_new);
      s.cNOT = dscale(s.tautilda, s.c_new / s.omega_new);
      break;
    }
    case KOP_QMR_END:
      loop_update(s, t.n);
      if (!s.done) qmr_check_beta(s);
      break;
    case KOP_BIS_RO:
      bis_start(s, t.a);
      break;
    case KOP_BIS_ALPHA:  // DDA/BicgStab.cpp:93-95
      s.alpha = ddivc(s.ro_new, t.a);
      s.mAlpha = dneg(s.alpha);
      break;
    case KOP_BIS_S:  // DDA/BicgStab.cpp:96-98
      s.sNorm = t.n;
      s.skipmv = t.n < s.epsB ? 1 : 0;
      break;
    case KOP_BIS_OMEGA:  // DDA/BicgStab.cpp:101-105
      s.omega = dscale(t.a, 1.0 / t.n);
      break;
    case KOP_BIS_END: {  // DDA/BicgStab.cpp:98-111
      double next;
      if (s.skipmv) {
        next = s.sNorm;
      } else {
        next = t.n;
        s.ro_old = s.ro_new;
      }
      s.skipmv = 0;
      loop_update(s, next);
      if (!s.done) bis_start(s, t.a);
      break;
    }
    case KOP_BICG_RO:
      bicg_start(s, t.a);
      break;
    case KOP_BICG_MU: {  // DDA/BicgCs.cpp:76-79
      double dtmp2 = dabsc(t.a) / s.abs_ro_new;
      if (dtmp2 < 10e-10) { kfail(s, KS_BREAKDOWN); break; }
      s.alpha = ddivc(s.ro_new, t.a);
      s.mAlpha = dneg(s.alpha);
      break;
    }
    case KOP_BICG_END:
      s.ro_old = s.ro_new;
      loop_update(s, t.n);
      if (!s.done) bicg_start(s, t.a);
      break;
    case KOP_CGNR_RO:  // DDA/Cgnr.cpp:49-63
      s.ro_new = dc(t.n, 0);
      if (s.count > 0) s.beta = dc(t.n / s.ro_old.x, 0);
      break;
    case KOP_CGNR_ALPHA:
      s.alpha = dc(s.ro_new.x / t.n, 0);
      s.mAlpha = dneg(s.alpha);
      break;
    case KOP_CGNR_END:
      s.ro_old = s.ro_new;
      loop_update(s, t.n);
      break;
    case KOP_NORM:
      s.last = t.n;
      s.sNorm = t.n;
      break;
    default:
      break;
  }
}

}  // namespace dda
