// farfield_kernels.cuh -- scattered far field of the dipole polarisations for
// many directions at once.
//
// FieldCalculator::calcField (DDA/CpuFieldCalculator.cpp:48-98, GPU kernel
// DDA/GpuFieldCalculatorInst.cl:27-70, launched once per direction from a
// host loop in DDA/FarFieldCalc.cpp:131-155) computes for one direction n
//   S = sum_j P_j exp(-i kd n.r_j),  E = i k^2 exp(-i k origin.n) (S - n (n.S)).
// Here a CTA takes DB directions of one right-hand side and walks the
// dipoles line by line: the y/z phase is one sincos per line and direction,
// the x phase comes from a per-CTA table, and all sums are FP64.
#pragma once

#include "fft_engine.cuh"

namespace dda {

struct FfGeom {
  int nv, nvs, by, nlines, bx;
  double kd, k;             // kd and wave number
  double ox, oy, oz;        // particle origin (metres)
};

template <typename T, int NT, int DB>
__global__ void __launch_bounds__(NT) k_farfield(const typename C2<T>::t* __restrict__ pol,
                                                 const uint32_t* __restrict__ line_off,
                                                 const uint32_t* __restrict__ dip,
                                                 const uint32_t* __restrict__ perm,
                                                 const double* __restrict__ dirs, int ndir, FfGeom g,
                                                 double2* __restrict__ out) {
  typedef typename C2<T>::t T2;
  extern __shared__ __align__(16) unsigned char ffsm[];
  double2* tx = reinterpret_cast<double2*>(ffsm);  // [DB][bx]
  __shared__ double nd[DB][3];
  __shared__ double2 red[NT / 32][DB][3];
  const int d0 = blockIdx.x * DB, b = blockIdx.y;
  const int nd_here = min(DB, ndir - d0);
  if (threadIdx.x < DB * 3) {
    const int d = threadIdx.x / 3, a = threadIdx.x % 3;
    nd[d][a] = d < nd_here ? dirs[(size_t)(d0 + d) * 3 + a] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < DB * g.bx; i += NT) {
    const int d = i / g.bx, x = i % g.bx;
    double s, c;
    sincos(-g.kd * nd[d][0] * (double)x, &s, &c);
    tx[i] = make_double2(c, s);
  }
  __syncthreads();
  const T2* P = pol + (size_t)b * 3 * g.nvs;
  double2 acc[DB][3];
#pragma unroll
  for (int d = 0; d < DB; d++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[d][c] = make_double2(0, 0);
  for (int L = threadIdx.x; L < g.nlines; L += NT) {
    const uint32_t j0 = line_off[L], j1 = line_off[L + 1];
    if (j0 == j1) continue;
    const int z = L / g.by, y = L - z * g.by;
    double2 ls[DB][3];
#pragma unroll
    for (int d = 0; d < DB; d++)
#pragma unroll
      for (int c = 0; c < 3; c++) ls[d][c] = make_double2(0, 0);
    for (uint32_t j = j0; j < j1; j++) {
      const int x = (int)(dip[j] & 0xffffu);
      const uint32_t jj = perm ? perm[j] : j;
      double2 p[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const T2 v = P[c * g.nvs + jj];
        p[c] = make_double2(v.x, v.y);
      }
#pragma unroll
      for (int d = 0; d < DB; d++) {
        const double2 t = tx[d * g.bx + x];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          ls[d][c].x += p[c].x * t.x - p[c].y * t.y;
          ls[d][c].y += p[c].x * t.y + p[c].y * t.x;
        }
      }
    }
#pragma unroll
    for (int d = 0; d < DB; d++) {
      double s, c;
      sincos(-g.kd * (nd[d][1] * y + nd[d][2] * z), &s, &c);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        acc[d][k].x += ls[d][k].x * c - ls[d][k].y * s;
        acc[d][k].y += ls[d][k].x * s + ls[d][k].y * c;
      }
    }
  }
  // block reduction in a fixed order
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 0; d < DB; d++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 v = acc[d][c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
      }
      if (lane == 0) red[w][d][c] = v;
    }
  __syncthreads();
  if (threadIdx.x < nd_here) {
    const int d = threadIdx.x;
    double2 S[3];
    for (int c = 0; c < 3; c++) {
      S[c] = make_double2(0, 0);
      for (int ww = 0; ww < NT / 32; ww++) {
        S[c].x += red[ww][d][c].x;
        S[c].y += red[ww][d][c].y;
      }
    }
    const double* n = nd[d];
    const double2 ndS = make_double2(n[0] * S[0].x + n[1] * S[1].x + n[2] * S[2].x,
                                     n[0] * S[0].y + n[1] * S[1].y + n[2] * S[2].y);
    double s, c;
    sincos(-g.k * (g.ox * n[0] + g.oy * n[1] + g.oz * n[2]), &s, &c);
    const double k2 = g.k * g.k;
    // f = i k^2 exp(-i k origin.n)
    const double fx = -k2 * s, fy = k2 * c;
    for (int a = 0; a < 3; a++) {
      const double tx_ = S[a].x - n[a] * ndS.x, ty_ = S[a].y - n[a] * ndS.y;
      out[((size_t)(d0 + d) * gridDim.y + b) * 3 + a] = make_double2(fx * tx_ - fy * ty_, fx * ty_ + fy * tx_);
    }
  }
}

}  // namespace dda
