// dmatrix_kernels.cuh -- D-matrix generation on the GPU in FP64.
//
// DMatrixCpu::createDMatrix (DDA/DMatrixCpu.cpp:133-205) fills the Green's
// tensor G_mu,nu(r) (DDA/DMatrixCpu.cpp:49-63) on the stencil
// |i| < bx, |j| < by, |k| < bz with G(0) = 0, transforms it with a 3-D FFT
// and divides by -(Gx Gy Gz); the reference GPU path copies that host result
// (DDA/DMatrixGpu.cpp:30-41, a TODO there).  Here each component is filled,
// transformed with the project FFT kernels and compressed to the octant
// kx <= Gx/2, kz <= Gz/2, ky <= Gy/2 directly on the device.
//
// Units: the tensor is evaluated in grid units (r = rho * d), i.e. the stored
// D is the reference D times d^3; the couple constants are scaled by d^-3/2
// to match, which leaves sqrt(cc) D sqrt(cc) unchanged and keeps FP32
// values near 1.
#pragma once

#include "fft_engine.cuh"

namespace dda {

__global__ void k_dfill(double2* __restrict__ full, int Gx, int Gy, int Gz, int bx, int by, int bz,
                        double kd, int mu, int nu) {
  const long long N = (long long)Gx * Gy * Gz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(idx % Gx);
    const int y = (int)((idx / Gx) % Gy);
    const int z = (int)(idx / ((long long)Gx * Gy));
    const int i = x <= Gx / 2 ? x : x - Gx;
    const int j = y <= Gy / 2 ? y : y - Gy;
    const int k = z <= Gz / 2 ? z : z - Gz;
    double2 v = make_double2(0, 0);
    if (abs(i) < bx && abs(j) < by && abs(k) < bz && (i | j | k)) {
      const double r[3] = {(double)i, (double)j, (double)k};
      const double rho = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const double qmunu = (r[mu] / rho) * (r[nu] / rho);
      const double kr = kd * rho;
      const double kr2 = kr * kr;
      double s, c;
      sincos(kr, &s, &c);
      const double inv = 1.0 / (rho * rho * rho);
      const double ex = c * inv, ey = s * inv;
      double bx_ = (3 - kr2) * qmunu, by_ = -3 * kr * qmunu;
      if (mu == nu) {
        bx_ += kr2 - 1;
        by_ += kr;
      }
      v = make_double2(ex * bx_ - ey * by_, ex * by_ + ey * bx_);
    }
    full[idx] = v;
  }
}

// full[z][y][x] (x fastest, each axis in the digit-reversed order the
// forward transforms leave; px/py/pz map a frequency to its position) ->
// octant [ax][az][ay][comp] scaled by -1/N.
__global__ void k_dcompress(const double2* __restrict__ full, double2* __restrict__ d64,
                            float2* __restrict__ d32, int Gx, int Gy, int Gz, int comp,
                            const int* __restrict__ px, const int* __restrict__ py,
                            const int* __restrict__ pz) {
  const int hx = Gx / 2 + 1, hy = Gy / 2 + 1, hz = Gz / 2 + 1;
  const long long M = (long long)hx * hy * hz;
  const double scale = -1.0 / ((double)Gx * Gy * Gz);
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < M;
       o += (long long)gridDim.x * blockDim.x) {
    const int ay = (int)(o % hy);
    const int az = (int)((o / hy) % hz);
    const int ax = (int)(o / ((long long)hy * hz));
    const double2 v = full[((long long)pz[az] * Gy + py[ay]) * Gx + px[ax]];
    const double2 d = make_double2(v.x * scale, v.y * scale);
    if (d64) d64[o * 6 + comp] = d;
    if (d32) d32[o * 6 + comp] = make_float2((float)d.x, (float)d.y);
  }
}

__global__ void k_d64_to_d32(const double2* __restrict__ a, float2* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}

template <typename A2, typename B2>
__global__ void k_convert(const A2* __restrict__ a, B2* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    B2 r;
    r.x = a[i].x;
    r.y = a[i].y;
    b[i] = r;
  }
}

}  // namespace dda
