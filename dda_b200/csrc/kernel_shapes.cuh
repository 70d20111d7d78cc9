// kernel_shapes.cuh -- threads per CTA of the matvec kernels, shared by the
// host code (dda_cuda.cu) and the kernel-table parts (mv_inst.cu).
#pragma once

namespace dda {

constexpr int kNtX = 256;  // k_xfwd / k_xinv
// k_yz / k_yrows: 512 threads in FP32; 256 in FP64, whose FFT stages need
// more than the 128 registers a 512-thread CTA leaves per thread.
template <typename T> struct NtYz;
template <> struct NtYz<float> { static constexpr int v = 512; };
template <> struct NtYz<double> { static constexpr int v = 256; };
constexpr int kNtC = 256;  // k_fft_cols / k_fft_rows

}  // namespace dda
