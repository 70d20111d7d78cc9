// mv_inst.cu -- one part of the matvec kernel tables (matvec_dispatch.cuh),
// compiled once per part and precision:
//   nvcc -DDDA_MV_PART=<0..5> -DDDA_MV_DOUBLE=<0|1> -c mv_inst.cu
// Part 0: x passes; 1: split path and runtime-planned kernels; 2: fused
// plane kernels; 3: cluster plane kernels; 4: two-CTA plane kernels; 5: x
// passes of FP32 engines over FP64 vectors.  The parts hold the several
// hundred compile-time plan instantiations and build in parallel.
#include "kernel_shapes.cuh"
#include "matvec_dispatch.cuh"

#if !defined(DDA_MV_PART) || !defined(DDA_MV_DOUBLE)
#error "build with -DDDA_MV_PART=<0..5> -DDDA_MV_DOUBLE=<0|1>"
#endif

namespace dda {

#if DDA_MV_DOUBLE
typedef double MvT;
#else
typedef float MvT;
#endif

#if DDA_MV_PART == 0
void mv_part_x(MvKernels<MvT>& k, int gx) { planned_x<MvT, kNtX, false>(k, gx); }
#elif DDA_MV_PART == 1
void mv_part_split(MvKernels<MvT>& k, int gy, int gz, bool generic) {
  if (generic) generic_kernels<MvT, kNtX, NtYz<MvT>::v, kNtC>(k);
  else planned_split<MvT, NtYz<MvT>::v, kNtC>(k, gy, gz);
}
#elif DDA_MV_PART == 2
void mv_part_fused(MvKernels<MvT>& k, int gy, int gz, int by, int bz) {
  planned_fused<MvT, NtYz<MvT>::v>(k, gy, gz, by, bz);
}
#elif DDA_MV_PART == 3
void mv_part_slot(MvKernels<MvT>& k, int gy, int gz, int by, int bz) {
  planned_slot<MvT, NtYz<MvT>::v>(k, gy, gz, by, bz);
}
#elif DDA_MV_PART == 4
void mv_part_pair(MvKernels<MvT>& k, int gy, int gz, int by, int bz) {
  planned_pair<MvT, NtYz<MvT>::v>(k, gy, gz, by, bz);
}
#elif DDA_MV_PART == 5
void mv_part_xm(MvKernels<MvT>& k, int gx) { planned_x<MvT, kNtX, true>(k, gx); }
#endif

}  // namespace dda
