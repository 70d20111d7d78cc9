/*
 * dda_cuda.h -- C ABI of the B200 DDA solver (libdda_b200.so).
 *
 * The library runs the hot path of steffen-kiess/dda on one NVIDIA B200:
 * the FFT-convolution matvec of the DDA system A x = x + sqrt(cc) D sqrt(cc) x,
 * the four Krylov solvers built on it, and the D-matrix setup they need.
 * Every entry point below names the reference interface it stands in for
 * (paths relative to the reference tree).
 *
 * Conventions
 *  - Return value 0 on success, a negative DDA_ERR_* code otherwise; the
 *    message of the last failure is available from dda_last_error().
 *  - No C++ exception crosses this boundary.
 *  - Dipole vectors use the reference layout (DDA/DDAParams.hpp:176-186):
 *    structure of arrays [x: nvs][y: nvs][z: nvs] of complex numbers, with
 *    nvs = nv rounded up to a multiple of 16 and the padding zero.  Batches of
 *    right-hand sides are stored one after another: [rhs][3][nvs].
 *    Complex numbers are (re, im) pairs.
 *  - Host buffers are owned by the caller; device buffers passed to
 *    dda_matvec() are owned by the caller; everything else is owned by the
 *    context.  One context per host thread at a time.
 */
#ifndef DDA_CUDA_H
#define DDA_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDA_OK 0
#define DDA_ERR_ARG (-1)         /* invalid argument */
#define DDA_ERR_CUDA (-2)        /* CUDA runtime failure */
#define DDA_ERR_OOM (-3)         /* device allocation failed */
#define DDA_ERR_UNSUPPORTED (-4) /* grid not 2,3,5,7-smooth, size limits */
#define DDA_ERR_BREAKDOWN (-5)   /* Krylov breakdown guard fired */
#define DDA_ERR_MAXITER (-6)     /* "Too many iterations" */
#define DDA_ERR_NOPROGRESS (-7)  /* "Too many iterations w/o increase" */
#define DDA_ERR_CANCELLED (-8)   /* stopped by dda_cancel / dda_serve_cancel */

/* Arithmetic of the matvec and of the Krylov vectors. */
#define DDA_PREC_FP64 0  /* everything in FP64 (the reference's --ftype double) */
#define DDA_PREC_FP32 1  /* complex FP32 vectors/FFTs, FP64 scalars and dot products */
#define DDA_PREC_MIXED 2 /* FP32 inner solves refined by an outer FP64 residual */

/* Solvers, the reference's --iter names (DDA/DDAMain.cpp:647-656). */
#define DDA_SOLVER_QMR 0      /* qmr:      DDA/QmrCs.cpp, DDA/GpuQmrCs.cpp */
#define DDA_SOLVER_BICGSTAB 1 /* bicgstab: DDA/BicgStab.cpp, DDA/GpuBicgStab.cpp */
#define DDA_SOLVER_BICG 2     /* bicg:     DDA/BicgCs.cpp, DDA/GpuBicgCs.cpp */
#define DDA_SOLVER_CGNR 3     /* cgnr:     DDA/Cgnr.cpp, DDA/GpuCgnr.cpp */

typedef struct dda_ctx dda_ctx;

/* Problem description: the fields of DDAParams (DDA/DDAParams.hpp:52-217)
 * the matvec needs. */
typedef struct dda_problem {
  uint32_t nv;               /* occupied dipoles */
  uint32_t box[3];           /* particle box bx, by, bz (dipoles) */
  uint32_t grid[3];          /* FFT grid Gx, Gy, Gz: even, >= 2*box, 2,3,5,7-smooth */
  const uint32_t* positions; /* host, nv*3 grid coordinates (x, y, z) per dipole */
  const uint8_t* materials;  /* host, nv material indices, NULL = all 0 */
  uint32_t nmat;             /* number of materials (<= 256) */
  double kd;                 /* wave number times grid unit */
  double grid_unit;          /* grid unit d in metres */
  const double* dmatrix;     /* optional host D matrix in the reference layout
                                ([Gx][Gz][Gy][6] complex FP64, the output of
                                DMatrixCpu::createDMatrix); NULL = generate it
                                on the GPU from kd */
  int32_t max_rhs;           /* right-hand sides per batch (>= 1) */
  int32_t device;            /* CUDA device ordinal */
  uint32_t flags;            /* DDA_FLAG_* */
} dda_problem;

/* dda_problem.flags: run the y/z passes through three kernels and a plane
 * buffer even when a kx plane fits in shared memory (the path large grids
 * take); used by tests and tuning. */
#define DDA_FLAG_SPLIT_YZ 1u
/* dda_problem.flags: use the runtime-planned FFT kernels even when every grid
 * edge has a compile-time plan; used by tests and tuning. */
#define DDA_FLAG_RUNTIME_PLANS 2u
/* dda_problem.flags: run the y/z passes through the cluster kernel (a
 * thread-block cluster per kx plane exchanging through an L2-resident plane
 * buffer, the path for planes beyond one CTA's shared memory) even when a
 * plane fits; used by tests and tuning.  DDA_FLAG_SPLIT_YZ takes precedence. */
#define DDA_FLAG_SLOT_YZ 4u
/* dda_problem.flags: keep the default y/z batching instead of timing the
 * candidates at dda_create (the autotuner picks, per grid shape, the rows
 * per batch of the plane kernels and the cluster size of the cluster
 * kernel; neither changes the results). */
#define DDA_FLAG_NO_AUTOTUNE 8u
/* dda_problem.flags: launch every solver iteration kernel by kernel instead of
 * replaying captured CUDA graphs of eight iterations (the results are the
 * same; used by tests). */
#define DDA_FLAG_NO_GRAPHS 16u
/* dda_problem.flags: run the fused plane kernel as two groups of half the
 * CTA (or, with DDA_FLAG_YZ_GROUPS4, four groups of a quarter) with their own
 * barriers (the autotuner otherwise chooses between one, two and four
 * groups; the results are the same); used by tests. */
#define DDA_FLAG_YZ_GROUPS2 32u
#define DDA_FLAG_YZ_GROUPS4 64u
/* dda_problem.flags: run the planned y/z passes with one kx plane per cluster
 * of two CTAs (each holding half the plane; the autotuner otherwise chooses
 * between this and one CTA per plane; the results are the same); used by
 * tests. */
#define DDA_FLAG_YZ_PAIR 128u

typedef struct dda_stats {
  int64_t iterations;   /* Krylov iterations (summed over inner solves for MIXED) */
  int64_t matvecs;      /* matvecs issued for this right-hand side */
  int64_t refinements;  /* outer FP64 residual steps (MIXED) */
  double rel_residual;  /* sqrt(best |r|^2 / |b|^2) at exit */
  double res_scale;     /* 1 / |b|^2 */
  int32_t status;       /* 0 or a DDA_ERR_* code */
  int32_t pad;
} dda_stats;

/* Builds the device-side problem: geometry tables, FFT plans and the D
 * matrix (generated on the GPU in FP64 when prob->dmatrix is NULL).
 * Replaces GpuMatVec<T>::create (DDA/GpuMatVec.hpp:85-86),
 * DMatrixGpu<T>::createDMatrix (DDA/DMatrixGpu.cpp:30-41) and
 * DMatrixCpu<T>::createDMatrix (DDA/DMatrixCpu.hpp:42). */
int dda_create(const dda_problem* prob, int precision, dda_ctx** out);

/* Frees every device resource of the context. */
int dda_destroy(dda_ctx* ctx);

/* Message of the last failure on this context (or of the last failed
 * dda_create when ctx is NULL). */
const char* dda_last_error(const dda_ctx* ctx);

/* nvs, the per-component stride of dipole vectors. */
int64_t dda_vec_stride(const dda_ctx* ctx);

/* Sets the couple-constant square roots sqrt(cc) of right-hand side `rhs`:
 * nmat*3 complex FP64 (DiagMatrix3 per material), in reference units.
 * Values that are not finite are rejected (DDA_ERR_ARG).
 * Replaces MatVec<T>::setCoupleConstants (DDA/MatVec.hpp:46) and
 * GpuMatVec<T>::setCoupleConstants (DDA/GpuMatVec.hpp:89). */
int dda_set_cc(dda_ctx* ctx, int rhs, const double* cc_sqrt);

/* result = A arg (conj != 0: conj(A conj(arg)), the adjoint product CGNR
 * uses) for `nrhs` right-hand sides in device memory.  `precision` selects
 * the buffers' element type: DDA_PREC_FP64 (double pairs) or DDA_PREC_FP32
 * (float pairs).  `stream` is a cudaStream_t (NULL = the context stream).
 * Replaces GpuMatVec<T>::apply (DDA/GpuMatVec.hpp:99). */
int dda_matvec(dda_ctx* ctx, const void* d_arg, void* d_res, int conj, int nrhs,
               int precision, void* stream);

/* The same product on host FP64 buffers (copies in, matvec, copies out;
 * FP32 contexts convert on the device).  Replaces MatVec<T>::apply
 * (DDA/MatVec.hpp:54) as implemented by MatVecGpu<T>::apply
 * (DDA/MatVecGpu.cpp:51-68). */
int dda_matvec_host(dda_ctx* ctx, const double* arg, double* res, int conj, int nrhs);

/* Solves A x = sqrt(cc) Einc for `nrhs` right-hand sides (incident fields
 * einc, host FP64, [nrhs][3][nvs]) to relative residual eps and writes the
 * dipole polarisations P = sqrt(cc) x to pol_out (host FP64, same layout).
 * start (may be NULL) holds start polarisations (--load-start-dip-pol).
 * max_iter <= 0 means unlimited.  history (may be NULL) receives the
 * per-iteration relative residuals (the RE_ lines), history_cap per rhs.
 * stats (may be NULL) receives nrhs records.  Returns the first non-zero
 * per-rhs status.  An FP32 context copies the FP64 host vectors as they are
 * and rounds them on the device; from pinned host memory both copies are
 * plain DMA.  Replaces IterativeSolverBase<T>::getPolVec
 * (DDA/IterativeSolverBase.hpp:59) with the GPU solver classes
 * (DDA/GpuIterativeSolver.hpp, DDA/Gpu{QmrCs,BicgStab,BicgCs,Cgnr}.hpp). */
int dda_solve(dda_ctx* ctx, int solver, int nrhs, const double* einc, double eps,
              int64_t max_iter, const double* start, double* pol_out, double* history,
              int64_t history_cap, dda_stats* stats);

/* dda_solve with single-precision host arrays (complex float pairs, same
 * [nrhs][3][nvs] layout): the vectors of the reference's --ftype float path
 * (IterativeSolverBase<float>::getPolVec, DDA/IterativeSolverBase.hpp:59,
 * with std::vector<std::complex<float> >).  On an FP32 context the arrays
 * cross the bus as they are, half the bytes of dda_solve, and the result is
 * dda_solve's rounded to float (the same device arithmetic).  FP64 and
 * MIXED contexts widen the arrays on the host and run dda_solve. */
int dda_solve_f32(dda_ctx* ctx, int solver, int nrhs, const float* einc, double eps, int64_t max_iter,
                  const float* start, float* pol_out, double* history, int64_t history_cap, dda_stats* stats);

/* dda_solve on device buffers of the context precision (double pairs for
 * DDA_PREC_FP64 and DDA_PREC_MIXED, whose outer residual is FP64; float
 * pairs for DDA_PREC_FP32):
 * d_einc [nrhs][3][nvs] in, d_pol [nrhs][3][nvs] out, d_start may be NULL.
 * All work is queued on the context stream; the call returns when the solve
 * has finished.  Replaces GpuIterativeSolver<T>::getPolVec's device part
 * (DDA/GpuIterativeSolver.cpp:78-144) without the host copies. */
int dda_solve_device(dda_ctx* ctx, int solver, int nrhs, const void* d_einc, double eps,
                     int64_t max_iter, const void* d_start, void* d_pol, dda_stats* stats);

/* Asks the solve running on `ctx` (dda_solve / dda_solve_device, called
 * from another thread) to stop: it ends after the round of iterations in
 * flight (at most eight), with every unfinished right-hand side reported as
 * DDA_ERR_CANCELLED and the polarisations of the iterate reached.  A cancel
 * issued while no solve runs stops the next one at its first round; each
 * solve clears the request when it returns.  Safe to call from any thread.
 * No counterpart in the reference (its solves run to completion, exit or
 * abort, DDA/IterativeSolverBase.cpp:56-98). */
int dda_cancel(dda_ctx* ctx);

/* The context stream (a cudaStream_t) on which the library queues its work. */
void* dda_stream(dda_ctx* ctx);

/* Number of kernels the context has launched so far (matvec passes,
 * Krylov steps, setup); a profiling counter. */
int64_t dda_launch_count(const dda_ctx* ctx);

/* FFT grid for a particle box.  DDA_GRID_REFERENCE: fftFit(2 box) per axis,
 * the reference's choice (DDA/DDAParams.cpp:290-335).  DDA_GRID_TUNED: per
 * axis the smallest length >= 2 box with compile-time FFT plans, y and z
 * equal so the y/z passes use them, unless that more than doubles the grid.
 * Any grid >= 2 box gives the same matvec up to rounding (the zero padding
 * makes the circular convolution the exact linear one); the reference's
 * --fft-grid sets it the same way. */
#define DDA_GRID_REFERENCE 0
#define DDA_GRID_TUNED 1
int dda_choose_grid(const uint32_t* box, int policy, uint32_t* grid);

/* Upper bound of the device memory dda_create(prob, precision) takes:
 * `resident` = what the context keeps, `peak` = resident plus the temporary
 * FP64 grid of the D-matrix generation.  Used to admit requests by HBM
 * footprint; no counterpart in the reference. */
int dda_footprint(const dda_problem* prob, int precision, int64_t* resident, int64_t* peak);

/* Layout the context chose for its matvec (working precision: FP32 for
 * DDA_PREC_FP32 and DDA_PREC_MIXED, FP64 otherwise), 8 values:
 * [0] y/z path (0 fused plane kernel, 1 cluster kernel, 2 split path),
 * [1] resident clusters (cluster kernel) or CTAs per kx plane (fused
 * kernels: 1, or 2 for the two-CTA kernel), [2] CTAs per cluster (cluster kernel) or thread
 * groups per CTA (fused kernel: 1, 2 or 4), [3] rows per y batch,
 * [4] dynamic shared memory of the y/z kernel (bytes), [5] grid lines per
 * x tile, [6] compile-time FFT plans (1) or runtime plans (0),
 * [7] device bytes the context holds.  A diagnostic for tuning and
 * benchmark reports; no counterpart in the reference. */
int dda_matvec_layout(const dda_ctx* ctx, int64_t* out);

/* Times the stages of one matvec of nrhs right-hand sides with CUDA events
 * (`reps` repetitions after one warm-up) and writes the mean milliseconds of
 * each stage to ms[4]: x forward, y/z passes, x inverse, total.  The
 * per-phase attribution of the reference's --sync profiling
 * (DDA/GpuMatVec.cpp:149-153). */
int dda_profile_matvec(dda_ctx* ctx, int nrhs, int reps, double* ms);

/* Scattered far field E(n) = i k^2 exp(-i k origin.n) (S - n (n.S)),
 * S = sum_j P_j exp(-i kd n.r_j), for ndir unit directions `dirs` (host,
 * ndir*3, particle frame) and nrhs right-hand sides: out[ndir][nrhs][3]
 * complex (host).  P is `pol` (host, [nrhs][3][nvs]) or, when pol is NULL,
 * the polarisations of the last dda_solve / dda_solve_device on the context.
 * Replaces FieldCalculator<T>::calcField (DDA/FieldCalculator.hpp:57-58,
 * DDA/CpuFieldCalculator.cpp:48-98, DDA/GpuFieldCalculatorInst.cl:27-70) and
 * its per-direction host loop (DDA/FarFieldCalc.cpp:131-155). */
int dda_far_field(dda_ctx* ctx, int nrhs, const double* pol, int64_t ndir, const double* dirs, double* out);

/* dda_far_field(ctx, nrhs, NULL, ndir, dirs, out) without any allocation:
 * the far field of the polarisations of the last solve on the context, with
 * the device copies of `dirs` and `out` kept in one fixed scratch array of
 * 1 MiB per device that is part of the library's device image.  No
 * counterpart in the reference (its far field, DDA/FarFieldCalc.cpp:131-155,
 * allocates its device buffers per call).
 *
 * For callers that must not allocate device memory while they evaluate far
 * fields: a serving loop that keeps solves of other contexts in flight on
 * other streams of the same device (cudaFree waits for the whole device,
 * which would stall those solves), or a process that has handed the free
 * device memory to its solver contexts (dda_far_field's per-call cudaMalloc
 * then fails with DDA_ERR_OOM).
 *
 * Limit: 24*ndir bytes rounded up to 256, plus 48*ndir*nrhs bytes, at most
 * 1 MiB (14,560 directions for one right-hand side, 8,736 for two); larger
 * requests return DDA_ERR_ARG with the sizes in dda_last_error and touch
 * nothing.  Nothing in the scratch needs to start at zero: each call writes
 * every byte it reads.  The first call on each device looks up the scratch
 * address (cudaGetSymbolAddress with that device current) and keeps it for
 * the life of the process, so make that first call before any stream
 * capture begins, and do not call it on a device after cudaDeviceReset (or
 * any other reset of that device's primary context) in the same process:
 * the kept address would no longer be valid.  Every context on
 * a device shares the one scratch array: calls that overlap in time (from
 * two host threads, on any contexts of the same device) race on it and must
 * be serialised by the caller.  Each call returns after `out` is written. */
int dda_far_field_noalloc(dda_ctx* ctx, int nrhs, int64_t ndir, const double* dirs, double* out);

/* Copies the D matrix out in the reference layout ([Gx][Gz][Gy][6] complex
 * FP64, reference units), expanded from the octant the context stores. */
int dda_get_dmatrix(dda_ctx* ctx, double* out);

/* Waits for all work queued on the context stream. */
int dda_synchronize(dda_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* DDA_CUDA_H */
