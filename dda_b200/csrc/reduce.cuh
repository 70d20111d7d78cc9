// reduce.cuh -- deterministic block reductions in FP64 with a last-block
// finaliser.
//
// Every CTA of a reduction writes its partial sums to a fixed slot; the CTA
// that takes the last ticket sums the slots in a fixed order and runs the
// finaliser (the Krylov scalar recurrence of the solver step).  The result is
// independent of CTA scheduling, so a solve gives bit-identical results alone
// and in a batch.  This replaces the reference's two-launch reductions with a
// serial per-work-group sum (LinAlg/GpuLinCombInst.cl:27-169) and its
// host-side scalar round trips (DDA/GpuQmrCs.cpp:146-177).
#pragma once

#include <cuda_runtime.h>

namespace dda {

struct RedSums {
  double2 a;  // complex sum (a dot product)
  double2 b;  // second complex sum
  double n;   // real sum (a squared norm)
  double m;   // second real sum
};

__device__ __forceinline__ double2 dadd2(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}

__device__ __forceinline__ RedSums red_add(RedSums p, RedSums q) {
  RedSums r;
  r.a = dadd2(p.a, q.a);
  r.b = dadd2(p.b, q.b);
  r.n = p.n + q.n;
  r.m = p.m + q.m;
  return r;
}

__device__ __forceinline__ RedSums red_zero() {
  RedSums r;
  r.a = make_double2(0, 0);
  r.b = make_double2(0, 0);
  r.n = 0;
  r.m = 0;
  return r;
}

__device__ __forceinline__ double shfl_d(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }

__device__ __forceinline__ RedSums warp_reduce(RedSums v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.a.x += shfl_d(v.a.x, o); v.a.y += shfl_d(v.a.y, o);
    v.b.x += shfl_d(v.b.x, o); v.b.y += shfl_d(v.b.y, o);
    v.n += shfl_d(v.n, o); v.m += shfl_d(v.m, o);
  }
  return v;
}

// Block-wide sum; the result is valid in thread 0.  NT must be a multiple
// of 32 and at most 1024.
template <int NT>
__device__ __forceinline__ RedSums block_reduce(RedSums v) {
  __shared__ RedSums ws[NT / 32];
  v = warp_reduce(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < NT / 32 ? ws[lane] : red_zero();
    v = warp_reduce(v);
  }
  return v;
}

// Partial-sum slots and tickets for one reduction per right-hand side.
struct RedTarget {
  RedSums* parts;     // [nrhs][nparts]
  unsigned* tickets;  // [nrhs], zero between reductions
  int nparts;         // CTAs contributing per right-hand side
};

// Writes this CTA's partial (slot `part` of `rhs`) and returns true in every
// thread of the CTA that completes the set; `total` (thread 0) then holds the
// fixed-order sum of all slots and the ticket is reset for the next use.
template <int NT>
static __device__ bool block_finish(RedSums v, const RedTarget& t, int rhs, int part, RedSums& total) {
  __shared__ bool last;
  v = block_reduce<NT>(v);
  if (threadIdx.x == 0) {
    t.parts[(size_t)rhs * t.nparts + part] = v;
    __threadfence();
    unsigned k = atomicAdd(&t.tickets[rhs], 1u);
    last = (k == (unsigned)t.nparts - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // fixed-order sum: thread i adds slots i, i+NT, ... in order, then a fixed tree
  RedSums s = red_zero();
  const volatile RedSums* P = t.parts + (size_t)rhs * t.nparts;
  for (int i = threadIdx.x; i < t.nparts; i += NT) {
    RedSums q;
    q.a.x = P[i].a.x; q.a.y = P[i].a.y; q.b.x = P[i].b.x; q.b.y = P[i].b.y;
    q.n = P[i].n; q.m = P[i].m;
    s = red_add(s, q);
  }
  s = block_reduce<NT>(s);
  if (threadIdx.x == 0) {
    total = s;
    t.tickets[rhs] = 0;
  }
  return true;
}

}  // namespace dda
