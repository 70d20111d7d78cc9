// matvec_pair.cuh -- the y/z passes of the matvec with one kx plane per
// cluster of two CTAs (k_yz_pair), for planes whose slab leaves one CTA too
// little shared memory for y work.
//
// k_yz_p keeps the whole slab of a plane (Gz x 3 by complex after the z
// transform) in one CTA; for the 128-rhs spheroid (Gz = 128, by = 64) that is
// 198 KB and leaves room for 10 kz rows of y work, so most warps wait at the
// y stages' barriers.  Here the two CTAs of a cluster share the plane: CTA r
// holds the z positions [r Gz/2, (r+1) Gz/2) of every column.  With an even
// first z radix R0 those are exactly the outputs m < R0/2 (r = 0) or
// m >= R0/2 (r = 1) of every stage-0 butterfly, and every later z stage works
// inside one half.  So:
//
//   z stage 0     each CTA takes half of the columns, reads them from HBM and
//                 stores each butterfly's outputs into the CTA that owns
//                 their positions (distributed shared memory);
//   -- cluster barrier --
//   z stages 1..  each CTA on its half;
//   y pass        each CTA on its Gz/2 kz rows, with room for four times the
//                 row buffers (D-hat multiply as in k_yz_p);
//   z stages ..1  inverse, each CTA on its half;
//   -- cluster barrier --
//   z stage 0     inverse, each CTA on half of the columns, reading the
//                 positions of both halves (distributed shared memory), and
//                 writes z < bz to HBM;
//   -- cluster barrier -- (neither CTA leaves while the other reads it)
//
// Every butterfly does the arithmetic of k_yz_p, so the results are the same
// bits.  GR > 1 splits each CTA into thread groups with named barriers as in
// k_yz_p.
#pragma once

#include <cooperative_groups.h>

#include "matvec_planned.cuh"

namespace dda {

// Shared memory (complex offsets): z twiddles [0, Gz), y twiddles
// [Gz, Gz+Gy), the half slab [Gz/2][q], then the row buffers [nrw][3][py].
__host__ __device__ inline int pair_slab_off(const MvGeom& g) { return g.Gz + g.Gy; }
__host__ __device__ inline int pair_rows_off(const MvGeom& g, const YzGeom& y) {
  return g.Gz + g.Gy + (g.Gz / 2) * y.q;
}

// z stage 0 on columns [l0, l0+lw): outputs m < R/2 to slab0 (position p),
// m >= R/2 to slab1 (position p - Gz/2).
template <typename T, int G, typename PZ, bool HALF>
__device__ __forceinline__ void zpair_first(const typename C2<T>::t* __restrict__ plane,
                                            typename C2<T>::t* slab0, typename C2<T>::t* slab1, int q,
                                            int by, int bz, int tid, int l0, int lw, int bar) {
  typedef typename C2<T>::t T2;
  constexpr int R = PZ::r[0], S0 = PZ::N / R, HZ = PZ::N / 2;
  const T2* sm = smem_at<T>(0);
  const int nb = by * bz;
  for (int b = tid; b < lw * S0; b += G) {
    const int j = b / lw, l = l0 + (b - j * lw);
    const int c = l / by, y = l - c * by;
    T2 v[R];
#pragma unroll
    for (int m = 0; m < R; m++) {
      const int z = j + m * S0;
      v[m] = (HALF ? m < R / 2 : z < bz) ? plane[c * nb + z * by + y] : czero<T2>();
    }
    butterfly<PZ, 0, false>(v, j, sm);
#pragma unroll
    for (int m = 0; m < R; m++) {
      const int p = j + m * S0;
      if (m < R / 2) slab0[p * q + l] = v[m];
      else slab1[(p - HZ) * q + l] = v[m];
    }
  }
  group_sync<G>(bar);
}

// inverse z stage 0 on columns [l0, l0+lw), reading both halves, writing
// z < bz to the plane.
template <typename T, int G, typename PZ, bool HALF>
__device__ __forceinline__ void zpair_last(typename C2<T>::t* __restrict__ plane, const typename C2<T>::t* slab0,
                                           const typename C2<T>::t* slab1, int q, int by, int bz, int tid,
                                           int l0, int lw) {
  typedef typename C2<T>::t T2;
  constexpr int R = PZ::r[0], S0 = PZ::N / R, HZ = PZ::N / 2;
  const T2* sm = smem_at<T>(0);
  const int nb = by * bz;
  for (int b = tid; b < lw * S0; b += G) {
    const int j = b / lw, l = l0 + (b - j * lw);
    const int c = l / by, y = l - c * by;
    T2 v[R];
#pragma unroll
    for (int m = 0; m < R; m++) {
      const int p = j + m * S0;
      v[m] = m < R / 2 ? slab0[p * q + l] : slab1[(p - HZ) * q + l];
    }
    butterfly<PZ, 0, true>(v, j, sm);
#pragma unroll
    for (int m = 0; m < R; m++) {
      const int z = j + m * S0;
      if (HALF ? m < R / 2 : z < bz) plane[c * nb + z * by + y] = v[m];
    }
  }
}

// grid (2 Gx, nrhs) in clusters of two CTAs along x: cluster kx = blockIdx.x / 2.
template <typename T, int NT, typename PZ, typename PY, bool HALF = false, int GR = 1>
__global__ void __launch_bounds__(NT, 1) k_yz_pair(typename C2<T>::t* __restrict__ xhat,
                                                const typename C2<T>::t* __restrict__ dc, MvGeom g, YzGeom y,
                                                FftPlanDev pz, FftPlanDev pyp,
                                                const KrylovState* __restrict__ st, int mvskip) {
  static_assert(PY::K >= 2 && PZ::K >= 2, "tuned plans have at least two stages");
  static_assert(PZ::r[0] % 2 == 0, "the halves need an even first z radix");
  static_assert(!HALF || PY::r[0] % 2 == 0, "HALF needs an even first radix");
  typedef typename C2<T>::t T2;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int kx = blockIdx.x >> 1, b = blockIdx.y;  // kx: position after the x transform
  if (rhs_idle(st, b, mvskip)) return;  // the same for both CTAs of the cluster
  constexpr int HZ = PZ::N / 2;
  const int soff = pair_slab_off(g), roff = pair_rows_off(g, y);
  T2* S = smem_at<T>(soff);  // this CTA's half: positions [rank HZ, (rank+1) HZ)
  T2* peer = cluster.map_shared_rank(S, rank ^ 1);
  T2* slab0 = rank == 0 ? S : peer;
  T2* slab1 = rank == 0 ? peer : S;
  T2* plane = xhat + ((size_t)b * g.Gx + kx) * 3 * g.nlines;
  stage_twiddles<T, NT>(0, pz);
  stage_twiddles0<T, NT, PY>(g.Gz, pyp);  // only y stage 0 has twiddles in two-stage plans
  __syncthreads();
  constexpr int G = NT / GR;
  const int grp = GR == 1 ? 0 : (int)threadIdx.x / G;
  const int tid = (int)threadIdx.x - grp * G;
  const int bar = GR == 1 ? 0 : 1 + grp;
  const int w3 = 3 * g.by;
  // z stage 0: this CTA's half of the columns, split between its groups
  const int cw = w3 / 2, c0 = rank * cw, cn = rank == 1 ? w3 - cw : cw;
  const int l0 = c0 + grp * (cn / GR), lw = grp == GR - 1 ? cn - grp * (cn / GR) : cn / GR;
  // the peer's slab is written below: it must have started (cluster-wide
  // barrier before the first distributed shared-memory access)
  cluster.sync();
  zpair_first<T, G, PZ, HALF>(plane, slab0, slab1, y.q, g.by, g.bz, tid, l0, lw, bar);
  cluster.sync();  // both halves complete
  // z stages 1.. on this CTA's half, all columns, split between its groups
  const int m0 = grp * (w3 / GR), mw = grp == GR - 1 ? w3 - m0 : w3 / GR;
  pstages<T, PZ, false, G, 1, PZ::K, 2>(soff + m0, mw, 1, y.q, 0, tid, bar);
  if (GR > 1) __syncthreads();
  {
    const int kxf = g.fx[kx];
    const int nrg = y.nrw / GR;
    const int rog = roff + grp * nrg * 3 * y.py;
    for (int r0 = grp * nrg; r0 < HZ; r0 += GR * nrg) {  // local rows; position rank HZ + r0
      const int nr = min(nrg, HZ - r0);
      rows_stage0<T, G, PY, false, HALF>(S, r0, nr, y.q, g.by, rog, y.py, g.Gz, tid, bar);
      pstages<T, PY, false, G, 1, PY::K - 1>(rog, 3 * nr, y.py, 1, g.Gz, tid, bar);
      rows_dmul<T, G, PY, PZ>(rank * HZ + r0, nr, rog, y.py, dc, g, kxf, tid, bar);
      pstages<T, PY, true, G, 1, PY::K - 1>(rog, 3 * nr, y.py, 1, g.Gz, tid, bar);
      rows_stage0<T, G, PY, true, HALF>(S, r0, nr, y.q, g.by, rog, y.py, g.Gz, tid, bar);
    }
  }
  if (GR > 1) __syncthreads();
  pstages<T, PZ, true, G, 1, PZ::K, 2>(soff + m0, mw, 1, y.q, 0, tid, bar);
  cluster.sync();  // both halves transformed back
  zpair_last<T, G, PZ, HALF>(plane, slab0, slab1, y.q, g.by, g.bz, tid, l0, lw);
  cluster.sync();  // the peer has read this CTA's half
}

}  // namespace dda
