// matvec_slot.cuh -- the y/z passes of the matvec for kx planes too large for
// one CTA's shared memory (k_yz_slot).
//
// A thread-block cluster of `cl` CTAs owns one kx plane at a time and walks a
// list of (kx, rhs) items (persistent: the grid holds as many clusters as
// can be resident).  The plane passes through a per-cluster buffer, the
// slot S[kz][wp] (row kz holds the three components' y < by after the z
// transform), that is small enough to stay in L2:
//
//   phase Z    each CTA takes column tiles (tc columns of the 3 by plane
//              columns): read from xhat (z < bz, zero padded to Gz), forward
//              z FFT in shared memory, store to the slot;
//   -- cluster barrier --
//   phase Y    each CTA takes batches of kz rows: read from the slot (y < by,
//              zero padded to Gy), forward y FFT, D-hat multiply, inverse y
//              FFT, store y < by back to the slot;
//   -- cluster barrier --
//   phase Z'   each CTA takes the same column tiles as in phase Z: read the
//              slot, inverse z FFT, store z < bz to xhat.
//
// The barrier (barrier.cluster arrive.release / wait.acquire) orders the
// slot stores of one phase before the loads of the next across the
// cluster's CTAs; the slot is read with ld.global.cg so no stale L1 line of
// an earlier item is seen.  The plane is read through the non-coherent path:
// within the kernel only the cluster that owns an item reads or writes its
// plane, and it reads a plane's elements before it writes them.  A CTA writes in phase Z only the columns it
// reads back in phase Z', so consecutive items need no third barrier.
#pragma once

#include <cooperative_groups.h>

#include "matvec_kernels.cuh"
#include "matvec_planned.cuh"

namespace dda {

struct SlotGeom {
  int wp;   // slot row pitch (>= 3 by)
  int nrw;  // rows per y batch
  int py;   // row buffer pitch (Gy + 1)
};

// z tile width: a 128-byte row segment per tile row in either precision.
template <typename T> struct SlotTc { static constexpr int value = sizeof(T) == 4 ? 32 : 16; };
// Global loads a thread issues before it consumes the first of them (the
// loads are volatile asm, kept in program order, so batching is explicit).
template <typename T> struct SlotU { static constexpr int value = sizeof(T) == 4 ? 8 : 4; };

// L2 eviction priorities (createpolicy, sm_80+).  The clusters' slots (one
// [Gz][wp] buffer each, together up to about 100 MB) are written and read
// back four times per item and are marked evict_last; the planes of xhat are
// read once and written once per item and are marked evict_first, so that the
// stream of planes does not push the slots out of the 126 MB L2.
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// slot: L2 only (ld/st .cg), with a cache policy
__device__ __forceinline__ float2 slot_ld(const float2* a, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.cg.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double2 slot_ld(const double2* a, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void slot_st(float2* a, float2 v, uint64_t pol) {
  asm volatile("st.global.cg.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(v.x), "f"(v.y), "l"(pol));
}
__device__ __forceinline__ void slot_st(double2* a, double2 v, uint64_t pol) {
  asm volatile("st.global.cg.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol));
}
// plane: read-only within the kernel (non-coherent path) / plain store
__device__ __forceinline__ float2 plane_ld(const float2* a, uint64_t pol) {
  float2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double2 plane_ld(const double2* a, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void plane_st(float2* a, float2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(v.x), "f"(v.y), "l"(pol));
}
__device__ __forceinline__ void plane_st(double2* a, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(v.x), "d"(v.y), "l"(pol));
}

// Shared memory (complex offsets): z twiddles [0, Gz), y twiddles
// [Gz, Gz+Gy), then either the z tile [Gz][tc+1] or the row buffers
// [nrw][3][py].
__host__ __device__ inline int slot_work_off(const MvGeom& g) { return g.Gz + g.Gy; }

template <typename T>
__host__ inline size_t slot_smem_bytes(const MvGeom& g, int nrw) {
  const size_t s = sizeof(typename C2<T>::t);
  const size_t tile = (size_t)g.Gz * (SlotTc<T>::value + 1);
  const size_t rows = (size_t)nrw * 3 * (g.Gy + 1);
  return ((size_t)g.Gz + g.Gy + std::max(tile, rows)) * s;
}

// HALF (planned plans only): the box is half the grid in y and z and the first
// radices are even, so stage-0 input m is zero padding exactly for m >= R / 2
// and the inverse keeps exactly the outputs m < R / 2 (as in k_yz_p).
template <typename P>
__host__ __device__ constexpr bool even_first_radix() {
  if constexpr (std::is_void<P>::value) return false;
  else return P::r[0] % 2 == 0;
}

// ---- phase Z: column tile [c0, c0+tc) of the plane -------------------------
template <typename T, int NT, typename PZ, bool HALF = false>
__device__ __forceinline__ void slot_cols_fwd(const typename C2<T>::t* __restrict__ plane,
                                              typename C2<T>::t* __restrict__ slot, const MvGeom& g,
                                              const SlotGeom& sg, const FftPlanDev& pz, int c0, uint64_t keep,
                                              uint64_t stream) {
  typedef typename C2<T>::t T2;
  constexpr int TC = SlotTc<T>::value, P = TC + 1;
  const int toff = slot_work_off(g);
  T2* tile = smem_at<T>(toff);
  const int W = 3 * g.by, nb = g.by * g.bz;
  if constexpr (std::is_void<PZ>::value) {
    constexpr int U = SlotU<T>::value;
    for (int i0 = 0; i0 < g.Gz * TC; i0 += U * NT) {
      T2 v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * NT + threadIdx.x;
        const int z = i / TC, l = i - z * TC, gl = c0 + l;
        v[u] = czero<T2>();
        if (i < g.Gz * TC && z < g.bz && gl < W) {
          const int c = gl / g.by, y = gl - c * g.by;
          v[u] = plane_ld(plane + c * nb + z * g.by + y, stream);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * NT + threadIdx.x;
        const int z = i / TC, l = i - z * TC;
        if (i < g.Gz * TC) tile[z * P + l] = v[u];
      }
    }
    __syncthreads();
    fft_lines<T, NT, false>(toff, TC, 1, P, true, pz, 0);
  } else {
    constexpr int R = PZ::r[0], S0 = PZ::N / R;
    constexpr int UI = SlotU<T>::value * 2 / R > 0 ? SlotU<T>::value * 2 / R : 1;  // items per batch
    for (int b0 = 0; b0 < TC * S0; b0 += UI * NT) {
      T2 v[UI][R];
#pragma unroll
      for (int u = 0; u < UI; u++) {
        const int b = b0 + u * NT + threadIdx.x;
        const int j = b / TC, l = b - j * TC, gl = c0 + l;
        const bool live = b < TC * S0 && gl < W;
        const int c = live ? gl / g.by : 0, y = gl - c * g.by;
#pragma unroll
        for (int m = 0; m < R; m++) {
          const int z = j + m * S0;
          v[u][m] = (live && (HALF ? m < R / 2 : z < g.bz)) ? plane_ld(plane + c * nb + z * g.by + y, stream)
                                                             : czero<T2>();
        }
      }
#pragma unroll
      for (int u = 0; u < UI; u++) {
        const int b = b0 + u * NT + threadIdx.x;
        if (b < TC * S0) {
          const int j = b / TC, l = b - j * TC;
          butterfly<PZ, 0, false>(v[u], j, smem_at<T>(0));
#pragma unroll
          for (int m = 0; m < R; m++) tile[(j + m * S0) * P + l] = v[u][m];
        }
      }
    }
    __syncthreads();
    plines<T, PZ, NT, false, 1, PZ::K>(toff, TC, 1, P, 0);
  }
  for (int i = threadIdx.x; i < g.Gz * TC; i += NT) {
    const int kz = i / TC, l = i - kz * TC;
    if (c0 + l < W) slot_st(slot + (size_t)kz * sg.wp + c0 + l, tile[kz * P + l], keep);
  }
  __syncthreads();
}

// ---- phase Z': inverse of the same column tile -----------------------------
template <typename T, int NT, typename PZ, bool HALF = false>
__device__ __forceinline__ void slot_cols_inv(typename C2<T>::t* __restrict__ plane,
                                              const typename C2<T>::t* __restrict__ slot, const MvGeom& g,
                                              const SlotGeom& sg, const FftPlanDev& pz, int c0, uint64_t keep,
                                              uint64_t stream) {
  typedef typename C2<T>::t T2;
  constexpr int TC = SlotTc<T>::value, P = TC + 1;
  const int toff = slot_work_off(g);
  T2* tile = smem_at<T>(toff);
  const int W = 3 * g.by, nb = g.by * g.bz;
  constexpr int U = SlotU<T>::value;
  for (int i0 = 0; i0 < g.Gz * TC; i0 += U * NT) {
    T2 v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + u * NT + threadIdx.x;
      const int kz = i / TC, l = i - kz * TC;
      v[u] = (i < g.Gz * TC && c0 + l < W) ? slot_ld(slot + (size_t)kz * sg.wp + c0 + l, keep) : czero<T2>();
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + u * NT + threadIdx.x;
      const int kz = i / TC, l = i - kz * TC;
      if (i < g.Gz * TC) tile[kz * P + l] = v[u];
    }
  }
  __syncthreads();
  if constexpr (std::is_void<PZ>::value) {
    fft_lines<T, NT, true>(toff, TC, 1, P, true, pz, 0);
    for (int i = threadIdx.x; i < g.bz * TC; i += NT) {
      const int z = i / TC, l = i - z * TC, gl = c0 + l;
      if (gl < W) {
        const int c = gl / g.by, y = gl - c * g.by;
        plane_st(plane + c * nb + z * g.by + y, tile[z * P + l], stream);
      }
    }
  } else {
    plines<T, PZ, NT, true, 1, PZ::K>(toff, TC, 1, P, 0);
    constexpr int R = PZ::r[0], S0 = PZ::N / R;
    for (int b = threadIdx.x; b < TC * S0; b += NT) {
      const int j = b / TC, l = b - j * TC, gl = c0 + l;
      T2 v[R];
#pragma unroll
      for (int m = 0; m < R; m++) v[m] = tile[(j + m * S0) * P + l];
      butterfly<PZ, 0, true>(v, j, smem_at<T>(0));
      if (gl < W) {
        const int c = gl / g.by, y = gl - c * g.by;
#pragma unroll
        for (int m = 0; m < R; m++) {
          const int z = j + m * S0;
          if (HALF ? m < R / 2 : z < g.bz) plane_st(plane + c * nb + z * g.by + y, v[m], stream);
        }
      }
    }
  }
  __syncthreads();
}

// ---- phase Y: kz rows [kz0, kz0+nr) -----------------------------------------
// Planned: y stage 0 fused with the slot read / write, the last forward
// stage, D-hat and the first inverse stage in registers (rows_dmul).
template <typename T, int NT, typename PY, bool INV, bool HALF = false>
__device__ __forceinline__ void slot_rows_stage0(typename C2<T>::t* __restrict__ slot, const MvGeom& g,
                                                 const SlotGeom& sg, int kz0, int nr, int ro, uint64_t keep) {
  typedef typename C2<T>::t T2;
  constexpr int R = PY::r[0], S0 = PY::N / R;
  T2* sm = smem_at<T>(0);
  const int total = nr * 3 * S0;
  if (!INV) {
    constexpr int UI = SlotU<T>::value * 2 / R > 0 ? SlotU<T>::value * 2 / R : 1;
    for (int i0 = 0; i0 < total; i0 += UI * NT) {
      T2 v[UI][R];
#pragma unroll
      for (int u = 0; u < UI; u++) {
        const int it = i0 + u * NT + threadIdx.x;
        const int j = it % S0, rc = it / S0;
        const int row = rc / 3, c = rc - 3 * row;
        const T2* srow = slot + (size_t)(kz0 + row) * sg.wp + c * g.by;
#pragma unroll
        for (int m = 0; m < R; m++) {
          const int yy = j + m * S0;
          v[u][m] = (it < total && (HALF ? m < R / 2 : yy < g.by)) ? slot_ld(srow + yy, keep) : czero<T2>();
        }
      }
#pragma unroll
      for (int u = 0; u < UI; u++) {
        const int it = i0 + u * NT + threadIdx.x;
        if (it < total) {
          const int j = it % S0, rc = it / S0;
          butterfly<PY, 0, false>(v[u], j, sm + g.Gz);
#pragma unroll
          for (int m = 0; m < R; m++) sm[ro + rc * sg.py + j + m * S0] = v[u][m];
        }
      }
    }
  } else {
    for (int it = threadIdx.x; it < total; it += NT) {
      const int j = it % S0, rc = it / S0;
      const int row = rc / 3, c = rc - 3 * row;
      T2* srow = slot + (size_t)(kz0 + row) * sg.wp + c * g.by;
      const int rb = ro + rc * sg.py;
      T2 v[R];
#pragma unroll
      for (int m = 0; m < R; m++) v[m] = sm[rb + j + m * S0];
      butterfly<PY, 0, true>(v, j, sm + g.Gz);
#pragma unroll
      for (int m = 0; m < R; m++) {
        const int yy = j + m * S0;
        if (HALF ? m < R / 2 : yy < g.by) slot_st(srow + yy, v[m], keep);
      }
    }
  }
  __syncthreads();
}

template <typename T, int NT, typename PY, typename PZ, bool HALF = false>
__device__ __forceinline__ void slot_rows(typename C2<T>::t* __restrict__ slot,
                                          const typename C2<T>::t* __restrict__ dc, const MvGeom& g,
                                          const SlotGeom& sg, const FftPlanDev& pyp, int kxf, int kz0, int nr,
                                          uint64_t keep) {
  typedef typename C2<T>::t T2;
  const int ro = slot_work_off(g);
  if constexpr (std::is_void<PY>::value) {
    T2* Rb = smem_at<T>(ro);
    constexpr int U = SlotU<T>::value;
    const int total = nr * 3 * g.Gy;
    for (int i0 = 0; i0 < total; i0 += U * NT) {
      T2 v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * NT + threadIdx.x;
        const int rc = i / g.Gy, yy = i - rc * g.Gy;
        const int row = rc / 3, c = rc - 3 * row;
        v[u] = (i < total && yy < g.by) ? slot_ld(slot + (size_t)(kz0 + row) * sg.wp + c * g.by + yy, keep)
                                        : czero<T2>();
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * NT + threadIdx.x;
        const int rc = i / g.Gy, yy = i - rc * g.Gy;
        if (i < total) Rb[rc * sg.py + yy] = v[u];
      }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int row = w; row < nr; row += NT / 32)
      warp_row<T>(ro + row * 3 * sg.py, dc, g, sg.py, pyp, g.Gz, kxf, g.fz[kz0 + row], lane);
    __syncthreads();
    for (int i = threadIdx.x; i < nr * 3 * g.by; i += NT) {
      const int rc = i / g.by, yy = i - rc * g.by;
      const int row = rc / 3, c = rc - 3 * row;
      slot_st(slot + (size_t)(kz0 + row) * sg.wp + c * g.by + yy, Rb[rc * sg.py + yy], keep);
    }
    __syncthreads();
  } else {
    slot_rows_stage0<T, NT, PY, false, HALF>(slot, g, sg, kz0, nr, ro, keep);
    pstages<T, PY, false, NT, 1, PY::K - 1>(ro, 3 * nr, sg.py, 1, g.Gz, threadIdx.x);
    rows_dmul<T, NT, PY, PZ>(kz0, nr, ro, sg.py, dc, g, kxf, (int)threadIdx.x, 0);
    pstages<T, PY, true, NT, 1, PY::K - 1>(ro, 3 * nr, sg.py, 1, g.Gz, threadIdx.x);
    slot_rows_stage0<T, NT, PY, true, HALF>(slot, g, sg, kz0, nr, ro, keep);
  }
}

// grid: (clusters x cl) CTAs in clusters of cl along x.  Items are (kx, rhs)
// pairs, item i = (order[i / nrhs], i % nrhs): `order` lists the kx
// positions so that the two planes sharing a D-hat octant plane (kx and
// -kx) come together.  slots: one [Gz][wp] buffer per cluster.
template <typename T, int NT, typename PZ, typename PY, bool HALF = false>
__global__ void __launch_bounds__(NT, 1) k_yz_slot(typename C2<T>::t* __restrict__ xhat,
                                                const typename C2<T>::t* __restrict__ dc, MvGeom g,
                                                SlotGeom sg, const uint32_t* __restrict__ order, int nrhs,
                                                typename C2<T>::t* __restrict__ slots, FftPlanDev pz,
                                                FftPlanDev pyp, const KrylovState* __restrict__ st,
                                                int mvskip) {
  typedef typename C2<T>::t T2;
  static_assert(std::is_void<PZ>::value == std::is_void<PY>::value, "both axes planned or neither");
  static_assert(!HALF || (even_first_radix<PZ>() && even_first_radix<PY>()),
                "HALF needs planned axes with an even first radix");
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int cl = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int cid = blockIdx.x / cl, ncl = gridDim.x / cl;
  constexpr int TC = SlotTc<T>::value;
  T2* slot = slots + (size_t)cid * g.Gz * sg.wp;
  stage_twiddles<T, NT>(0, pz);
  stage_twiddles<T, NT>(g.Gz, pyp);
  __syncthreads();
  const int W = 3 * g.by;
  const int nchunks = (W + TC - 1) / TC;
  const int nbatches = (g.Gz + sg.nrw - 1) / sg.nrw;
  const int nitems = g.Gx * nrhs;
  const uint64_t keep = l2_evict_last(), stream = l2_evict_first();
  for (int it = cid; it < nitems; it += ncl) {
    const int kx = (int)order[it / nrhs], b = it % nrhs;
    if (rhs_idle(st, b, mvskip)) continue;  // the same for every CTA of the cluster
    T2* plane = xhat + ((size_t)b * g.Gx + kx) * 3 * g.nlines;
    for (int ch = rank; ch < nchunks; ch += cl) slot_cols_fwd<T, NT, PZ, HALF>(plane, slot, g, sg, pz, ch * TC, keep, stream);
    cluster.sync();
    const int kxf = g.fx[kx];
    for (int bt = rank; bt < nbatches; bt += cl) {
      const int kz0 = bt * sg.nrw;
      slot_rows<T, NT, PY, PZ, HALF>(slot, dc, g, sg, pyp, kxf, kz0, min(sg.nrw, g.Gz - kz0), keep);
    }
    cluster.sync();
    for (int ch = rank; ch < nchunks; ch += cl) slot_cols_inv<T, NT, PZ, HALF>(plane, slot, g, sg, pz, ch * TC, keep, stream);
  }
}

}  // namespace dda
