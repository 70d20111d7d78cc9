// matvec_planned.cuh -- the y/z passes of the matvec with compile-time FFT
// plans (fft_plan.cuh) for the tuned grid lengths.
//
// Per kx plane (k_yz_p), shared memory as for k_yz:
//   z stage 0 runs on the fly while the plane is read from HBM (zero rows
//   z >= bz are never stored), the remaining z stages run on the slab;
//   each warp then takes kz rows: y stage 0 reads the row straight from the
//   slab (zero padded), middle stages run on the warp's row buffer, and the
//   last forward stage, the D-hat multiply and the first inverse stage are
//   done in registers by one thread for all three components (the blocks of
//   the last stage are contiguous, so no shared-memory pass separates them);
//   the inverse y stage 0 writes the kept y < by entries back to the slab;
//   the inverse z stages end with stage 0 writing z < bz to HBM.
#pragma once

#include <vector>

#include "fft_plan.cuh"
#include "matvec_kernels.cuh"

namespace dda {

// Grid lengths with compile-time plans, and those whose kx plane the fused
// plane kernel k_yz_p handles (y and z both of that length).
#define DDA_TUNED_LENGTHS(X)                                                                               \
  X(32) X(48) X(56) X(64) X(80) X(96) X(100) X(112) X(120) X(128) X(144) X(160) X(168) X(192) X(200) X(224) \
  X(240) X(256) X(288) X(320) X(384) X(512)
#define DDA_FUSED_LENGTHS(X) X(32) X(48) X(56) X(64) X(80) X(96) X(100) X(112) X(120) X(128)

// Tuned plans: a large first radix and a last radix of at most 8, so the
// fused last stage holds 3 x R_last complex values per thread.
template <int N> struct PlanFor { typedef void type; };
template <> struct PlanFor<32> { typedef Plan<4, 8> type; };
template <> struct PlanFor<48> { typedef Plan<6, 8> type; };
template <> struct PlanFor<56> { typedef Plan<7, 8> type; };
template <> struct PlanFor<64> { typedef Plan<8, 8> type; };
template <> struct PlanFor<80> { typedef Plan<10, 8> type; };
template <> struct PlanFor<96> { typedef Plan<12, 8> type; };
template <> struct PlanFor<100> { typedef Plan<20, 5> type; };
template <> struct PlanFor<112> { typedef Plan<14, 8> type; };
template <> struct PlanFor<120> { typedef Plan<15, 8> type; };
template <> struct PlanFor<128> { typedef Plan<16, 8> type; };
template <> struct PlanFor<144> { typedef Plan<18, 8> type; };
template <> struct PlanFor<160> { typedef Plan<20, 8> type; };
template <> struct PlanFor<168> { typedef Plan<21, 8> type; };
template <> struct PlanFor<192> { typedef Plan<24, 8> type; };
template <> struct PlanFor<200> { typedef Plan<25, 8> type; };
template <> struct PlanFor<224> { typedef Plan<28, 8> type; };
template <> struct PlanFor<240> { typedef Plan<30, 8> type; };
template <> struct PlanFor<256> { typedef Plan<8, 4, 8> type; };
template <> struct PlanFor<288> { typedef Plan<6, 6, 8> type; };
template <> struct PlanFor<320> { typedef Plan<5, 8, 8> type; };
template <> struct PlanFor<384> { typedef Plan<6, 8, 8> type; };
template <> struct PlanFor<512> { typedef Plan<8, 8, 8> type; };

// Radices of the tuned plan for n (host side), empty when there is none.
inline std::vector<int> tuned_radices(int n) {
  auto get = [](auto p) { return std::vector<int>(std::begin(decltype(p)::r), std::end(decltype(p)::r)); };
  switch (n) {
#define C(N) \
  case N: return get(typename PlanFor<N>::type());
    DDA_TUNED_LENGTHS(C)
#undef C
    default: return {};
  }
}


// ---- z stage 0 fused with the plane read / write (whole CTA) -------------
// HALF: the box is half the grid along the transformed axis (bz = Gz / 2,
// first radix even), so inputs z = j + m S0 are zero exactly for m >= R / 2
// and the inverse keeps exactly the outputs m < R / 2: with that known at
// compile time the zero operands and the unused outputs fold away.
// Columns [l0, l0 + lw) of the W = 3 by columns, by the G threads of a group
// (tid in [0, G), barrier `bar`: 0 = the whole CTA).
template <typename T, int G, typename PZ, bool HALF = false>
__device__ __forceinline__ void zp_first(const typename C2<T>::t* __restrict__ plane, int soff, int q,
                                         int by, int bz, int twz, int tid, int l0, int lw, int bar) {
  typedef typename C2<T>::t T2;
  constexpr int R = PZ::r[0], S0 = PZ::N / R;
  T2* sm = smem_at<T>(0);
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
    butterfly<PZ, 0, false>(v, j, sm + twz);
#pragma unroll
    for (int m = 0; m < R; m++) sm[soff + (j + m * S0) * q + l] = v[m];
  }
  group_sync<G>(bar);
}

template <typename T, int G, typename PZ, bool HALF = false>
__device__ __forceinline__ void zp_last(typename C2<T>::t* __restrict__ plane, int soff, int q, int by,
                                        int bz, int twz, int tid, int l0, int lw) {
  typedef typename C2<T>::t T2;
  constexpr int R = PZ::r[0], S0 = PZ::N / R;
  T2* sm = smem_at<T>(0);
  const int nb = by * bz;
  for (int b = tid; b < lw * S0; b += G) {
    const int j = b / lw, l = l0 + (b - j * lw);
    const int c = l / by, y = l - c * by;
    T2 v[R];
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = sm[soff + (j + m * S0) * q + l];
    butterfly<PZ, 0, true>(v, j, sm + twz);
#pragma unroll
    for (int m = 0; m < R; m++) {
      const int z = j + m * S0;
      if (HALF ? m < R / 2 : z < bz) plane[c * nb + z * by + y] = v[m];
    }
  }
}

// ---- fused last y stage: forward, D-hat, inverse in registers -------------
// Row buffer at shared offset ro (three lines, pitch py); kx, kz are
// frequencies.  One warp.
template <typename T, typename PY>
__device__ __forceinline__ void row_dmul_stage(int ro, int py, const typename C2<T>::t* __restrict__ dc,
                                               const MvGeom& g, int kx, int kz, int lane) {
  typedef typename C2<T>::t T2;
  constexpr int K = PY::K;
  constexpr int R = PY::r[K - 1];
  constexpr int NB = PY::N / R;
  T2* sm = smem_at<T>(0);
  for (int t = lane; t < NB; t += 32) {
    T2 v0[R], v1[R], v2[R];
    const int base = ro + t * R;
#pragma unroll
    for (int m = 0; m < R; m++) {
      v0[m] = sm[base + m];
      v1[m] = sm[base + py + m];
      v2[m] = sm[base + 2 * py + m];
    }
    DftN<R, false, T2>::run(v0);
    DftN<R, false, T2>::run(v1);
    DftN<R, false, T2>::run(v2);
#pragma unroll
    for (int m = 0; m < R; m++) {
      T2 d[6];
      load_dhat<T>(dc, g.Gx, g.Gy, g.Gz, kx, PY::freq_of(t * R + m), kz, d);
      dmul(d, v0[m], v1[m], v2[m]);
    }
    DftN<R, true, T2>::run(v0);
    DftN<R, true, T2>::run(v1);
    DftN<R, true, T2>::run(v2);
#pragma unroll
    for (int m = 0; m < R; m++) {
      sm[base + m] = v0[m];
      sm[base + py + m] = v1[m];
      sm[base + 2 * py + m] = v2[m];
    }
  }
  __syncwarp();
}

// y stage 0 fused with the row read from the slab (row kz, y < by) or the
// write back; items (component, butterfly) over the warp's lanes.
template <typename T, typename PY, bool INV>
__device__ __forceinline__ void row_stage0(typename C2<T>::t* S, int kz, int q, int by, int ro, int py,
                                           int twy, int lane) {
  typedef typename C2<T>::t T2;
  constexpr int R = PY::r[0], S0 = PY::N / R;
  T2* sm = smem_at<T>(0);
  for (int it = lane; it < 3 * S0; it += 32) {
    const int c = it / S0, j = it - c * S0;
    T2 v[R];
    if (!INV) {
#pragma unroll
      for (int m = 0; m < R; m++) {
        const int y = j + m * S0;
        v[m] = y < by ? S[kz * q + c * by + y] : czero<T2>();
      }
      butterfly<PY, 0, false>(v, j, sm + twy);
#pragma unroll
      for (int m = 0; m < R; m++) sm[ro + c * py + j + m * S0] = v[m];
    } else {
#pragma unroll
      for (int m = 0; m < R; m++) v[m] = sm[ro + c * py + j + m * S0];
      butterfly<PY, 0, true>(v, j, sm + twy);
#pragma unroll
      for (int m = 0; m < R; m++) {
        const int y = j + m * S0;
        if (y < by) S[kz * q + c * by + y] = v[m];
      }
    }
  }
  __syncwarp();
}

// ---- CTA-wide batches of kz rows ------------------------------------------
// Rows [kz0, kz0+nr) of the slab are transformed together by the whole CTA:
// row r, component c lives in the row buffers at ro + (3 r + c) py.

// y stage 0 fused with the read from (INV: write to) the slab, zero padded;
// the y twiddles at `twy` are staged by stage_twiddles0 (two-stage plans).
template <typename T, int G, typename PY, bool INV, bool HALF = false>
__device__ __forceinline__ void rows_stage0(typename C2<T>::t* S, int kz0, int nr, int q, int by, int ro,
                                            int py, int twy, int tid, int bar) {
  typedef typename C2<T>::t T2;
  constexpr int R = PY::r[0], S0 = PY::N / R;
  T2* sm = smem_at<T>(0);
  const int total = nr * 3 * S0;
  for (int it = tid; it < total; it += G) {
    const int j = it % S0, rc = it / S0;
    const int row = rc / 3, c = rc - 3 * row;
    const int srow = (kz0 + row) * q + c * by;
    const int rb = ro + rc * py;
    T2 v[R];
    if (!INV) {
#pragma unroll
      for (int m = 0; m < R; m++) {
        const int yy = j + m * S0;
        v[m] = (HALF ? m < R / 2 : yy < by) ? S[srow + yy] : czero<T2>();
      }
      butterfly0<PY, false>(v, j, sm + twy);
#pragma unroll
      for (int m = 0; m < R; m++) sm[rb + j + m * S0] = v[m];
    } else {
#pragma unroll
      for (int m = 0; m < R; m++) v[m] = sm[rb + j + m * S0];
      butterfly0<PY, true>(v, j, sm + twy);
#pragma unroll
      for (int m = 0; m < R; m++) {
        const int yy = j + m * S0;
        if (HALF ? m < R / 2 : yy < by) S[srow + yy] = v[m];
      }
    }
  }
  group_sync<G>(bar);
}

// last forward y stage, D-hat multiply, first inverse y stage, in registers
// (kz positions kz0.. map to frequencies through PZ).
template <typename T, int G, typename PY, typename PZ>
__device__ __forceinline__ void rows_dmul(int kz0, int nr, int ro, int py,
                                          const typename C2<T>::t* __restrict__ dc, const MvGeom& g, int kx,
                                          int tid, int bar) {
  typedef typename C2<T>::t T2;
  constexpr int K = PY::K;
  constexpr int R = PY::r[K - 1];
  constexpr int NB = PY::N / R;
  T2* sm = smem_at<T>(0);
  // A thread reads R contiguous elements of each component.  With even R,
  // neighbouring butterflies of one row are 2R words apart and share banks
  // (16-way for R = 8), so neighbouring threads take neighbouring rows
  // instead (3 py complex apart); with odd R they take neighbouring
  // butterflies.
  constexpr bool ROW_FAST = R % 2 == 0;
  for (int it = tid; it < nr * NB; it += G) {
    const int t = ROW_FAST ? it / nr : it % NB, row = ROW_FAST ? it - t * nr : it / NB;
    const int kz = PZ::freq_of(kz0 + row);
    const int base = ro + 3 * row * py + t * R;
    T2 v0[R], v1[R], v2[R];
#pragma unroll
    for (int m = 0; m < R; m++) {
      v0[m] = sm[base + m];
      v1[m] = sm[base + py + m];
      v2[m] = sm[base + 2 * py + m];
    }
    DftN<R, false, T2>::run(v0);
    DftN<R, false, T2>::run(v1);
    DftN<R, false, T2>::run(v2);
#pragma unroll
    for (int m = 0; m < R; m++) {
      T2 d[6];
      load_dhat<T>(dc, g.Gx, g.Gy, g.Gz, kx, PY::freq_of(t * R + m), kz, d);
      dmul(d, v0[m], v1[m], v2[m]);
    }
    DftN<R, true, T2>::run(v0);
    DftN<R, true, T2>::run(v1);
    DftN<R, true, T2>::run(v2);
#pragma unroll
    for (int m = 0; m < R; m++) {
      sm[base + m] = v0[m];
      sm[base + py + m] = v1[m];
      sm[base + 2 * py + m] = v2[m];
    }
  }
  group_sync<G>(bar);
}

// GR = 2: the CTA works as two groups of NT/2 threads with their own named
// barriers.  The z passes split the columns between the groups, the y pass
// gives each group every other batch of kz rows (in its own half of the row
// buffers), and only the two hand-overs between the z and y passes are
// CTA-wide: a group that waits at its barrier leaves the SM to the other
// group.  Every butterfly does the same arithmetic as with GR = 1, so the
// results are identical.
template <typename T, int NT, typename PZ, typename PY, bool HALF = false, int GR = 1>
__global__ void __launch_bounds__(NT, 1) k_yz_p(typename C2<T>::t* __restrict__ xhat,
                                             const typename C2<T>::t* __restrict__ dc, MvGeom g,
                                             YzGeom y, FftPlanDev pz, FftPlanDev pyp,
                                             const KrylovState* __restrict__ st, int mvskip) {
  static_assert(PY::K >= 2 && PZ::K >= 2, "tuned plans have at least two stages");
  static_assert(!HALF || (PY::r[0] % 2 == 0 && PZ::r[0] % 2 == 0), "HALF needs an even first radix");
  typedef typename C2<T>::t T2;
  const int kx = blockIdx.x, b = blockIdx.y;  // kx: position after the x transform
  if (rhs_idle(st, b, mvskip)) return;
  const int soff = yz_slab_off(g), roff = yz_rows_off(g, y);
  T2* S = smem_at<T>(soff);
  T2* plane = xhat + ((size_t)b * g.Gx + kx) * 3 * g.nlines;
  stage_twiddles<T, NT>(0, pz);
  stage_twiddles0<T, NT, PY>(g.Gz, pyp);  // only y stage 0 has twiddles in two-stage plans
  __syncthreads();
  constexpr int G = NT / GR;
  const int grp = GR == 1 ? 0 : (int)threadIdx.x / G;
  const int tid = (int)threadIdx.x - grp * G;
  const int bar = GR == 1 ? 0 : 1 + grp;
  const int w3 = 3 * g.by;
  const int l0 = grp * (w3 / GR), lw = grp == GR - 1 ? w3 - l0 : w3 / GR;  // this group's columns
  zp_first<T, G, PZ, HALF>(plane, soff, y.q, g.by, g.bz, 0, tid, l0, lw, bar);
  pstages<T, PZ, false, G, 1, PZ::K>(soff + l0, lw, 1, y.q, 0, tid, bar);
  if (GR > 1) __syncthreads();  // every column transformed before the rows
  {
    const int kxf = g.fx[kx];
    const int nrg = y.nrw / GR;  // rows per batch of a group
    const int rog = roff + grp * nrg * 3 * y.py;
    for (int kz0 = grp * nrg; kz0 < g.Gz; kz0 += GR * nrg) {  // kz: positions after the z transform
      const int nr = min(nrg, g.Gz - kz0);
      rows_stage0<T, G, PY, false, HALF>(S, kz0, nr, y.q, g.by, rog, y.py, g.Gz, tid, bar);
      pstages<T, PY, false, G, 1, PY::K - 1>(rog, 3 * nr, y.py, 1, g.Gz, tid, bar);
      rows_dmul<T, G, PY, PZ>(kz0, nr, rog, y.py, dc, g, kxf, tid, bar);
      pstages<T, PY, true, G, 1, PY::K - 1>(rog, 3 * nr, y.py, 1, g.Gz, tid, bar);
      rows_stage0<T, G, PY, true, HALF>(S, kz0, nr, y.q, g.by, rog, y.py, g.Gz, tid, bar);
    }
  }
  if (GR > 1) __syncthreads();  // every row back in the slab before the z inverse
  pstages<T, PZ, true, G, 1, PZ::K>(soff + l0, lw, 1, y.q, 0, tid, bar);
  zp_last<T, G, PZ, HALF>(plane, soff, y.q, g.by, g.bz, 0, tid, l0, lw);
}

// Split path rows with a compile-time y plan: each warp one kz row, copied
// into its row buffer (zero padded), then the fused pipeline, then back.
template <typename T, int NT, typename PY>
__global__ void __launch_bounds__(NT, 1) k_yrows_p(typename C2<T>::t* __restrict__ zbuf,
                                                const typename C2<T>::t* __restrict__ dc, MvGeom g,
                                                YzGeom y, FftPlanDev pyp,
                                                const KrylovState* __restrict__ st, int mvskip) {
  typedef typename C2<T>::t T2;
  const int kx = blockIdx.y, b = blockIdx.z;
  if (rhs_idle(st, b, mvskip)) return;
  const int kz0 = blockIdx.x * y.nrw;
  const int nr = min(y.nrw, g.Gz - kz0);
  T2* base = zbuf + ((size_t)b * g.Gx + kx) * 3 * (size_t)g.Gz * g.by;
  const size_t cs = (size_t)g.Gz * g.by;
  const int roff = g.Gy;
  T2* R = smem_at<T>(roff);
  stage_twiddles<T, NT>(0, pyp);
  for (int i = threadIdx.x; i < nr * 3 * g.Gy; i += NT) {
    const int rc = i / g.Gy, yy = i - rc * g.Gy;
    const int row = rc / 3, c = rc - 3 * row;
    R[rc * y.py + yy] = yy < g.by ? base[c * cs + (size_t)(kz0 + row) * g.by + yy] : czero<T2>();
  }
  __syncthreads();
  {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < nr) {
      const int ro = roff + w * 3 * y.py;
      pstages<T, PY, false, 32, 0, PY::K - 1>(ro, 3, y.py, 1, 0, lane);
      row_dmul_stage<T, PY>(ro, y.py, dc, g, g.fx[kx], g.fz[kz0 + w], lane);
      pstages<T, PY, true, 32, 0, PY::K - 1>(ro, 3, y.py, 1, 0, lane);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < nr * 3 * g.by; i += NT) {
    const int rc = i / g.by, yy = i - rc * g.by;
    const int row = rc / 3, c = rc - 3 * row;
    base[c * cs + (size_t)(kz0 + row) * g.by + yy] = R[rc * y.py + yy];
  }
}

}  // namespace dda
