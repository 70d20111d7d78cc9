// matvec_kernels.cuh -- the FFT-convolution matvec of the DDA system
//   y = x + sqrt(cc) . IFFT3( D-hat . FFT3( pad( sqrt(cc) . x ) ) )
// (GpuMatVec<T>::apply, DDA/GpuMatVec.cpp:144-431; CPU twin
// DDA/MatVecCpu.cpp:67-150) as three fused passes over HBM:
//
//   k_xfwd : scatter sqrt(cc).x into a shared-memory tile of grid lines along
//            x (initXMatrix, DDA/GpuMatVecInst.cl:31-61), forward FFT along x,
//            store the x-spectrum plane-major: xhat[b][kx][c][z][y].
//   k_yz   : one kx plane per CTA, resident in shared memory: forward FFT
//            along z (zero padded bz -> Gz), then per kz row forward FFT along
//            y (by -> Gy), the symmetric 3x3 D-hat multiply (innerLoop,
//            DDA/GpuMatVecInst.cl:104-121), inverse FFT along y, inverse FFT
//            along z, store back.  Replaces the four GpuTransposePlan calls
//            and the slab loop of DDA/GpuMatVec.cpp:226-363.
//   k_xinv : inverse FFT along x, gather, y = sqrt(cc).X + x and the optional
//            Krylov dot products of the result (createResVec,
//            DDA/GpuMatVecInst.cl:63-102).
//
// When a kx plane does not fit in shared memory, k_yz is replaced by
// k_fft_cols (z forward) -> k_yrows (y forward, D-hat, y inverse) ->
// k_fft_cols (z inverse) through a plane buffer zbuf[b][kx][c][kz][y].
//
// D-hat is stored as the first octant [kx<=Gx/2][kz<=Gz/2][ky<=Gy/2][6]: the
// Green's tensor is even in every axis on the diagonal and odd in the two
// axes of an off-diagonal component, and so is its DFT.
#pragma once

#include "fft_engine.cuh"
#include "fft_plan.cuh"
#include "reduce.cuh"
#include "krylov_ops.cuh"

namespace dda {

struct MvGeom {
  int Gx, Gy, Gz;
  int bx, by, bz;
  int nv, nvs;
  int nlines;  // by*bz
  int nmat;
  int tl;      // grid lines per k_xfwd / k_xinv tile
  int pitchx;  // shared row pitch of those tiles (Gx + 1)
  // frequency held at each position after a forward FFT along x, y, z
  // (the transforms leave their output in digit-reversed order)
  const int* fx;
  const int* fy;
  const int* fz;
};

// D-hat at (kx, ky, kz) from the octant store.
template <typename T>
__device__ __forceinline__ void load_dhat(const typename C2<T>::t* __restrict__ dc, int Gx, int Gy,
                                          int Gz, int kx, int ky, int kz,
                                          typename C2<T>::t d[6]) {
  typedef typename C2<T>::t T2;
  const int hx = Gx / 2 + 1, hy = Gy / 2 + 1, hz = Gz / 2 + 1;
  const bool fx = kx > Gx / 2, fy = ky > Gy / 2, fz = kz > Gz / 2;
  const int ax = fx ? Gx - kx : kx, ay = fy ? Gy - ky : ky, az = fz ? Gz - kz : kz;
  const T2* p = dc + ((size_t)(ax * hz + az) * hy + ay) * 6;
#pragma unroll
  for (int i = 0; i < 6; i++) d[i] = p[i];
  if (fx != fy) { d[1].x = -d[1].x; d[1].y = -d[1].y; }  // xy: odd in x and y
  if (fx != fz) { d[2].x = -d[2].x; d[2].y = -d[2].y; }  // xz
  if (fy != fz) { d[4].x = -d[4].x; d[4].y = -d[4].y; }  // yz
  (void)hx;
}

// y = D x for the symmetric 3x3 matrix (xx, xy, xz, yy, yz, zz)
// (Math/SymMatrix3.hpp:86-92).
template <typename T2>
__device__ __forceinline__ void dmul(const T2 d[6], T2& a, T2& b, T2& c) {
  T2 x = a, y = b, z = c;
  a = cadd(cadd(cmul(d[0], x), cmul(d[1], y)), cmul(d[2], z));
  b = cadd(cadd(cmul(d[1], x), cmul(d[3], y)), cmul(d[4], z));
  c = cadd(cadd(cmul(d[2], x), cmul(d[4], y)), cmul(d[5], z));
}

// True when right-hand side b needs no work: solved or failed, or (mvskip)
// the BiCGStab half-step exit made the second matvec unnecessary.
__device__ __forceinline__ bool rhs_idle(const KrylovState* st, int b, int mvskip) {
  return st && (st[b].done || (mvskip && st[b].skipmv));
}

// Shared-memory layout of k_xfwd / k_xinv (offsets in complex elements):
//   [0, Gx)            twiddles of the x transform
//   [Gx, Gx + nmat)    sqrt(cc) of component c per material
//   [xtile, ...)       tile of tl grid lines, pitch pitchx = Gx + 1
__host__ __device__ inline int x_tile_off(const MvGeom& g) { return g.Gx + g.nmat; }

// Grid lines per x tile, at most.
constexpr int kXTileMax = 64;
// Global loads a thread of the x passes issues before it waits for the first
// of them: a tile's loads are independent, and with three CTAs per SM one
// load per thread at a time leaves HBM latency uncovered.
constexpr int kXBatch = 8;

// Line within the tile of CSR entry j: the largest l < nl with soff[l] <= j
// (soff: the tile's nl + 1 line offsets; empty lines are passed over).
__device__ __forceinline__ int tile_line(const uint32_t* soff, int nl, uint32_t j) {
  int l = 0;
#pragma unroll
  for (int step = kXTileMax / 2; step > 0; step >>= 1)
    if (l + step <= nl && soff[l + step] <= j) l += step;
  return l;
}

// Element i = kx nl + l of a tile's spectrum, walked by one thread in steps
// of NT without a division per element.
template <int NT>
struct TileWalk {
  int kx, l, dkx, dl;
  __device__ __forceinline__ TileWalk(int nl) {
    kx = threadIdx.x / nl;
    l = threadIdx.x - kx * nl;
    dkx = NT / nl;
    dl = NT - dkx * nl;
  }
  __device__ __forceinline__ void next(int nl) {
    l += dl;
    kx += dkx;
    if (l >= nl) {
      l -= nl;
      kx++;
    }
  }
};

// A solver step whose result is the next matvec's argument, run in
// k_xfwd's load instead of a pass of its own: the argument is computed from
// the solver's vectors, written back for the later steps and transformed.
// The linear combinations are the reference's (bo = -beta omega, mAlpha =
// -alpha, from the device state).
enum XPreOp {
  XP_NONE = 0,
  XP_BIS_P,   // out = first ? v2 : out beta + v1 bo + v2   (p, v, r)   DDA/BicgStab.cpp:88
  XP_BIS_S,   // out = v1 mAlpha + v2; n = |out|^2          (s, v, r)   DDA/BicgStab.cpp:96
  XP_BICG_P,  // out = first ? v1 : out beta + v1           (p, r)      DDA/BicgCs.cpp:73
  XP_CGNR_P,  // out = out beta + v1                        (p, A^H r)  DDA/Cgnr.cpp:62
};
struct XPre {
  int op;
  int first;         // iteration 0 variant
  void* out;         // the matvec argument (vector precision)
  const void* v1;
  const void* v2;
  KrylovStep step;   // sums over out, finalised by the last CTA (XP_BIS_S)
};

__device__ __forceinline__ bool xpre_reads_out(int op, int first) {
  return op == XP_CGNR_P || ((op == XP_BIS_P || op == XP_BICG_P) && !first);
}
__device__ __forceinline__ bool xpre_reads_v1(int op, int first) { return !(op == XP_BIS_P && first); }
__device__ __forceinline__ bool xpre_reads_v2(int op) { return op == XP_BIS_P || op == XP_BIS_S; }

template <typename A2>
__device__ __forceinline__ A2 xpre_value(int op, int first, A2 p, A2 v1, A2 v2, A2 beta, A2 bo, A2 mAlpha) {
  switch (op) {
    case XP_BIS_P: return first ? v2 : cadd(cadd(cmul(p, beta), cmul(v1, bo)), v2);
    case XP_BIS_S: return cadd(cmul(v1, mAlpha), v2);
    case XP_BICG_P: return first ? v1 : cadd(cmul(p, beta), v1);
    default: return cadd(cmul(p, beta), v1);
  }
}

// ------------------------------------------------------------ k_xfwd ----
// grid (ceil(nlines/tl), 3, nrhs).  PX: compile-time plan of the x
// transform, or void for the runtime-planned engine.  A2: the vectors'
// element type (double2 with T = float: FP64 Krylov vectors, rounded to FP32
// as they are read).  PRE: the argument is pre.op's result (XPreOp), which
// this kernel writes back, padding included.
template <typename T, int NT, typename PX = void, typename A2 = typename C2<T>::t, int PRE = 0>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) k_xfwd(const A2* __restrict__ arg,
                                             typename C2<T>::t* __restrict__ xhat,
                                             const uint32_t* __restrict__ line_off,
                                             const uint32_t* __restrict__ dip,
                                             const uint32_t* __restrict__ perm,
                                             const typename C2<T>::t* __restrict__ ccs, int conj,
                                             MvGeom g, FftPlanDev px, KrylovState* st, int mvskip, XPre pre) {
  typedef typename C2<T>::t T2;
  const int b = blockIdx.z, c = blockIdx.y;
  // the BiCGStab s step decides the half-step exit itself: it runs whenever
  // the right-hand side is not done
  if (rhs_idle(st, b, PRE ? 0 : mvskip)) return;
  const int toff = x_tile_off(g);
  T2* scc = smem_at<T>(g.Gx);
  T2* sm = smem_at<T>(toff);
  const int L0 = blockIdx.x * g.tl;
  const int nl = min(g.tl, g.nlines - L0);
  __shared__ uint32_t soff[kXTileMax + 1];
  stage_twiddles<T, NT>(0, px);
  for (int i = threadIdx.x; i < g.nmat; i += NT) scc[i] = ccs[((size_t)b * g.nmat + i) * 3 + c];
  for (int i = threadIdx.x; i <= nl; i += NT) soff[i] = line_off[L0 + i];
  for (int i = threadIdx.x; i < nl * g.pitchx; i += NT) sm[i] = czero<T2>();
  __syncthreads();
  // the tile's dipoles are one contiguous CSR range: every thread takes
  // entries of it independently, so many loads are in flight at once
  const size_t voff = ((size_t)b * 3 + c) * g.nvs;
  const A2* a = arg + voff;
  A2* po = PRE ? reinterpret_cast<A2*>(pre.out) + voff : nullptr;
  const A2* p1 = PRE && pre.v1 ? reinterpret_cast<const A2*>(pre.v1) + voff : nullptr;
  const A2* p2 = PRE && pre.v2 ? reinterpret_cast<const A2*>(pre.v2) + voff : nullptr;
  A2 beta = czero<A2>(), bo = czero<A2>(), mAlpha = czero<A2>();
  if (PRE) {
    beta = cvt<A2>(st[b].beta);
    bo = cvt<A2>(st[b].bo);
    mAlpha = cvt<A2>(st[b].mAlpha);
  }
  const int op = pre.op, first = pre.first;
  const bool rd_out = PRE && xpre_reads_out(op, first), rd1 = PRE && xpre_reads_v1(op, first);
  const bool rd2 = PRE && xpre_reads_v2(op);
  RedSums acc = red_zero();
  // loads in flight per thread: fewer where each entry has three inputs or
  // wider elements, within the registers of three CTAs per SM
  constexpr int XB = PRE ? (sizeof(A2) == 16 && sizeof(T) == 4 ? 2 : 4)
                         : (sizeof(A2) > sizeof(T2) ? kXBatch / 2 : kXBatch);
  const uint32_t je = soff[nl];
  uint32_t j = soff[0] + threadIdx.x;
  int l = j < je ? tile_line(soff, nl, j) : 0;
  for (; j < je; j += XB * NT) {
    int o[XB];  // shared offset of entry j + u NT, -1 past the tile
    uint32_t d[XB], jj[XB];
#pragma unroll
    for (int u = 0; u < XB; u++) {
      const uint32_t ju = j + u * NT;
      o[u] = -1;
      if (ju < je) {
        while (soff[l + 1] <= ju) l++;  // stops at nl - 1: soff[nl] = je > ju
        d[u] = dip[ju];
        jj[u] = perm ? perm[ju] : ju;
        o[u] = l * g.pitchx;
      }
    }
    A2 v[XB], w1[XB], w2[XB];
#pragma unroll
    for (int u = 0; u < XB; u++)
      if (o[u] >= 0) {
        if (!PRE) {
          v[u] = a[jj[u]];
        } else {
          v[u] = rd_out ? po[jj[u]] : czero<A2>();
          w1[u] = rd1 ? p1[jj[u]] : czero<A2>();
          w2[u] = rd2 ? p2[jj[u]] : czero<A2>();
        }
      }
#pragma unroll
    for (int u = 0; u < XB; u++)
      if (o[u] >= 0) {
        if (PRE) {
          v[u] = xpre_value<A2>(op, first, v[u], w1[u], w2[u], beta, bo, mAlpha);
          po[jj[u]] = v[u];
          if (op == XP_BIS_S) acc.n += (double)v[u].x * v[u].x + (double)v[u].y * v[u].y;
        }
        T2 x = cvt<T2>(v[u]);
        if (conj) x.y = -x.y;
        sm[o[u] + (d[u] & 0xffffu)] = cmul(x, scc[d[u] >> 16]);
      }
  }
  if (PRE && blockIdx.x == 0)
    for (int i = g.nv + threadIdx.x; i < g.nvs; i += NT) po[i] = czero<A2>();
  __syncthreads();
  if constexpr (std::is_void<PX>::value) fft_lines<T, NT, false>(toff, nl, g.pitchx, 1, false, px, 0);
  else plines<T, PX, NT, false>(toff, nl, g.pitchx, 1, 0);
  T2* out = xhat + ((size_t)b * g.Gx * 3 + c) * g.nlines + L0;
  const size_t kstride = (size_t)3 * g.nlines;
  for (TileWalk<NT> w(nl); w.kx < g.Gx; w.next(nl)) out[w.kx * kstride + w.l] = sm[w.l * g.pitchx + w.kx];
  if (PRE && pre.step.op != KOP_NONE) {
    RedSums tot;
    const int part = blockIdx.y * gridDim.x + blockIdx.x;
    if (block_finish<NT>(acc, pre.step.red, b, part, tot) && threadIdx.x == 0)
      krylov_finalize(st[b], pre.step, tot);
  }
}

// ------------------------------------------------------------ k_xinv ----
// grid (ceil(nlines/tl), 3, nrhs).  Epilogue: res = conj?(sqrt(cc).X +
// conj?(arg)), padding nv..nvs zeroed, and optional sums over the result for
// the solver step `op` (finalised by the last CTA of each right-hand side).
// With FP64 vectors (A2 = double2, T = float) the convolution term is
// rounded in FP32 and the identity term added in FP64:
// res = arg + conj?(sqrt(cc).X).
template <typename T, int NT, typename PX = void, typename A2 = typename C2<T>::t>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 2 : 3) k_xinv(const A2* __restrict__ arg,
                                             A2* __restrict__ res,
                                             const typename C2<T>::t* __restrict__ xhat,
                                             const uint32_t* __restrict__ line_off,
                                             const uint32_t* __restrict__ dip,
                                             const uint32_t* __restrict__ perm,
                                             const typename C2<T>::t* __restrict__ ccs, int conj,
                                             MvGeom g, FftPlanDev px, KrylovState* st,
                                             KrylovStep step, int mvskip) {
  typedef typename C2<T>::t T2;
  const int b = blockIdx.z, c = blockIdx.y;
  if (rhs_idle(st, b, mvskip)) return;
  const int toff = x_tile_off(g);
  T2* scc = smem_at<T>(g.Gx);
  T2* sm = smem_at<T>(toff);
  const int L0 = blockIdx.x * g.tl;
  const int nl = min(g.tl, g.nlines - L0);
  __shared__ uint32_t soff[kXTileMax + 1];
  stage_twiddles<T, NT>(0, px);
  for (int i = threadIdx.x; i < g.nmat; i += NT) scc[i] = ccs[((size_t)b * g.nmat + i) * 3 + c];
  for (int i = threadIdx.x; i <= nl; i += NT) soff[i] = line_off[L0 + i];
  const T2* in = xhat + ((size_t)b * g.Gx * 3 + c) * g.nlines + L0;
  const size_t kstride = (size_t)3 * g.nlines;
  for (TileWalk<NT> w(nl); w.kx < g.Gx;) {
    T2 v[kXBatch];
    int o[kXBatch];  // shared offset, -1 past the tile
#pragma unroll
    for (int u = 0; u < kXBatch; u++) {
      o[u] = -1;
      if (w.kx < g.Gx) {
        v[u] = in[w.kx * kstride + w.l];
        o[u] = w.l * g.pitchx + w.kx;
      }
      w.next(nl);
    }
#pragma unroll
    for (int u = 0; u < kXBatch; u++)
      if (o[u] >= 0) sm[o[u]] = v[u];
  }
  __syncthreads();
  if constexpr (std::is_void<PX>::value) fft_lines<T, NT, true>(toff, nl, g.pitchx, 1, false, px, 0);
  else plines<T, PX, NT, true>(toff, nl, g.pitchx, 1, 0);
  const size_t voff = ((size_t)b * 3 + c) * g.nvs;
  const A2* a = arg + voff;
  A2* r = res + voff;
  const A2* w = step.w ? reinterpret_cast<const A2*>(step.w) + voff : nullptr;
  RedSums acc = red_zero();
  const uint32_t je = soff[nl];
  uint32_t j = soff[0] + threadIdx.x;
  int l = j < je ? tile_line(soff, nl, j) : 0;
  constexpr int U = kXBatch / 2;
  for (; j < je; j += U * NT) {
    int o[U];  // shared offset of entry j + u NT, -1 past the tile
    uint32_t d[U], jj[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t ju = j + u * NT;
      o[u] = -1;
      if (ju < je) {
        while (soff[l + 1] <= ju) l++;  // stops at nl - 1: soff[nl] = je > ju
        d[u] = dip[ju];
        jj[u] = perm ? perm[ju] : ju;
        o[u] = l * g.pitchx;
      }
    }
    A2 a0[U], wv[U];
#pragma unroll
    for (int u = 0; u < U; u++)
      if (o[u] >= 0) {
        a0[u] = a[jj[u]];
        if (w) wv[u] = w[jj[u]];
      }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (o[u] >= 0) {
        const T2 x = sm[o[u] + (d[u] & 0xffffu)];
        A2 y;
        if constexpr (std::is_same<A2, T2>::value) {
          T2 av = a0[u];
          if (conj) av.y = -av.y;
          y = cadd(cmul(x, scc[d[u] >> 16]), av);
          if (conj) y.y = -y.y;
        } else {
          T2 cv = cmul(x, scc[d[u] >> 16]);
          if (conj) cv.y = -cv.y;
          y = a0[u];
          y.x += cv.x;
          y.y += cv.y;
        }
        r[jj[u]] = y;
        if (step.op != KOP_NONE) acc = epilogue_terms<A2>(acc, y, a0[u], w ? wv[u] : a0[u], step.mode);
      }
  }
  if (blockIdx.x == 0)
    for (int i = g.nv + threadIdx.x; i < g.nvs; i += NT) r[i] = czero<A2>();
  if (step.op != KOP_NONE) {
    RedSums tot;
    const int part = blockIdx.y * gridDim.x + blockIdx.x;
    if (block_finish<NT>(acc, step.red, b, part, tot) && threadIdx.x == 0)
      krylov_finalize(st[b], step, tot);
  }
}

// -------------------------------------------------------------- k_yz ----
// One (rhs, kx) plane per CTA.  Shared memory (complex offsets):
//   [0, Gz) z twiddles, [Gz, Gz+Gy) y twiddles,
//   slab S[Gz][q] at Gz+Gy (row kz holds the three components' y < by),
//   row buffers R[nrw][3][py] after the slab.
struct YzGeom {
  int q;    // slab row pitch (>= 3 by, odd)
  int nrw;  // row buffers: warps that run rows (or rows per CTA pass)
  int py;   // row buffer pitch (Gy + 1)
};

__host__ __device__ inline int yz_slab_off(const MvGeom& g) { return g.Gz + g.Gy; }
__host__ __device__ inline int yz_rows_off(const MvGeom& g, const YzGeom& y) {
  return g.Gz + g.Gy + g.Gz * y.q;
}

// y forward FFT of the three components of one row (held at shared offset
// roff, pitch py, zero padded by -> Gy), D-hat multiply and y inverse FFT, by
// one warp.  kx and kz are frequencies; the y positions are mapped to
// frequencies through g.fy.
template <typename T>
__device__ __forceinline__ void warp_row(int roff, const typename C2<T>::t* __restrict__ dc,
                                         const MvGeom& g, int py, const FftPlanDev& pyp, int twy,
                                         int kx, int kz, int lane) {
  typedef typename C2<T>::t T2;
  fft_group<T, 32, false>(roff, 3, py, 1, false, g.Gy, pyp.packed, pyp.nst, twy);
  T2* R = smem_at<T>(roff);
  for (int p = lane; p < g.Gy; p += 32) {
    T2 d[6];
    load_dhat<T>(dc, g.Gx, g.Gy, g.Gz, kx, g.fy[p], kz, d);
    T2 a = R[p], b = R[py + p], c = R[2 * py + p];
    dmul(d, a, b, c);
    R[p] = a; R[py + p] = b; R[2 * py + p] = c;
  }
  __syncwarp();
  fft_group<T, 32, true>(roff, 3, py, 1, false, g.Gy, pyp.packed, pyp.nst, twy);
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_yz(typename C2<T>::t* __restrict__ xhat,
                                           const typename C2<T>::t* __restrict__ dc, MvGeom g,
                                           YzGeom y, FftPlanDev pz, FftPlanDev pyp,
                                           const KrylovState* __restrict__ st, int mvskip) {
  typedef typename C2<T>::t T2;
  const int kx = blockIdx.x, b = blockIdx.y;  // kx: position after the x transform
  if (rhs_idle(st, b, mvskip)) return;
  const int soff = yz_slab_off(g), roff = yz_rows_off(g, y);
  T2* S = smem_at<T>(soff);
  T2* plane = xhat + ((size_t)b * g.Gx + kx) * 3 * g.nlines;
  const int nb = g.by * g.bz;
  stage_twiddles<T, NT>(0, pz);
  stage_twiddles<T, NT>(g.Gz, pyp);
  for (int i = threadIdx.x; i < 3 * nb; i += NT) {
    const int c = i / nb, rem = i - c * nb;
    const int z = rem / g.by, yy = rem - z * g.by;
    S[z * y.q + c * g.by + yy] = plane[i];
  }
  const int w3 = 3 * g.by;
  for (int i = threadIdx.x; i < (g.Gz - g.bz) * w3; i += NT) {
    const int zz = i / w3;
    S[(g.bz + zz) * y.q + (i - zz * w3)] = czero<T2>();
  }
  __syncthreads();
  fft_lines<T, NT, false>(soff, w3, 1, y.q, true, pz, 0);
  {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kxf = g.fx[kx];
    if (w < y.nrw) {
      const int ro = roff + w * 3 * y.py;
      T2* R = smem_at<T>(ro);
      for (int kz = w; kz < g.Gz; kz += y.nrw) {  // kz: position after the z transform
        for (int c = 0; c < 3; c++)
          for (int yy = lane; yy < g.Gy; yy += 32)
            R[c * y.py + yy] = yy < g.by ? S[kz * y.q + c * g.by + yy] : czero<T2>();
        __syncwarp();
        warp_row<T>(ro, dc, g, y.py, pyp, g.Gz, kxf, g.fz[kz], lane);
        for (int c = 0; c < 3; c++)
          for (int yy = lane; yy < g.by; yy += 32) S[kz * y.q + c * g.by + yy] = R[c * y.py + yy];
        __syncwarp();
      }
    }
    __syncthreads();
  }
  fft_lines<T, NT, true>(soff, w3, 1, y.q, true, pz, 0);
  for (int i = threadIdx.x; i < 3 * nb; i += NT) {
    const int c = i / nb, rem = i - c * nb;
    const int z = rem / g.by, yy = rem - z * g.by;
    plane[i] = S[z * y.q + c * g.by + yy];
  }
}

// ----------------------------------------------- split path: k_yrows ----
// grid (ceil(Gz/nrw), Gx, nrhs) over zbuf[b][kx][c][kz][y] (y < by), kx and
// kz positions after the forward x and z transforms; each CTA runs nrw rows,
// one per warp.  Shared memory: y twiddles at 0, rows R[nrw][3][py] at Gy.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_yrows(typename C2<T>::t* __restrict__ zbuf,
                                              const typename C2<T>::t* __restrict__ dc,
                                              MvGeom g, YzGeom y, FftPlanDev pyp,
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
    if (w < nr) warp_row<T>(roff + w * 3 * y.py, dc, g, y.py, pyp, 0, g.fx[kx], g.fz[kz0 + w], lane);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < nr * 3 * g.by; i += NT) {
    const int rc = i / g.by, yy = i - rc * g.by;
    const int row = rc / 3, c = rc - 3 * row;
    base[c * cs + (size_t)(kz0 + row) * g.by + yy] = R[rc * y.py + yy];
  }
}

// ------------------------------------------- generic strided column FFT ----
// Transforms along the middle axis of arrays [batch][axis][inner] (inner
// contiguous).  Input axis length n_in <= n is zero padded, output keeps the
// first n_out <= n entries.  grid (ceil(inner/ti), nbatch).  Shared memory:
// twiddles at 0, tile [n][pitch] at n.
struct ColGeom {
  long long in_bs, in_as;    // input batch / axis strides (elements)
  long long out_bs, out_as;  // output batch / axis strides
  int inner, ti, pitch;      // inner extent, tile width, smem pitch
  int n_in, n_out;
  int batches_per_rhs;       // for skipping converged right-hand sides
};

template <typename T, int NT, typename PL = void>
__global__ void __launch_bounds__(NT, sizeof(T) == 8 ? 1 : 2) k_fft_cols(const typename C2<T>::t* in,
                                                 typename C2<T>::t* out, ColGeom cg,
                                                 FftPlanDev pl, int inverse,
                                                 const KrylovState* __restrict__ st, int mvskip) {
  typedef typename C2<T>::t T2;
  const long long batch = blockIdx.y;
  if (rhs_idle(st, (int)(batch / cg.batches_per_rhs), mvskip)) return;
  const int n = pl.n;
  T2* sm = smem_at<T>(n);
  const int i0 = blockIdx.x * cg.ti;
  const int ti = min(cg.ti, cg.inner - i0);
  stage_twiddles<T, NT>(0, pl);
  const T2* ib = in + batch * cg.in_bs + i0;
  for (int i = threadIdx.x; i < n * ti; i += NT) {
    const int e = i / ti, k = i - e * ti;
    sm[e * cg.pitch + k] = e < cg.n_in ? ib[e * cg.in_as + k] : czero<T2>();
  }
  __syncthreads();
  if constexpr (std::is_void<PL>::value) fft_lines_dir<T, NT>(n, ti, 1, cg.pitch, true, pl, 0, inverse != 0);
  else if (inverse) plines<T, PL, NT, true>(n, ti, 1, cg.pitch, 0);
  else plines<T, PL, NT, false>(n, ti, 1, cg.pitch, 0);
  T2* ob = out + batch * cg.out_bs + i0;
  for (int i = threadIdx.x; i < cg.n_out * ti; i += NT) {
    const int e = i / ti, k = i - e * ti;
    ob[e * cg.out_as + k] = sm[e * cg.pitch + k];
  }
}

// -------------------------------------------- generic contiguous row FFT ----
// grid (ceil(count/tl)); lines of length n at `stride` elements apart.
// Shared memory: twiddles at 0, tile [tl][pitch] at n.
template <typename T, int NT>
__global__ void __launch_bounds__(NT, 2) k_fft_rows(typename C2<T>::t* data, long long count,
                                                 long long stride, int tl, int pitch,
                                                 FftPlanDev pl, int inverse) {
  typedef typename C2<T>::t T2;
  const int n = pl.n;
  T2* sm = smem_at<T>(n);
  const long long l0 = (long long)blockIdx.x * tl;
  const int nl = (int)min((long long)tl, count - l0);
  stage_twiddles<T, NT>(0, pl);
  for (int i = threadIdx.x; i < nl * n; i += NT) {
    const int l = i / n, e = i - l * n;
    sm[l * pitch + e] = data[(l0 + l) * stride + e];
  }
  __syncthreads();
  fft_lines_dir<T, NT>(n, nl, pitch, 1, false, pl, 0, inverse != 0);
  for (int i = threadIdx.x; i < nl * n; i += NT) {
    const int l = i / n, e = i - l * n;
    data[(l0 + l) * stride + e] = sm[l * pitch + e];
  }
}

}  // namespace dda
